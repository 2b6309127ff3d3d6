"""ORACLE — test infrastructure only: a whole bake on the CPU, restated from the reference's bake()
(crates/lightbaker/src/bake.rs:94-421, volume.rs:34-147), for a scene without a cache (every tile baked).

Independent of the product from the layout on: the scene file is read here (scene.rs:140-161), the
Params are built here (bake.rs:107-119), every tile is rasterised by oracle/bake_ref.cpp
(raster.rs:39-114), the passes run on the oracle's tracer (trace_ref.cpp), and the texel work between
them (per-tile post, gather selection, bounce filters, write_light, the volume's inside fill and the
fallback, the composite) is bake_ref.cpp's. The product supplies only what the bake reads before it
begins: the layout (charts and tiles, layout.rs:89-116), the BVH (bvh.rs:50-104) and the materials.
The charts' affines are recomputed here (layout.rs:76-85) and compared with the product's.

The result is the reference's Bake (bake.rs:36-47) as numpy arrays, plus the intermediate per-tile
arrays the tests compare stage by stage.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import struct

import numpy as np

from . import Scene, _p, lib, run

TEXEL = np.dtype([("pos", "<f4", 4), ("normal", "<f4", 4), ("dx", "<f4", 4), ("dy", "<f4", 4)])


class Params(C.Structure):
    """lb_params (include/lightbaker.h; the shader's uniform block, gpu/mod.rs:11-23)."""

    _fields_ = [("sun_dir", C.c_float * 4), ("sun_irr", C.c_float * 4), ("zenith", C.c_float * 4),
                ("horizon", C.c_float * 4), ("ground", C.c_float * 4), ("fallback", C.c_float * 4),
                ("counts", C.c_uint32 * 4), ("reach", C.c_float * 4), ("atlas", C.c_uint32 * 4)]


class Chart(C.Structure):
    _fields_ = [("u", C.c_float * 3), ("v", C.c_float * 3), ("min", C.c_float * 2), ("turned", C.c_uint32),
                ("x", C.c_uint32), ("y", C.c_uint32), ("id", C.c_uint32)]


class PostSettings(C.Structure):
    _fields_ = [("inside_share", C.c_float), ("ao_strength", C.c_float), ("ao_floor", C.c_float),
                ("ao_contrast", C.c_float), ("sdf_radius", C.c_float), ("sun_irradiance", C.c_float * 3),
                ("sun_dir", C.c_float * 3), ("grid", C.c_int), ("padding", C.c_uint32)]


def _declare():
    l = lib()
    if getattr(l, "_bake_declared", False):
        return l
    vp, sz, u32 = C.c_void_p, C.c_size_t, C.c_uint32
    l.or_chart_affine.restype = None
    l.or_chart_affine.argtypes = [vp, u32, u32, C.c_float, u32, vp]
    l.or_raster_tile.restype = None
    l.or_raster_tile.argtypes = [C.c_int, C.c_int, vp, sz, vp, vp, C.c_float, u32, vp]
    l.or_tile_post.restype = sz
    l.or_tile_post.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    l.or_gather_select.restype = None
    l.or_gather_select.argtypes = [C.c_int, C.c_int, vp, vp, u32, vp]
    l.or_bounce_tile.restype = sz
    l.or_bounce_tile.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, u32, u32, vp]
    l.or_write_light.restype = None
    l.or_write_light.argtypes = [u32, u32, C.c_int, C.c_int, u32, vp, vp, vp, vp]
    l.or_volume_fill.restype = None
    l.or_volume_fill.argtypes = [u32, u32, u32, vp]
    l.or_volume_fallback.restype = sz
    l.or_volume_fallback.argtypes = [C.c_int, C.c_int, vp, vp, u32, u32, u32, vp, C.c_float, vp, vp, vp, vp, vp,
                                     vp, vp, vp]
    l.or_composite.restype = None
    l.or_composite.argtypes = [u32, u32, u32, sz, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    l._bake_declared = True
    return l


# ---- the scene file (scene.rs:140-161) ----

def read_scene(data: bytes):
    """(header dict, per mesh float32 positions (3 * triangles, 3))."""
    if len(data) < 12 or data[:4] != b"LBSC":
        raise ValueError("not a lightbaker scene")
    version, n = struct.unpack_from("<II", data, 4)
    if version != 1:
        raise ValueError(f"scene format {version}")
    header = json.loads(data[12:12 + n])
    at = (12 + n + 3) & ~3
    positions = []
    for m in header["meshes"]:
        k = int(m["triangles"]) * 9
        positions.append(np.frombuffer(data, np.float32, k, at).reshape(-1, 3).copy())
        at = (at + k * 4 + 3) & ~3
    if at != len(data):
        raise ValueError("bytes after the last mesh")
    return header, positions


def f32(v) -> np.float32:
    """A JSON number as serde reads an f32 (through f64)."""
    return np.float32(float(v))


def _normalize(v):
    """glam Vec3::normalize: v * (1 / |v|), in f32."""
    v = np.asarray(v, np.float32)
    d = np.float32(np.float32(v[0] * v[0]) + np.float32(v[1] * v[1])) + np.float32(v[2] * v[2])
    r = np.float32(np.float32(1.0) / np.float32(np.sqrt(d)))
    return (v * r).astype(np.float32)


def make_params(header, atlas_width: int, atlas_height: int) -> Params:
    """bake.rs:104-119."""
    b, sun, sky = header["bake"], header["sun"], header["sky"]
    s = _normalize([f32(x) for x in sun["direction"]])
    g = int(np.float32(np.sqrt(np.float32(b["sunSamples"]))))
    rad = np.float32(f32(sun["radiusDeg"]) * np.float32(np.float32(math.pi) / np.float32(180.0)))
    zen = np.array([f32(x) for x in sky["zenith"]], np.float32)
    hor = np.array([f32(x) for x in sky["horizon"]], np.float32)
    avg = ((zen + hor) * np.float32(0.5)).astype(np.float32) * np.float32(math.pi)
    p = Params()
    libm = C.CDLL("libm.so.6")  # f32::tan is the C library's tanf
    libm.tanf.restype, libm.tanf.argtypes = C.c_float, [C.c_float]
    p.sun_dir[:] = [s[0], s[1], s[2], libm.tanf(float(rad))]
    p.sun_irr[:] = [*[f32(x) for x in sun["irradiance"]], 0.0]
    p.zenith[:] = [*zen, 0.0]
    p.horizon[:] = [*hor, 0.0]
    p.ground[:] = [*[f32(x) for x in sky["ground"]], min(np.float32(0.3), f32(b["aoReach"]))]
    p.fallback[:] = [*avg.astype(np.float32), 0.0]
    p.counts[:] = [g, int(b["aoRays"]), int(b["giRays"]), 0]
    p.reach[:] = [f32(b["aoReach"]), f32(b["giReach"]), np.float32(0.01), 0.0]
    p.atlas[:] = [atlas_width, atlas_height, 0, int(np.float32(f32(b["insideShare"])).view(np.uint32))]
    return p


def _chart_struct(c: dict, index: int) -> Chart:
    ch = Chart()
    ch.u[:] = list(c["u"])
    ch.v[:] = list(c["v"])
    ch.min[:] = list(c["min"])
    ch.turned, ch.x, ch.y, ch.id = int(c["turned"]), c["x"], c["y"], index
    return ch


def raster_tile(layout: dict, tile: dict, t: int, positions, density: float, padding: int) -> np.ndarray:
    """raster.rs:39-114 for tile t: (h * w) texels."""
    l = _declare()
    ids = layout["tile_charts"][t]
    charts = (Chart * max(1, len(ids)))()
    starts = np.zeros(len(ids) + 1, np.uint32)
    pos = []
    for k, ci in enumerate(ids):
        c = layout["charts"][int(ci)]
        charts[k] = _chart_struct(c, int(ci))
        p = positions[c["mesh"]].reshape(-1, 9)
        pos.append(p[c["tris"].astype(np.int64)])
        starts[k + 1] = starts[k] + len(c["tris"])
    pos = np.ascontiguousarray(np.concatenate(pos) if pos else np.zeros((0, 9), np.float32), np.float32)
    out = np.zeros(tile["w"] * tile["h"], TEXEL)
    l.or_raster_tile(tile["w"], tile["h"], charts, len(ids), _p(starts), _p(pos), float(density), padding, _p(out))
    return out


def chart_affines(layout: dict, tiles: list, density: float, padding: int) -> np.ndarray:
    """layout.rs:76-85 for every chart, in its tile."""
    l = _declare()
    out = np.zeros((len(layout["charts"]), 8), np.float32)
    for t, ids in enumerate(layout["tile_charts"]):
        for ci in ids:
            ch = _chart_struct(layout["charts"][int(ci)], int(ci))
            row = (C.c_float * 8)()
            l.or_chart_affine(C.byref(ch), tiles[t]["x"], tiles[t]["y"], float(density), padding, row)
            out[int(ci)] = list(row)
    return out


def volume_probes(vs: dict, tile_size: float):
    """volume.rs:36-77: the grid's size, and the probe items in chunk order (BTreeMap by tile key)."""
    vmin = [f32(x) for x in vs["min"]]
    vmax = [f32(x) for x in vs["max"]]
    step = f32(vs["step"])

    def n(a):
        q = np.float32(np.float32(vmax[a] - vmin[a]) / step)
        return max(int(math.floor(float(q) + 0.5)) + 1, 2)  # f32::round: half away from zero (q >= 0)

    nx, ny, nz = n(0), n(1), n(2)
    chunks: dict = {}
    ts = f32(tile_size)
    for k in range(nx * ny * nz):
        x = np.float32(vmin[0] + np.float32(np.float32(k % nx) * step))
        y = np.float32(vmin[1] + np.float32(np.float32(k // (nx * nz)) * step))
        z = np.float32(vmin[2] + np.float32(np.float32((k // nx) % nz) * step))
        key = (int(math.floor(float(np.float32(x / ts)))), int(math.floor(float(np.float32(z / ts)))))
        chunks.setdefault(key, []).append((k, x, y, z))
    items = []
    for key in sorted(chunks):
        items.extend(chunks[key])
    arr = np.zeros(len(items), TEXEL)
    for i, (k, x, y, z) in enumerate(items):
        arr[i]["pos"] = [x, y, z, 1.0]
        arr[i]["normal"] = [0.0, 1.0, 0.0, np.uint32(k).view(np.float32)]
    return (nx, ny, nz), np.array([it[0] for it in items], np.int64), arr


def build_bvh(scene: bytes, layout: dict):
    """bvh.rs:50-104 over the scene (oracle/bvh_ref.cpp), each triangle's chart taken from the layout:
    (nodes, tris) as raw records (32 and 48 bytes)."""
    l = lib()
    if not getattr(l, "_bvh_declared", False):
        vp, sz = C.c_void_p, C.c_size_t
        l.or_bvh_build.restype = sz
        l.or_bvh_build.argtypes = [vp, vp, sz, vp, vp, vp, vp, sz, vp, C.POINTER(sz)]
        l._bvh_declared = True
    header, positions = read_scene(scene)
    meshes = header["meshes"]
    first = np.zeros(len(meshes) + 1, np.uint32)
    for i, m in enumerate(meshes):
        first[i + 1] = first[i] + int(m["triangles"])
    pos = np.ascontiguousarray(np.concatenate([p.reshape(-1, 9) for p in positions]) if positions
                               else np.zeros((0, 9), np.float32), np.float32)
    mat = np.array([int(m["material"]) for m in meshes], np.uint32)
    casts = np.array([1 if m.get("casts", True) else 0 for m in header["materials"]], np.uint8)
    chart = np.full(int(first[-1]), 0xFFFFFFFF, np.uint32)
    for ci, c in enumerate(layout["charts"]):
        chart[int(first[c["mesh"]]) + c["tris"].astype(np.int64)] = ci
    n = max(1, int(first[-1]))
    nodes = np.zeros((2 * n + 1, 8), np.uint32)
    tris = np.zeros((n, 12), np.uint32)
    nt = C.c_size_t()
    nn = l.or_bvh_build(_p(pos), _p(first), len(meshes), _p(mat), _p(casts), _p(chart), _p(nodes), len(nodes),
                        _p(tris), C.byref(nt))
    return nodes[:nn], tris[:nt.value]


class OracleBake:
    """A whole bake (no cache) on the CPU. Attributes: `direct` (h, w, 2), `validity` (h, w), `indirect`
    (ih, iw, 3), `volume` (probes, 4, 4) or None; per tile `texels` (raster, before any move), `known`,
    `state`, `field`, `ao`, `direct_light`, `indirect_light`, `gathered`; `light` (the last light atlas),
    `params`, `affines`, `rays` (direct, gather, volume)."""

    def __init__(self, scene: bytes, prepared, threads: int = 0, watertight: bool = False):
        l = _declare()
        header, positions = read_scene(scene)
        lm, b = header["lightmap"], header["bake"]
        density, padding, ds = f32(lm["texelsPerMeter"]), int(lm["padding"]), int(lm["indirectDownscale"])
        info = prepared.info
        aw, ah = int(info.atlas_width), int(info.atlas_height)
        layout = prepared.layout()
        tiles = prepared.tiles
        self.params = P = make_params(header, aw, ah)
        self.affines = chart_affines(layout, tiles, density, padding)
        sc = Scene(prepared.nodes, prepared.tris, prepared.materials, self.affines,
                   prepared.verts if watertight else None)
        sun_dir = np.array(list(P.sun_dir)[:3], np.float32)
        irr = np.array([f32(x) for x in header["sun"]["irradiance"]], np.float32)
        st = PostSettings()
        st.inside_share, st.ao_strength = f32(b["insideShare"]), f32(b["aoStrength"])
        st.ao_floor, st.ao_contrast, st.sdf_radius = f32(b["aoFloor"]), f32(b["aoContrast"]), f32(b["sdfRadius"])
        st.sun_irradiance[:] = list(irr)
        st.sun_dir[:] = list(sun_dir)
        st.grid, st.padding = int(P.counts[0]), padding

        # raster (bake.rs:141-149)
        T = len(tiles)
        self.texels = [raster_tile(layout, tiles[t], t, positions, density, padding) for t in range(T)]
        work = [tx.copy() for tx in self.texels]
        cov = [tx["pos"][:, 3] > 0.5 for tx in work]
        chart = [np.where(c, tx["normal"][:, 3].view(np.uint32), np.uint32(0xffffffff)).astype(np.uint32)
                 for tx, c in zip(work, cov)]
        normal = [np.ascontiguousarray(tx["normal"][:, :3], np.float32) for tx in work]
        covered = np.concatenate([tx[c] for tx, c in zip(work, cov)]) if T else np.zeros(0, TEXEL)
        rec, cnt = run(0, sc, P, covered, None, threads)
        self.direct_records = rec
        rays = {"direct": cnt["rays"], "gather": 0, "volume": 0}

        # per tile post (bake.rs:197-275)
        self.valid, self.known, self.state, self.field, self.ao, self.direct_light = [], [], [], [], [], []
        k = 0
        for t in range(T):
            w, h = tiles[t]["w"], tiles[t]["h"]
            n = w * h
            va, kn, sa = (np.zeros(n, np.uint8) for _ in range(3))
            fi, ao, dl = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
            used = l.or_tile_post(w, h, _p(work[t]), _p(np.ascontiguousarray(rec[k:])), C.byref(st), _p(va), _p(kn),
                                  _p(sa), _p(fi), _p(ao), _p(dl))
            k += used
            for lst, a in zip((self.valid, self.known, self.state, self.field, self.ao, self.direct_light),
                              (va, kn, sa, fi, ao, dl)):
                lst.append(a)
        self.indirect_light = [np.zeros((tl["w"] * tl["h"], 3), np.float32) for tl in tiles]

        def write_all(light):
            for t in range(T):
                l.or_write_light(tiles[t]["x"], tiles[t]["y"], tiles[t]["w"], tiles[t]["h"], aw, _p(self.known[t]),
                                 _p(self.direct_light[t]), _p(self.indirect_light[t]), _p(light))

        light = np.zeros((aw * ah, 4), np.float32)
        write_all(light)

        # gather selection (bake.rs:286-298) and the bounces (:300-330)
        self.gathered = []
        for t in range(T):
            g = np.zeros(tiles[t]["w"] * tiles[t]["h"], np.uint8)
            l.or_gather_select(tiles[t]["w"], tiles[t]["h"], _p(self.valid[t]), _p(chart[t]), ds, _p(g))
            self.gathered.append(g)
        gather = np.concatenate([work[t][self.gathered[t] != 0] for t in range(T)]) if T else np.zeros(0, TEXEL)
        radius, rings = int(b["giFilter"]) * ds, padding + 2 * ds + 2
        for bounce in range(int(b["giBounces"])):
            res, c2 = run(1, sc, P, gather, light, threads)
            self.gather_out = res
            rays["gather"] += c2["rays"]
            k = 0
            for t in range(T):
                e = np.zeros((tiles[t]["w"] * tiles[t]["h"], 3), np.float32)
                k += l.or_bounce_tile(tiles[t]["w"], tiles[t]["h"], _p(chart[t]), _p(normal[t]), _p(self.gathered[t]),
                                      _p(np.ascontiguousarray(res[k:])), radius, rings, _p(e))
                self.indirect_light[t] = e
            write_all(light)
        self.light = light
        self.gather_items = gather
        self.work = work

        # the volume (volume.rs:34-122) and the fallback (bake.rs:337-359)
        self.volume = None
        vs = header.get("volume")
        if vs is not None:
            (nx, ny, nz), ids, items = volume_probes(vs, lm["tileSize"])
            Pv = Params()
            C.memmove(C.byref(Pv), C.byref(P), C.sizeof(Params))
            Pv.counts[2] = int(vs["rays"])
            res, c3 = run(2, sc, Pv, items, light, threads)
            rays["volume"] = c3["rays"]
            probes = np.zeros((nx * ny * nz, 16), np.float32)
            probes[ids] = res.reshape(-1, 16)
            self.volume_raw = probes.copy()
            l.or_volume_fill(nx, ny, nz, _p(probes))
            self.volume = probes.reshape(-1, 4, 4)
            self.volume_size = (nx, ny, nz)
            origin = (C.c_float * 3)(*[f32(x) for x in vs["min"]])
            self.fallback = 0
            for t in range(T):
                self.fallback += l.or_volume_fallback(
                    tiles[t]["w"], tiles[t]["h"], _p(work[t]), _p(probes), nx, ny, nz, origin,
                    float(f32(vs["step"])), (C.c_float * 3)(*irr), (C.c_float * 3)(*sun_dir), _p(self.known[t]),
                    _p(self.state[t]), _p(self.field[t]), _p(self.ao[t]), _p(self.direct_light[t]),
                    _p(self.indirect_light[t]))

        # the atlases (bake.rs:364-421)
        iw, ih = (aw + ds - 1) // ds, (ah + ds - 1) // ds
        rects = np.array([[tl["x"], tl["y"], tl["w"], tl["h"]] for tl in tiles], np.uint32).reshape(-1)

        def ptrs(arrs):
            return (C.c_void_p * max(1, T))(*[a.ctypes.data for a in arrs])

        self.direct = np.zeros((ah, aw, 2), np.float32)
        self.validity = np.zeros((ah, aw), np.uint8)
        self.indirect = np.zeros((ih, iw, 3), np.float32)
        l.or_composite(aw, ah, ds, T, _p(rects), ptrs(self.known), ptrs(self.state), ptrs(self.field), ptrs(self.ao),
                       ptrs(self.indirect_light), _p(self.direct), _p(self.validity), _p(self.indirect))
        self.rays = rays
