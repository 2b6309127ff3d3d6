"""lightbaker-b200: the bake passes of lightbaker (sun shadows as a distance field, ambient occlusion,
bounced light, an L1 irradiance volume) on B200, behind the reference's own `Gpu` boundary.

The Python surface mirrors the reference crate's (crates/lightbaker/src/lib.rs:8-23):

    gpu = Gpu.new()                                  # gpu/mod.rs:74
    buffers = gpu.scene(nodes, tris, materials, charts)   # gpu/mod.rs:129
    out = gpu.run(Pass.DIRECT, buffers, params, texels, light)   # gpu/mod.rs:140
    baked = bake(scene_bytes, gpu, cache=..., log=print)      # bake.rs:94
    baked.write()                                    # output.rs:95

Everything runs in the native library (lightbaker_b200/liblightbaker_b200.so): CUDA kernels for the
passes, C++ for the host pipeline. Importing this package without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import enum
import json
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import HIT, NODE, RAY, TEXEL, TRI, LightbakerError, Params

__all__ = ["Pass", "Gpu", "SceneBuffers", "Prepared", "prepare", "bake", "Bake", "encode_scene", "blake3",
           "rgb9e5", "rgb9e5_decode", "bc4_block", "Params", "NODE", "TRI", "TEXEL", "RAY", "HIT", "LightbakerError", "Transport",
           "transport"]


class Pass(enum.IntEnum):
    """crates/lightbaker/src/gpu/mod.rs:26-33"""
    DIRECT = 0
    GATHER = 1
    VOLUME = 2

    @property
    def width(self) -> int:
        return 4 if self == Pass.VOLUME else 1


class SceneBuffers:
    """The scene as the passes read it, on the device (gpu/mod.rs:65-71)."""

    def __init__(self, handle: int, gpu: "Gpu"):
        self._h = handle
        self._gpu = gpu

    def set_vertices(self, verts: np.ndarray | None) -> None:
        """The triangles' exact vertices ((n_tris, 9) or (n_tris, 3, 3) float32, in the uploaded order;
        `Prepared.verts`): every walk over this scene then uses the watertight triangle test. None: the
        shader's test again (lb_scene_set_vertices)."""
        if verts is None:
            N.check(N.lib().lb_scene_set_vertices(self._gpu.handle, self._h, None, 0), "lb_scene_set_vertices")
            return
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 9)
        N.check(N.lib().lb_scene_set_vertices(self._gpu.handle, self._h, N.ptr(v), len(v)), "lb_scene_set_vertices")

    def bvh8(self) -> tuple[np.ndarray, np.ndarray]:
        """The 8-wide BVH built on the device at upload (lb_scene_get_bvh8): nodes as (n, 20) uint32 words
        and triangles as (m, 12) uint32 words (e2.w: the triangle's index in the uploaded array)."""
        nn, nt = C.c_uint64(), C.c_uint64()
        lib = N.lib()
        N.check(lib.lb_scene_get_bvh8(self._gpu.handle, self._h, None, None, C.byref(nn), C.byref(nt)), "lb_scene_get_bvh8")
        nodes = np.zeros((nn.value, 20), np.uint32)
        tris = np.zeros((nt.value, 12), np.uint32)
        N.check(lib.lb_scene_get_bvh8(self._gpu.handle, self._h, N.ptr(nodes), N.ptr(tris), None, None),
                "lb_scene_get_bvh8")
        return nodes, tris

    def close(self) -> None:
        if self._h:
            N.lib().lb_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Gpu:
    """One CUDA device (gpu/mod.rs:57-63). `adapter` names it."""

    def __init__(self, handle: int, adapter: str):
        self._h = handle
        self.adapter = adapter

    @staticmethod
    def new(device: int = 0) -> "Gpu":
        buf = C.create_string_buffer(256)
        h = N.lib().lb_gpu_open(device, buf, 256)
        if not h:
            raise LightbakerError(N.last_error())
        return Gpu(h, buf.value.decode())

    def close(self) -> None:
        if self._h:
            N.lib().lb_gpu_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h

    def scene(self, nodes: np.ndarray, tris: np.ndarray, materials: np.ndarray, charts: np.ndarray) -> SceneBuffers:
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        tris = np.ascontiguousarray(tris, dtype=TRI)
        materials = np.ascontiguousarray(materials, dtype=np.float32).reshape(-1, 4)
        charts = np.ascontiguousarray(charts, dtype=np.float32).reshape(-1, 8)
        h = N.lib().lb_scene_upload(self._h, N.ptr(nodes), len(nodes), N.ptr(tris), len(tris), N.ptr(materials),
                                    len(materials), N.ptr(charts) if len(charts) else None, len(charts))
        if not h:
            raise LightbakerError(N.last_error())
        return SceneBuffers(h, self)

    def run(self, pass_: Pass, scene: SceneBuffers, params: Params, texels: np.ndarray,
            light: np.ndarray | None = None) -> np.ndarray:
        """Each item's results: an (n * width, 4) float32 array (gpu/mod.rs:140-196)."""
        pass_ = Pass(pass_)
        texels = np.ascontiguousarray(texels, dtype=TEXEL)
        n = len(texels)
        out = np.zeros((n * pass_.width, 4), dtype=np.float32)
        if light is None or len(light) == 0:
            light_arr, nl = None, 0
        else:
            light_arr = np.ascontiguousarray(light, dtype=np.float32).reshape(-1, 4)
            nl = len(light_arr)
        N.check(N.lib().lb_run(self._h, scene._h, int(pass_), C.byref(params), N.ptr(texels), n,
                               N.ptr(light_arr), nl, N.ptr(out)), "GPU")
        return out

    def trace(self, scene: SceneBuffers, rays: np.ndarray, any_hit: bool = False, seed: int = 0) -> np.ndarray:
        """trace() (trace.wgsl:83-130) for each ray of a RAY array: a HIT array (t = tmax and tri =
        0xffffffff where none). seed: the bits of params.reach[3] (lb_trace)."""
        rays = np.ascontiguousarray(rays, dtype=RAY)
        out = np.zeros(len(rays), HIT)
        N.check(N.lib().lb_trace(self._h, scene._h, N.ptr(rays), len(rays), int(bool(any_hit)),
                                 int(seed) & 0xffffffff, N.ptr(out)), "lb_trace")
        return out

    @property
    def stream(self) -> int:
        """The handle's cudaStream_t, as an integer (every pass is enqueued on it)."""
        return N.lib().lb_gpu_stream(self._h) or 0

    def sync(self) -> None:
        N.check(N.lib().lb_gpu_sync(self._h), "lb_gpu_sync")

    def run_async(self, pass_: Pass, scene: SceneBuffers, params: Params, items_ptr: int, n: int, base: int,
                  light_ptr: int, n_light: int, out_ptr: int) -> None:
        """A pass over device-resident items (device pointers), enqueued on `stream`, not waited for."""
        N.check(N.lib().lb_run_async(self._h, scene._h, int(pass_), C.byref(params), C.c_void_p(items_ptr), n,
                                     base, C.c_void_p(light_ptr), n_light, C.c_void_p(out_ptr)), "GPU")

    def transfer(self, reset: bool = False) -> tuple:
        """(host-to-device bytes, device-to-host bytes) this handle copied."""
        h, d = C.c_uint64(), C.c_uint64()
        N.check(N.lib().lb_get_transfer(self._h, C.byref(h), C.byref(d), int(reset)), "lb_get_transfer")
        return h.value, d.value

    def set_pass_kernel(self, kind: int) -> None:
        """0: one thread an item (as the shader); 1: one warp an item. Same results."""
        N.check(N.lib().lb_set_pass_kernel(self._h, int(kind)), "lb_set_pass_kernel")

    def set_ray_order(self, direct: int, gather: int) -> None:
        """The warp kernels' ray order (see include/lightbaker.h lb_set_ray_order). Same results."""
        N.check(N.lib().lb_set_ray_order(self._h, int(direct), int(gather)), "lb_set_ray_order")

    def set_warp_walk(self, on: bool) -> None:
        N.check(N.lib().lb_set_warp_walk(self._h, int(bool(on))), "lb_set_warp_walk")

    def set_fetch(self, on: bool) -> None:
        N.check(N.lib().lb_set_fetch(self._h, int(bool(on))), "lb_set_fetch")

    def set_refill(self, on: bool) -> None:
        """Lane refill in the warp kernels (occlusion and gather rays over the BVH2). Same results."""
        N.check(N.lib().lb_set_refill(self._h, int(on)), "lb_set_refill")

    def set_near(self, on: bool) -> None:
        """Leaf lists for the warp kernels' occlusion rays (BVH2). Same results."""
        N.check(N.lib().lb_set_near(self._h, int(on)), "lb_set_near")

    def set_register_cap(self, blocks: int) -> None:
        """0: the compiler's register budget; 3 or 4: registers capped for that many blocks an SM."""
        N.check(N.lib().lb_set_register_cap(self._h, int(blocks)), "lb_set_register_cap")

    def set_bvh(self, width: int) -> None:
        """The BVH the warp kernels walk: 2 (the reference's) or 8 (8-wide, compressed). Same results."""
        N.check(N.lib().lb_set_bvh(self._h, int(width)), "lb_set_bvh")

    def set_counting(self, on: bool) -> None:
        N.check(N.lib().lb_set_counting(self._h, int(on)), "lb_set_counting")

    def counters(self) -> dict:
        c = N.Counters()
        N.check(N.lib().lb_get_counters(self._h, C.byref(c)), "lb_get_counters")
        return {"rays": c.rays, "nodes": c.nodes, "tris": c.tris, "mats": c.mats}


class Prepared:
    """A scene read and laid out with the BVH, materials, charts and Params the passes read
    (bake.rs:94-120)."""

    def __init__(self, scene: bytes):
        self._h = N.lib().lb_prepare(scene, len(scene))
        if not self._h:
            raise LightbakerError(N.last_error())
        info = N.PreparedInfo()
        N.check(N.lib().lb_prepared_get_info(self._h, C.byref(info)), "lb_prepared_get_info")
        self.info = info
        self.params = info.params.copy()
        self.nodes = np.zeros(info.n_nodes, NODE)
        self.tris = np.zeros(info.n_tris, TRI)
        N.check(N.lib().lb_prepared_get_bvh(self._h, N.ptr(self.nodes), N.ptr(self.tris)), "bvh")
        self.materials = np.zeros((info.n_materials, 4), np.float32)
        if info.n_materials:
            N.check(N.lib().lb_prepared_get_materials(self._h, N.ptr(self.materials)), "materials")
        self.charts = np.zeros((info.n_charts, 8), np.float32)
        if info.n_charts:
            N.check(N.lib().lb_prepared_get_charts(self._h, N.ptr(self.charts)), "charts")
        # each BVH triangle's vertices as the scene holds them (for the watertight test)
        self.verts = np.zeros((info.n_tris, 9), np.float32)
        N.check(N.lib().lb_prepared_get_vertices(self._h, N.ptr(self.verts)), "vertices")
        self.tiles = []
        for t in range(info.n_tiles):
            rect = (C.c_uint32 * 4)()
            key = (C.c_int32 * 2)()
            N.check(N.lib().lb_prepared_get_tile(self._h, t, rect, key), "tile")
            self.tiles.append({"x": rect[0], "y": rect[1], "w": rect[2], "h": rect[3], "key": (key[0], key[1])})

    def layout(self) -> dict:
        """The layout as data (layout.rs:20-66): per tile its charts in order; per chart its frame (mesh,
        turned, corner and size in its tile, tile key, normal, axes u and v, extent min/max) and its
        triangles (indices into its mesh)."""
        L = N.lib()
        tiles = []
        for t in range(len(self.tiles)):
            n = L.lb_prepared_get_tile_charts(self._h, t, None, 0)
            a = np.zeros(n, np.uint32)
            L.lb_prepared_get_tile_charts(self._h, t, N.ptr(a), n)
            tiles.append(a)
        charts = []
        for c in range(self.info.n_charts):
            f = N.ChartFrame()
            n = L.lb_prepared_get_chart(self._h, c, C.byref(f), None, 0)
            tris = np.zeros(n, np.uint32)
            L.lb_prepared_get_chart(self._h, c, None, N.ptr(tris), n)
            charts.append({"mesh": f.mesh, "turned": bool(f.turned), "x": f.x, "y": f.y, "w": f.w, "h": f.h,
                           "tile": (f.tile[0], f.tile[1]), "normal": np.array(f.normal, np.float32),
                           "u": np.array(f.u, np.float32), "v": np.array(f.v, np.float32),
                           "min": np.array(f.min, np.float32), "max": np.array(f.max, np.float32), "tris": tris})
        return {"tile_charts": tiles, "charts": charts}

    def rasterize(self, t: int) -> np.ndarray:
        """raster.rs:39-100: tile t's texels, (h, w) records."""
        tile = self.tiles[t]
        out = np.zeros(tile["w"] * tile["h"], TEXEL)
        N.check(N.lib().lb_prepared_rasterize(self._h, t, N.ptr(out)), "rasterize")
        return out.reshape(tile["h"], tile["w"])

    def covered_texels(self, tiles=None) -> np.ndarray:
        """The direct pass's items: every covered texel of the given tiles, in tile order then row-major
        (bake.rs:149)."""
        parts = []
        for t in range(len(self.tiles)) if tiles is None else tiles:
            tx = self.rasterize(t).reshape(-1)
            parts.append(tx[tx["pos"][:, 3] > 0.5])
        return np.concatenate(parts) if parts else np.zeros(0, TEXEL)

    def close(self):
        if self._h:
            N.lib().lb_prepared_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prepare(scene: bytes) -> Prepared:
    return Prepared(scene)


@dataclass
class Stats:
    tiles: int
    tiles_baked: int
    texels_baked: int
    chunks: int
    chunks_baked: int
    seconds: float
    rays_direct: int
    rays_gather: int
    rays_volume: int
    t_layout: float
    t_direct: float
    t_bounces: float
    t_volume: float
    t_composite: float

    @property
    def rays(self) -> int:
        return self.rays_direct + self.rays_gather + self.rays_volume


class Bake:
    """A bake's results (bake.rs:36-47): `direct` (h, w, 2) field and occlusion, `indirect` (ih, iw, 3),
    `validity` (h, w), `volume` (probes, 4, 4) or None, `stats`. The results are in host memory when the
    bake returns (in the handle); each array is copied out of it on first access."""

    def __init__(self, handle: int):
        self._h = handle
        info = N.BakeInfo()
        N.check(N.lib().lb_bake_get_info(handle, C.byref(info)), "lb_bake_get_info")
        self.info = info
        w, h, iw, ih = info.width, info.height, info.indirect_width, info.indirect_height
        self.width, self.height, self.indirect_size = w, h, (iw, ih)
        self._arrays = {}
        if info.has_volume:
            self.volume_size = tuple(info.volume_size)
            self.volume_origin = tuple(info.volume_origin)
            self.volume_step = info.volume_step
        self.stats = Stats(info.tiles, info.tiles_baked, info.texels_baked, info.chunks, info.chunks_baked,
                           info.seconds, info.rays_direct, info.rays_gather, info.rays_volume, info.t_layout,
                           info.t_direct, info.t_bounces, info.t_volume, info.t_composite)

    def _array(self, name, shape, dtype, getter):
        a = self._arrays.get(name)
        if a is None:
            if not self._h:
                raise LightbakerError("the bake is closed")
            a = np.zeros(shape, dtype)
            if a.size:
                N.check(getter(self._h, N.ptr(a)), name)
            self._arrays[name] = a
        return a

    @property
    def direct(self) -> np.ndarray:
        return self._array("direct", (self.height, self.width, 2), np.float32, N.lib().lb_bake_get_direct)

    @property
    def indirect(self) -> np.ndarray:
        iw, ih = self.indirect_size
        return self._array("indirect", (ih, iw, 3), np.float32, N.lib().lb_bake_get_indirect)

    @property
    def validity(self) -> np.ndarray:
        return self._array("validity", (self.height, self.width), np.uint8, N.lib().lb_bake_get_validity)

    @property
    def volume(self):
        if not self.info.has_volume:
            return None
        nx, ny, nz = self.volume_size
        return self._array("volume", (nx * ny * nz, 4, 4), np.float32, N.lib().lb_bake_get_volume)

    @property
    def charts(self) -> np.ndarray:
        return self._array("charts", (self.info.n_charts, 8), np.float32, N.lib().lb_bake_get_charts)

    @property
    def tri_charts(self) -> np.ndarray:
        return self._array("tri_charts", (self.info.n_triangles,), np.uint32, N.lib().lb_bake_get_tri_charts)

    @property
    def device_encoded(self) -> bool:
        """Whether the file's encodings (BC5, RGB9E5, probe bytes) were made on the device."""
        return bool(N.lib().lb_bake_device_encoded(self._h))

    def write(self) -> bytes:
        """The .lbake file (output.rs:95-154)."""
        p = C.POINTER(C.c_uint8)()
        n = C.c_size_t()
        N.check(N.lib().lb_bake_write(self._h, C.byref(p), C.byref(n)), "lb_bake_write")
        try:
            return C.string_at(p, n.value)
        finally:
            N.lib().lb_free(p)

    def close(self):
        if self._h:
            N.lib().lb_bake_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Exchange:
    """How the ranks of a bake split over processes add up what each baked (lb_exchange): element-wise sums of
    32-bit words over a torch.distributed process group (gloo for host memory; NCCL: host memory is staged
    through the device). Every rank bakes its share of the tiles and gets the whole bake."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self._dist, self._group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._cb = N.SUM_CB(self._sum)
        self.struct = N.Exchange(None, self.rank, self.world, self._cb)

    def _sum(self, ctx, data, count, device):
        import torch
        try:
            if device:
                t = torch.as_tensor(_DeviceWords(data, count), device="cuda")
                torch.cuda.synchronize()
                self._dist.all_reduce(t, group=self._group)
                torch.cuda.synchronize()
                return 0
            a = np.ctypeslib.as_array(C.cast(data, C.POINTER(C.c_int32)), shape=(count,))
            t = torch.from_numpy(a)
            if self._dist.get_backend(self._group) == "nccl":
                g = t.cuda()
                self._dist.all_reduce(g, group=self._group)
                t.copy_(g.cpu())
            else:
                self._dist.all_reduce(t, group=self._group)
            return 0
        except Exception:
            return 1


class _DeviceWords:
    """A device buffer of 32-bit words as __cuda_array_interface__ (for torch.as_tensor)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def _options(cache, log, autotune=False, trace_every_bounce=False, watertight=False, exchange=None):
    opts = N.BakeOptions()
    opts.cache_dir = str(cache).encode() if cache else None
    opts.autotune = int(bool(autotune))
    opts.trace_every_bounce = int(bool(trace_every_bounce))
    opts.watertight = int(bool(watertight))
    if exchange is not None:
        opts.exchange = C.pointer(exchange.struct)
    keep = None
    if log is not None:
        keep = N.LOG_CB(lambda ctx, line: log(line.decode("utf-8", "replace")))
        opts.log = keep
    return opts, keep


def bake(scene: bytes, gpu: Gpu, cache=None, log=None, watertight: bool = False, exchange: Exchange = None) -> Bake:
    """bake() (bake.rs:94-432): the whole bake with the passes on `gpu`; `watertight`: the watertight
    triangle test instead of the shader's; `exchange`: this process is one rank of a bake split over
    several (lb_bake_options)."""
    opts, keep = _options(cache, log, watertight=watertight, exchange=exchange)
    h = N.lib().lb_bake_run(gpu.handle, scene, len(scene), C.byref(opts))
    del keep
    if not h:
        raise LightbakerError(N.last_error())
    return Bake(h)


def bake_device(scene: bytes, gpu: Gpu, cache=None, log=None, autotune=False, trace_every_bounce=False,
                watertight=False, exchange: Exchange = None) -> Bake:
    """The device-resident bake: every dirty tile rebaked in one CUDA graph (same results as bake()).
    autotune: time the passes' ray order and grid on a sample of the texels first; trace_every_bounce:
    trace the gather rays in every bounce instead of evaluating the first bounce's records (lb_bake_options);
    exchange: this process is one rank of a bake split over several, which trace their shares of every pass
    and sum the passes' outputs on the device (every rank gets the whole bake)."""
    opts, keep = _options(cache, log, autotune, trace_every_bounce, watertight, exchange)
    h = N.lib().lb_bake_device(gpu.handle, scene, len(scene), C.byref(opts))
    del keep
    if not h:
        raise LightbakerError(N.last_error())
    return Bake(h)


class Plan:
    """A device bake in steps: the host work and the graph once (`Plan(scene, gpu)`), then `launch()`
    (the graph enqueued on gpu.stream; repeatable), `rays()`, `result()`."""

    def __init__(self, scene: bytes, gpu: Gpu, cache=None, log=None, autotune=False, trace_every_bounce=False,
                 watertight=False, exchange: Exchange = None):
        self._opts, self._keep = _options(cache, log, autotune, trace_every_bounce, watertight, exchange)
        self._exchange = exchange  # its callback lives as long as the plan
        self._h = N.lib().lb_plan_create(gpu.handle, scene, len(scene), C.byref(self._opts))
        if not self._h:
            raise LightbakerError(N.last_error())

    def launch(self) -> None:
        N.check(N.lib().lb_plan_launch(self._h), "lb_plan_launch")

    def rays(self) -> tuple:
        r = (C.c_uint64 * 3)()
        N.check(N.lib().lb_plan_rays(self._h, r), "lb_plan_rays")
        return r[0], r[1], r[2]

    def result(self) -> Bake:
        h = N.lib().lb_plan_result(self._h)
        if not h:
            raise LightbakerError(N.last_error())
        return Bake(h)

    def close(self) -> None:
        if self._h:
            N.lib().lb_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bake_with(scene: bytes, tracer: "N.Tracer", cache=None, log=None, exchange: Exchange = None) -> Bake:
    """The same bake with the passes on a caller's runner (an lb_tracer)."""
    opts, keep = _options(cache, log, exchange=exchange)
    h = N.lib().lb_bake_run_with(C.byref(tracer), scene, len(scene), C.byref(opts))
    del keep
    if not h:
        raise LightbakerError(N.last_error())
    return Bake(h)


def encode_scene(header: dict, positions: list) -> bytes:
    """Scene::write (scene.rs:164-181): an .lbscene from a header (the JSON object, camelCase keys) and
    each mesh's positions (float32, three vertices a triangle). The file is read back to validate it."""
    head = json.dumps(header, separators=(",", ":")).encode()
    arrs = [np.ascontiguousarray(p, dtype=np.float32).reshape(-1) for p in positions]
    ptrs = (C.c_void_p * max(1, len(arrs)))(*[a.ctypes.data for a in arrs])
    counts = (C.c_size_t * max(1, len(arrs)))(*[a.size for a in arrs])
    p = C.POINTER(C.c_uint8)()
    n = C.c_size_t()
    N.check(N.lib().lb_scene_encode(head, ptrs, counts, len(arrs), C.byref(p), C.byref(n)), "scene")
    try:
        return C.string_at(p, n.value)
    finally:
        N.lib().lb_free(p)


def bvh8_collapse(nodes: np.ndarray, tris: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The host's collapse of a BVH2 into the 8-wide BVH (lb_bvh8_collapse), in SceneBuffers.bvh8's form."""
    nodes = np.ascontiguousarray(nodes)
    tris = np.ascontiguousarray(tris)
    nn, nt = C.c_uint64(), C.c_uint64()
    lib = N.lib()
    N.check(lib.lb_bvh8_collapse(N.ptr(nodes), len(nodes), N.ptr(tris), len(tris), None, None, C.byref(nn),
                                 C.byref(nt)), "lb_bvh8_collapse")
    n8 = np.zeros((nn.value, 20), np.uint32)
    t8 = np.zeros((nt.value, 12), np.uint32)
    N.check(lib.lb_bvh8_collapse(N.ptr(nodes), len(nodes), N.ptr(tris), len(tris), N.ptr(n8), N.ptr(t8), None, None),
            "lb_bvh8_collapse")
    return n8, t8


def blake3(data: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    N.lib().lb_blake3(data, len(data), out)
    return bytes(out)


def rgb9e5(c) -> int:
    a = (C.c_float * 3)(*[float(x) for x in c])
    return int(N.lib().lb_rgb9e5(a))


def rgb9e5_decode(p: int):
    out = (C.c_float * 3)()
    N.lib().lb_rgb9e5_decode(p, out)
    return [out[0], out[1], out[2]]


def bc4_block(v) -> bytes:
    a = np.ascontiguousarray(v, dtype=np.uint8)
    assert a.size == 16
    out = np.zeros(8, np.uint8)
    N.lib().lb_bc4_block(N.ptr(a), N.ptr(out))
    return out.tobytes()


from .transport import Transport, transport  # noqa: E402
