"""ORACLE — test infrastructure only: the checker, never the product.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package. It loads
oracle/liboracle.so, the CPU restatement of the reference's passes (oracle/trace_ref.cpp follows
crates/lightbaker/src/gpu/trace.wgsl; oracle/filter_ref.cpp follows crates/lightbaker/src/filter.rs),
and offers it as numpy functions and as an lb_tracer the product's bake can run on.

Parity status: numeric parity with the reference's WGSL is unpinned (the reference cannot run here:
no Rust toolchain, no graphics stack, and its tests hold no numeric golden vectors). The restatement is
pinned by the reference's property tests (tests/bake.rs:95-154), its encode known-answer tests
(encode.rs:150-180) and published BLAKE3 values; see tests/.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class Counters(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("nodes", C.c_uint64), ("tris", C.c_uint64), ("mats", C.c_uint64),
                ("overflows", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < max(
                p.stat().st_mtime for p in (HERE / "trace_ref.cpp", HERE / "filter_ref.cpp", HERE / "bake_ref.cpp",
                                            HERE / "bvh_ref.cpp", HERE / "oracle.h")):
            import importlib.util
            spec = importlib.util.spec_from_file_location("oracle_build", HERE / "build.py")
            m = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(m)
            m.build()
        l = C.CDLL(str(LIB))
        vp, sz = C.c_void_p, C.c_size_t
        l.or_run.restype = C.c_int
        l.or_run.argtypes = [C.c_int, vp, sz, vp, sz, vp, sz, vp, sz, vp, vp, sz, vp, sz, vp, C.c_int, C.POINTER(Counters)]
        l.or_trace.restype = C.c_int
        l.or_trace.argtypes = [C.c_int, vp, sz, vp, sz, vp, sz, vp, vp, vp, C.c_float, C.c_int, C.c_uint32,
                               C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.POINTER(C.c_int)]
        l.or_run_ex.restype = C.c_int
        l.or_run_ex.argtypes = l.or_run.argtypes + [vp]
        l.or_trace_ex.restype = C.c_int
        l.or_trace_ex.argtypes = l.or_trace.argtypes + [vp]
        l.or_trace_rays.restype = C.c_int
        l.or_trace_rays.argtypes = [C.c_int, vp, sz, vp, sz, vp, sz, vp, vp, sz, C.c_int, vp, vp, vp, vp, C.c_int]
        l.or_rays_ambiguous.restype = C.c_int
        l.or_rays_ambiguous.argtypes = [vp, sz, vp, sz, vp, sz, vp, vp, sz, C.c_double, vp, C.c_int]
        l.or_ray_ambiguous.restype = C.c_int
        l.or_ray_ambiguous.argtypes = [vp, sz, vp, sz, vp, sz, vp, vp, vp, C.c_float, C.c_uint32, C.c_double]
        l.or_item_rays.restype = sz
        l.or_item_rays.argtypes = [C.c_int, vp, vp, sz, C.c_uint32, vp, vp, vp, vp, vp, vp, sz]
        l.or_gather_records.restype = C.c_int
        l.or_gather_records.argtypes = [vp, sz, vp, sz, vp, sz, vp, sz, vp, vp, sz, sz, vp, C.c_int]
        l.or_pcg.restype = C.c_uint32
        l.or_pcg.argtypes = [C.c_uint32]
        l.or_rand.restype = C.c_float
        l.or_rand.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        l.or_radical.restype = C.c_float
        l.or_radical.argtypes = [C.c_uint32]
        l.or_sincos.restype = None
        l.or_sincos.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        l.or_smooth.restype = None
        l.or_smooth.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, C.c_int, vp]
        l.or_fill.restype = None
        l.or_fill.argtypes = [C.c_int, C.c_int, vp, vp, C.c_int, vp, C.c_int]
        l.or_sun_field.restype = None
        l.or_sun_field.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_int, C.c_float, vp]
        _lib = l
    return _lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Scene:
    """The scene arrays the passes read (the same ones lb_scene_upload takes); with `verts` (9 floats a
    triangle) the FP32 walk uses the watertight triangle test, as lb_scene_set_vertices switches the
    kernels."""

    def __init__(self, nodes, tris, materials, charts, verts=None):
        self.nodes = np.ascontiguousarray(nodes)
        self.tris = np.ascontiguousarray(tris)
        self.materials = np.ascontiguousarray(materials, dtype=np.float32).reshape(-1, 4)
        self.charts = np.ascontiguousarray(charts, dtype=np.float32).reshape(-1, 8)
        self.verts = None if verts is None else np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 9)

    @staticmethod
    def of(prepared, watertight: bool = False) -> "Scene":
        return Scene(prepared.nodes, prepared.tris, prepared.materials, prepared.charts,
                     prepared.verts if watertight else None)


def run(pass_: int, scene: Scene, params, items: np.ndarray, light=None, threads: int = 0):
    """Gpu::run on the CPU: (out (n * width, 4) float32, counters dict)."""
    items = np.ascontiguousarray(items)
    n = len(items)
    width = 4 if int(pass_) == 2 else 1
    out = np.zeros((n * width, 4), np.float32)
    if light is None or len(light) == 0:
        la, nl = None, 0
    else:
        la = np.ascontiguousarray(light, dtype=np.float32).reshape(-1, 4)
        nl = len(la)
    cnt = Counters()
    rc = lib().or_run_ex(int(pass_), _p(scene.nodes), len(scene.nodes), _p(scene.tris), len(scene.tris),
                         _p(scene.materials), len(scene.materials), _p(scene.charts) if len(scene.charts) else None,
                         len(scene.charts), C.byref(params), _p(items), n, _p(la), nl, _p(out), int(threads),
                         C.byref(cnt), _p(scene.verts))
    if rc != 0:
        raise RuntimeError(f"oracle run failed: {rc}")
    return out, {"rays": cnt.rays, "nodes": cnt.nodes, "tris": cnt.tris, "mats": cnt.mats,
                 "overflows": cnt.overflows}


def trace(scene: Scene, params, o, d, tmax, any_hit, ray, precision=32):
    t = C.c_double()
    tri = C.c_uint32()
    back = C.c_int()
    oa = (C.c_float * 3)(*o)
    da = (C.c_float * 3)(*d)
    lib().or_trace_ex(precision, _p(scene.nodes), len(scene.nodes), _p(scene.tris), len(scene.tris),
                      _p(scene.materials), len(scene.materials), C.byref(params), oa, da, float(tmax), int(any_hit),
                      int(ray) & 0xffffffff, C.byref(t), C.byref(tri), C.byref(back), _p(scene.verts))
    return t.value, tri.value, bool(back.value)


RAY = np.dtype([("o", "<f4", 3), ("tmax", "<f4"), ("d", "<f4", 3), ("key", "<u4")])


def rays_of(r) -> np.ndarray:
    """An item_rays dict as a RAY array (the layout of lb_ray)."""
    out = np.zeros(len(r["d"]), RAY)
    out["o"], out["d"], out["tmax"], out["key"] = r["o"], r["d"], r["tmax"], r["key"]
    return out


def trace_rays(scene: Scene, params, rays: np.ndarray, any_hit: bool, precision: int = 32, threads: int = 0):
    """trace() of every ray of a RAY array: (t float64, tri uint32, back bool) arrays."""
    rays = np.ascontiguousarray(rays, dtype=RAY)
    n = len(rays)
    t = np.zeros(n, np.float64)
    tri = np.zeros(n, np.uint32)
    back = np.zeros(n, np.int32)
    lib().or_trace_rays(int(precision), _p(scene.nodes), len(scene.nodes), _p(scene.tris), len(scene.tris),
                        _p(scene.materials), len(scene.materials), C.byref(params), _p(rays), n, int(bool(any_hit)),
                        _p(scene.verts) if precision == 32 else None, _p(t), _p(tri), _p(back), int(threads))
    return t, tri, back.astype(bool)


def rays_ambiguous(scene: Scene, params, rays: np.ndarray, eps: float = 1e-4, threads: int = 0) -> np.ndarray:
    """ray_ambiguous of every ray of a RAY array, as a bool array."""
    rays = np.ascontiguousarray(rays, dtype=RAY)
    out = np.zeros(len(rays), np.int32)
    lib().or_rays_ambiguous(_p(scene.nodes), len(scene.nodes), _p(scene.tris), len(scene.tris), _p(scene.materials),
                            len(scene.materials), C.byref(params), _p(rays), len(rays), float(eps), _p(out),
                            int(threads))
    return out.astype(bool)


def ray_ambiguous(scene: Scene, params, o, d, tmax, ray, eps=1e-5) -> bool:
    oa = (C.c_float * 3)(*o)
    da = (C.c_float * 3)(*d)
    return bool(lib().or_ray_ambiguous(_p(scene.nodes), len(scene.nodes), _p(scene.tris), len(scene.tris),
                                       _p(scene.materials), len(scene.materials), C.byref(params), oa, da,
                                       float(tmax), int(ray) & 0xffffffff, float(eps)))


def item_rays(pass_: int, params, item, index: int, pick: int = 0, cap: int = 4096):
    """The rays the shader casts for one item (see oracle.h: or_item_rays)."""
    o = np.zeros((cap, 3), np.float32)
    d = np.zeros((cap, 3), np.float32)
    tmax = np.zeros(cap, np.float32)
    anyh = np.zeros(cap, np.int32)
    key = np.zeros(cap, np.uint32)
    kind = np.zeros(cap, np.int32)
    it = np.ascontiguousarray(np.asarray(item).reshape(1))
    n = lib().or_item_rays(int(pass_), C.byref(params), _p(it), int(index), int(pick), _p(o), _p(d), _p(tmax),
                           _p(anyh), _p(key), _p(kind), cap)
    n = min(n, cap)
    return {"o": o[:n], "d": d[:n], "tmax": tmax[:n], "any": anyh[:n], "key": key[:n], "kind": kind[:n]}


def gather_records(scene: Scene, params, items: np.ndarray, n_light: int, threads: int = 0) -> np.ndarray:
    """Every gather ray's outcome (oracle.h: or_gather_records): (n, rays, 4) uint32 of kind (0 sky,
    1 back face, 2 surface), material, atlas texel (0xffffffff: none), bits of the direction's y."""
    items = np.ascontiguousarray(items)
    rays = int(params.counts[2])
    out = np.zeros((len(items), rays, 4), np.uint32)
    rc = lib().or_gather_records(_p(scene.nodes), len(scene.nodes), _p(scene.tris), len(scene.tris),
                                 _p(scene.materials), len(scene.materials),
                                 _p(scene.charts) if len(scene.charts) else None, len(scene.charts), C.byref(params),
                                 _p(items), len(items), int(n_light), _p(out), int(threads))
    if rc != 0:
        raise RuntimeError(f"oracle gather records failed: {rc}")
    return out


def pcg(v: int) -> int:
    return int(lib().or_pcg(v & 0xffffffff))


def rand(a: int, b: int, seed: int = 0) -> float:
    return float(lib().or_rand(a & 0xffffffff, b & 0xffffffff, seed & 0xffffffff))


def radical(i: int) -> float:
    return float(lib().or_radical(i & 0xffffffff))


def sincos(a: float):
    s = C.c_float()
    c = C.c_float()
    lib().or_sincos(float(a), C.byref(s), C.byref(c))
    return s.value, c.value


def smooth(w, h, chart, normal, v, valid, r):
    v = np.ascontiguousarray(v, np.float32).reshape(w * h, -1)
    N = v.shape[1]
    out = np.zeros_like(v)
    lib().or_smooth(w, h, _p(np.ascontiguousarray(chart, np.uint32)), _p(np.ascontiguousarray(normal, np.float32)),
                    _p(v), N, _p(np.ascontiguousarray(valid, np.uint8)), int(r), _p(out))
    return out


def fill(w, h, chart, v, valid, rings):
    v = np.array(v, np.float32).reshape(w * h, -1)
    valid = np.array(valid, np.uint8)
    lib().or_fill(w, h, _p(np.ascontiguousarray(chart, np.uint32)), _p(v), v.shape[1], _p(valid), int(rings))
    return v, valid


def sun_field(w, h, chart, normal, hard, covered, g, radius):
    out = np.zeros(w * h, np.float32)
    lib().or_sun_field(w, h, _p(np.ascontiguousarray(chart, np.uint32)), _p(np.ascontiguousarray(normal, np.float32)),
                       _p(np.ascontiguousarray(hard, np.uint32)), _p(np.ascontiguousarray(covered, np.uint8)), int(g),
                       float(radius), _p(out))
    return out


def tracer(threads: int = 0):
    """An lb_tracer (include/lightbaker.h) whose passes run on this oracle, for the product's bake
    driver: returns (tracer, keepalive)."""
    import lightbaker_b200._native as N
    state = {}

    def scene_cb(ctx, nodes, n_nodes, tris, n_tris, mats, n_mats, charts, n_charts):
        nb = C.string_at(nodes, n_nodes * 32)
        tb = C.string_at(tris, n_tris * 48)
        mb = C.string_at(mats, n_mats * 16) if n_mats else b""
        cb = C.string_at(charts, n_charts * 32) if n_charts else b""
        state["scene"] = Scene(np.frombuffer(nb, N.NODE).copy(), np.frombuffer(tb, N.TRI).copy(),
                               np.frombuffer(mb, np.float32).copy(), np.frombuffer(cb, np.float32).copy())
        return 0

    def run_cb(ctx, pass_, params, items, n, light, n_light, out, rays):
        it = np.frombuffer(C.string_at(items, n * 64), N.TEXEL).copy()
        li = np.frombuffer(C.string_at(light, n_light * 16), np.float32).copy() if n_light else None
        res, cnt = run(pass_, state["scene"], params.contents, it, li, threads)
        C.memmove(out, res.ctypes.data, res.nbytes)
        rays[0] = cnt["rays"]
        return 0

    scb = N.SCENE_CB(scene_cb)
    rcb = N.RUN_CB(run_cb)
    t = N.Tracer(None, scb, rcb)
    return t, (scb, rcb, state)
