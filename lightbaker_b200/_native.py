"""ctypes declarations of the C ABI in include/lightbaker.h, loaded from the in-tree library.

The library is the product: if it cannot be loaded this module raises, it never substitutes anything.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liblightbaker_b200.so"

NODE = np.dtype([("min", "<f4", 3), ("first", "<u4"), ("max", "<f4", 3), ("count", "<u4")])
TRI = np.dtype([("v0", "<f4", 4), ("e1", "<f4", 4), ("e2", "<f4", 4)])
TEXEL = np.dtype([("pos", "<f4", 4), ("normal", "<f4", 4), ("dx", "<f4", 4), ("dy", "<f4", 4)])
RAY = np.dtype([("o", "<f4", 3), ("tmax", "<f4"), ("d", "<f4", 3), ("key", "<u4")])  # lb_ray
HIT = np.dtype([("t", "<f4"), ("tri", "<u4"), ("back", "<u4"), ("pad", "<u4")])     # lb_hit
assert NODE.itemsize == 32 and TRI.itemsize == 48 and TEXEL.itemsize == 64


class Params(C.Structure):
    """The passes' uniform block (crates/lightbaker/src/gpu/mod.rs:11-23)."""

    _fields_ = [("sun_dir", C.c_float * 4), ("sun_irr", C.c_float * 4), ("zenith", C.c_float * 4),
                ("horizon", C.c_float * 4), ("ground", C.c_float * 4), ("fallback", C.c_float * 4),
                ("counts", C.c_uint32 * 4), ("reach", C.c_float * 4), ("atlas", C.c_uint32 * 4)]

    def copy(self) -> "Params":
        p = Params()
        C.memmove(C.byref(p), C.byref(self), C.sizeof(Params))
        return p


assert C.sizeof(Params) == 144


class Counters(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("nodes", C.c_uint64), ("tris", C.c_uint64), ("mats", C.c_uint64)]


class PreparedInfo(C.Structure):
    _fields_ = [("n_nodes", C.c_size_t), ("n_tris", C.c_size_t), ("n_materials", C.c_size_t),
                ("n_charts", C.c_size_t), ("n_tiles", C.c_size_t), ("n_triangles", C.c_size_t),
                ("atlas_width", C.c_uint32), ("atlas_height", C.c_uint32), ("indirect_downscale", C.c_uint32),
                ("padding", C.c_uint32), ("gi_bounces", C.c_uint32), ("has_volume", C.c_uint32),
                ("params", Params)]


class ChartFrame(C.Structure):
    """lb_chart_frame: a chart of the layout (layout.rs:20-40)."""

    _fields_ = [("mesh", C.c_uint32), ("turned", C.c_uint32), ("x", C.c_uint32), ("y", C.c_uint32),
                ("w", C.c_uint32), ("h", C.c_uint32), ("tile", C.c_int32 * 2), ("normal", C.c_float * 3),
                ("u", C.c_float * 3), ("v", C.c_float * 3), ("min", C.c_float * 2), ("max", C.c_float * 2)]


class BakeInfo(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("indirect_width", C.c_uint32),
                ("indirect_height", C.c_uint32), ("has_volume", C.c_uint32), ("volume_size", C.c_uint32 * 3),
                ("volume_origin", C.c_float * 3), ("volume_step", C.c_float),
                ("tiles", C.c_uint64), ("tiles_baked", C.c_uint64), ("texels_baked", C.c_uint64),
                ("chunks", C.c_uint64), ("chunks_baked", C.c_uint64), ("seconds", C.c_double),
                ("rays_direct", C.c_uint64), ("rays_gather", C.c_uint64), ("rays_volume", C.c_uint64),
                ("t_layout", C.c_double), ("t_direct", C.c_double), ("t_bounces", C.c_double),
                ("t_volume", C.c_double), ("t_composite", C.c_double), ("n_charts", C.c_uint64),
                ("n_triangles", C.c_uint64)]


class TransportShape(C.Structure):
    _fields_ = [("n_materials", C.c_uint32), ("n_params", C.c_uint32), ("bounces", C.c_uint32),
                ("checkpoints", C.c_uint32), ("indirect_width", C.c_uint32), ("indirect_height", C.c_uint32),
                ("gathered", C.c_uint32), ("rays", C.c_uint32), ("records", C.c_uint64), ("lit_records", C.c_uint64),
                ("unlit_records", C.c_uint64), ("checkpoint_bytes", C.c_uint64)]


SCENE_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                       C.c_size_t, C.c_void_p, C.c_size_t)
RUN_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(Params), C.c_void_p, C.c_size_t, C.c_void_p,
                     C.c_size_t, C.c_void_p, C.POINTER(C.c_uint64))
LOG_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_char_p)


class Tracer(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("scene", SCENE_CB), ("run", RUN_CB)]


SUM_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int)


class Exchange(C.Structure):
    """lb_exchange: the ranks' element-wise sum of 32-bit words."""

    _fields_ = [("ctx", C.c_void_p), ("rank", C.c_int), ("world", C.c_int), ("sum", SUM_CB)]


class BakeOptions(C.Structure):
    _fields_ = [("cache_dir", C.c_char_p), ("log", LOG_CB), ("log_ctx", C.c_void_p), ("autotune", C.c_int),
                ("trace_every_bounce", C.c_int), ("watertight", C.c_int), ("exchange", C.POINTER(Exchange))]


# every exported entry point: name -> (restype, argtypes)
SIGNATURES = {
    "lb_last_error": (C.c_char_p, []),
    "lb_gpu_open": (C.c_void_p, [C.c_int, C.c_char_p, C.c_size_t]),
    "lb_gpu_close": (None, [C.c_void_p]),
    "lb_scene_upload": (C.c_void_p, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                     C.c_size_t, C.c_void_p, C.c_size_t]),
    "lb_scene_free": (None, [C.c_void_p]),
    "lb_bvh_check": (C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t]),
    "lb_scene_set_vertices": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
    "lb_scene_get_bvh8": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64)]),
    "lb_trace": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_uint32, C.c_void_p]),
    "lb_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(Params), C.c_void_p, C.c_size_t, C.c_void_p,
                         C.c_size_t, C.c_void_p]),
    "lb_set_counting": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_pass_kernel": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_ray_order": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "lb_set_bvh": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_warp_walk": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_fetch": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_refill": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_near": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_set_register_cap": (C.c_int, [C.c_void_p, C.c_int]),
    "lb_get_counters": (C.c_int, [C.c_void_p, C.POINTER(Counters)]),
    "lb_gpu_stream": (C.c_void_p, [C.c_void_p]),
    "lb_gpu_sync": (C.c_int, [C.c_void_p]),
    "lb_run_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(Params), C.c_void_p, C.c_size_t,
                               C.c_uint32, C.c_void_p, C.c_size_t, C.c_void_p]),
    "lb_get_transfer": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_int]),
    "lb_smooth": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                            C.c_void_p, C.c_int, C.c_void_p]),
    "lb_fill": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "lb_fill_fixed": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                C.c_int]),
    "lb_sun_field": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_uint32, C.c_float, C.c_void_p]),
    "lb_prepare": (C.c_void_p, [C.c_char_p, C.c_size_t]),
    "lb_prepared_free": (None, [C.c_void_p]),
    "lb_prepared_get_info": (C.c_int, [C.c_void_p, C.POINTER(PreparedInfo)]),
    "lb_prepared_get_bvh": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lb_prepared_get_materials": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_prepared_get_vertices": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_prepared_get_charts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_prepared_get_tile": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]),
    "lb_prepared_rasterize": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p]),
    "lb_prepared_get_tile_charts": (C.c_size_t, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]),
    "lb_prepared_get_chart": (C.c_size_t, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t]),
    "lb_bake_run": (C.c_void_p, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(BakeOptions)]),
    "lb_bake_run_with": (C.c_void_p, [C.POINTER(Tracer), C.c_char_p, C.c_size_t, C.POINTER(BakeOptions)]),
    "lb_bake_free": (None, [C.c_void_p]),
    "lb_bake_device": (C.c_void_p, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(BakeOptions)]),
    "lb_plan_create": (C.c_void_p, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(BakeOptions)]),
    "lb_plan_launch": (C.c_int, [C.c_void_p]),
    "lb_plan_rays": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "lb_plan_result": (C.c_void_p, [C.c_void_p]),
    "lb_plan_free": (None, [C.c_void_p]),
    "lb_plan_kernels": (C.c_int, [C.c_void_p]),
    "lb_plan_tuning": (C.c_char_p, [C.c_void_p]),
    "lb_transport_create": (C.c_void_p, [C.c_void_p, C.c_char_p, C.c_size_t, C.c_uint32]),
    "lb_transport_info": (C.c_int, [C.c_void_p, C.POINTER(TransportShape)]),
    "lb_transport_theta0": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_transport_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lb_transport_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lb_transport_forward_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lb_transport_backward_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lb_transport_bake_indirect": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_transport_export": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]),
    "lb_transport_free": (None, [C.c_void_p]),
    "lb_bake_get_info": (C.c_int, [C.c_void_p, C.POINTER(BakeInfo)]),
    "lb_bake_get_direct": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_bake_get_indirect": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_bake_get_validity": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_bake_get_volume": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_bake_get_charts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_bake_get_tri_charts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lb_bake_write": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]),
    "lb_free": (None, [C.c_void_p]),
    "lb_scene_encode": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), C.c_size_t,
                                  C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]),
    "lb_bvh8_check": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64),
                                C.POINTER(C.c_uint64)]),
    "lb_bvh8_collapse": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "lb_blake3": (None, [C.c_char_p, C.c_size_t, C.c_void_p]),
    "lb_rgb9e5": (C.c_uint32, [C.POINTER(C.c_float)]),
    "lb_rgb9e5_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "lb_bake_device_encoded": (C.c_int, [C.c_void_p]),
    "lb_rgb9e5_decode": (None, [C.c_uint32, C.POINTER(C.c_float)]),
    "lb_bc4_block": (None, [C.c_void_p, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library, with every signature declared. Raises OSError when it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} is not built: run `python -m lightbaker_b200.build`")
        l = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


class LightbakerError(RuntimeError):
    pass


def last_error() -> str:
    m = lib().lb_last_error()
    return m.decode("utf-8", "replace") if m else ""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise LightbakerError(f"{what}: {last_error()} (status {rc})")


def ptr(a: np.ndarray | None) -> C.c_void_p | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)
