"""The bounce transport of a bake and its adjoint (lb_transport_* in include/lightbaker.h).

    tr = Transport(scene_bytes, gpu)              # bakes once, records every gather ray's outcome
    theta = tr.theta0()                            # albedos, zenith, horizon, ground, sun scale
    indirect = tr.forward(theta)                   # (indirect_height, indirect_width, 3)
    g_theta = tr.backward(g_indirect)              # d(loss)/d(theta) for d(loss)/d(indirect)

`transport(theta, tr)` is the same pair as a torch autograd op on CUDA tensors.

No reference counterpart: the reference bakes at the scene's own values (crates/lightbaker/src/bake.rs:
300-421 is the function differentiated here).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import LightbakerError

_EXPORT_DTYPES = {
    "records": (np.uint32, 2), "gathered_index": (np.uint32, 1), "texels": (np.float32, 16), "sample_points": (np.float32, 4), "chart": (np.uint32, 1),
    "gathered": (np.uint8, 1), "known": (np.uint8, 1), "known_bounce": (np.uint8, 1), "state": (np.uint8, 1),
    "direct_light": (np.float32, 4), "fixed_indirect": (np.float32, 4), "owner": (np.uint32, 1),
    "light_flags": (np.uint8, 1), "tiles": (np.uint32, 5), "smooth_weights": (np.float32, 1), "shape": (np.uint32, 1),
    "direct_records": (np.float32, 4), "valid": (np.uint8, 1), "field": (np.float32, 1), "ao": (np.float32, 1),
    "direct": (np.float32, 4), "indirect_light": (np.float32, 4), "gather_out": (np.float32, 4),
    "light": (np.float32, 4), "probes": (np.float32, 16),
    "volume_records": (np.uint32, 2), "volume_items": (np.float32, 16), "volume_slots": (np.uint32, 1),
    "volume_raw": (np.float32, 16), "volume_grid": (np.uint32, 1),
}


class Transport:
    """The indirect atlas as a function of theta, with its adjoint. max_checkpoints bounds the light atlases
    the forward keeps (0: every bounce's); the backward recomputes the rest."""

    def __init__(self, scene: bytes, gpu, max_checkpoints: int = 0):
        self._gpu = gpu
        self._h = N.lib().lb_transport_create(gpu.handle, scene, len(scene), max_checkpoints)
        if not self._h:
            raise LightbakerError(N.last_error())
        s = N.TransportShape()
        N.check(N.lib().lb_transport_info(self._h, C.byref(s)), "lb_transport_info")
        self.shape = s
        self.n_materials = s.n_materials
        self.n_params = s.n_params
        self.iw, self.ih = s.indirect_width, s.indirect_height

    def theta0(self) -> np.ndarray:
        t = np.zeros(self.n_params, np.float32)
        N.check(N.lib().lb_transport_theta0(self._h, t.ctypes.data), "lb_transport_theta0")
        return t

    def forward(self, theta) -> np.ndarray:
        t = np.ascontiguousarray(theta, dtype=np.float32)
        if t.shape != (self.n_params,):
            raise LightbakerError(f"theta has {t.size} values, the transport takes {self.n_params}")
        out = np.zeros((self.ih, self.iw, 4), np.float32)
        N.check(N.lib().lb_transport_forward(self._h, t.ctypes.data, out.ctypes.data), "lb_transport_forward")
        return out[:, :, :3]

    def backward(self, g_indirect) -> np.ndarray:
        g = np.zeros((self.ih, self.iw, 4), np.float32)
        g[:, :, :3] = np.asarray(g_indirect, dtype=np.float32).reshape(self.ih, self.iw, 3)
        out = np.zeros(self.n_params, np.float32)
        N.check(N.lib().lb_transport_backward(self._h, g.ctypes.data, out.ctypes.data), "lb_transport_backward")
        return out

    def forward_async(self, d_theta: int, d_indirect: int) -> None:
        """Device pointers (theta: n_params floats; indirect: ih * iw float4), enqueued on gpu.stream."""
        N.check(N.lib().lb_transport_forward_async(self._h, C.c_void_p(d_theta), C.c_void_p(d_indirect)),
                "lb_transport_forward_async")

    def backward_async(self, d_g_indirect: int, d_g_theta: int) -> None:
        N.check(N.lib().lb_transport_backward_async(self._h, C.c_void_p(d_g_indirect), C.c_void_p(d_g_theta)),
                "lb_transport_backward_async")

    def bake_indirect(self) -> np.ndarray:
        out = np.zeros((self.ih, self.iw, 4), np.float32)
        N.check(N.lib().lb_transport_bake_indirect(self._h, out.ctypes.data), "lb_transport_bake_indirect")
        return out[:, :, :3]

    def export(self, name: str) -> np.ndarray:
        n = N.lib().lb_transport_export(self._h, name.encode(), None, 0)
        if n == 0 and N.last_error():
            raise LightbakerError(N.last_error())
        dtype, width = _EXPORT_DTYPES[name]
        out = np.zeros(n // np.dtype(dtype).itemsize, dtype)
        if n and N.lib().lb_transport_export(self._h, name.encode(), out.ctypes.data, n) != n:
            raise LightbakerError(N.last_error())
        return out.reshape(-1, width) if width > 1 else out

    def close(self) -> None:
        if self._h:
            N.lib().lb_transport_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def transport(theta, tr: Transport):
    """The transport as a torch autograd op: theta (CUDA float32, n_params) -> indirect (ih, iw, 3)."""
    import torch

    class _Op(torch.autograd.Function):
        @staticmethod
        def forward(ctx, th):
            th = th.detach().contiguous().float()
            out = torch.empty((tr.ih, tr.iw, 4), dtype=torch.float32, device=th.device)
            torch.cuda.current_stream().synchronize()
            tr.forward_async(th.data_ptr(), out.data_ptr())
            tr._gpu.sync()
            return out[:, :, :3]

        @staticmethod
        def backward(ctx, g):
            gi = torch.zeros((tr.ih, tr.iw, 4), dtype=torch.float32, device=g.device)
            gi[:, :, :3] = g
            gt = torch.empty(tr.n_params, dtype=torch.float32, device=g.device)
            torch.cuda.current_stream().synchronize()
            tr.backward_async(gi.data_ptr(), gt.data_ptr())
            tr._gpu.sync()
            return gt

    return _Op.apply(theta)
