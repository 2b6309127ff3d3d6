"""lb_fill_fixed, the fill for callers that cannot allocate device memory (a host application that owns
the GPU's memory through its own allocator, or a path where an allocation would synchronise the device):
it must give what lb_fill gives, call after call, with its scratch in the library's fixed device array.
This file runs last (pytest collects it after the others) and passes alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import _native as N
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


def _tile(seed):
    P = lb.prepare(scenes.small_map())
    tex = P.rasterize(0)
    h, w = tex.shape
    cov = (tex["pos"][:, :, 3] > 0.5).reshape(-1)
    chart = np.where(cov, tex["normal"][:, :, 3].reshape(-1).view(np.uint32), np.uint32(0xffffffff)).astype(np.uint32)
    rng = np.random.default_rng(seed)
    return w, h, chart, cov, rng


def test_fixed_scratch_fill_matches_lb_fill_twice(gpu):
    import torch
    for call, (channels, rings) in enumerate([(3, 8), (4, 5)]):
        w, h, chart, cov, rng = _tile(call)
        values = rng.uniform(0, 4, size=(w * h, channels)).astype(np.float32)
        valid = (cov & (rng.uniform(size=w * h) > 0.5)).astype(np.uint8)
        d_chart = torch.from_numpy(chart.view(np.int32)).cuda()
        a_v, a_k = torch.from_numpy(values).cuda(), torch.from_numpy(valid).cuda()
        b_v, b_k = torch.from_numpy(values).cuda(), torch.from_numpy(valid).cuda()
        torch.cuda.synchronize()
        N.check(N.lib().lb_fill(gpu.handle, w, h, d_chart.data_ptr(), a_v.data_ptr(), channels, a_k.data_ptr(),
                                rings), "lb_fill")
        N.check(N.lib().lb_fill_fixed(C.c_void_p(gpu.stream), w, h, d_chart.data_ptr(), b_v.data_ptr(), channels,
                                      b_k.data_ptr(), rings), "lb_fill_fixed")
        gpu.sync()
        # the same bits: both run the same kernels on the same inputs
        assert np.array_equal(a_k.cpu().numpy(), b_k.cpu().numpy())
        assert np.array_equal(a_v.cpu().numpy().view(np.uint32), b_v.cpu().numpy().view(np.uint32))


def test_fixed_scratch_rejects_oversized_tiles(gpu):
    import torch
    w, h = 1024, 512
    chart = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    v = torch.zeros(w * h, dtype=torch.float32, device="cuda")
    k = torch.zeros(w * h, dtype=torch.uint8, device="cuda")
    rc = N.lib().lb_fill_fixed(C.c_void_p(gpu.stream), w, h, chart.data_ptr(), v.data_ptr(), 1, k.data_ptr(), 2)
    assert rc == -7 and "512 x 512" in N.last_error()


def _driver():
    """The CUDA driver API (libcuda), for a context the test makes itself."""
    cu = C.CDLL("libcuda.so.1")
    for name in ("cuDeviceGet", "cuCtxCreate_v2", "cuCtxPopCurrent_v2", "cuCtxPushCurrent_v2", "cuCtxDestroy_v2",
                 "cuCtxSynchronize", "cuMemAlloc_v2", "cuMemFree_v2", "cuMemcpyHtoD_v2", "cuMemcpyDtoH_v2",
                 "cuStreamCreate", "cuStreamDestroy_v2", "cuStreamBeginCapture_v2", "cuStreamEndCapture",
                 "cuGraphDestroy"):
        getattr(cu, name).restype = C.c_int
    return cu


def _ok(rc, what):
    assert rc == 0, f"{what}: CUresult {rc}"


def test_fixed_scratch_fill_in_a_second_context(gpu):
    """A host application (an engine, an editor) may run the library in a context it created itself rather
    than the device's primary one. The fixed array then has another address in that context, so the cached
    address must follow the context: the fill in a second context on the same device, and again in the
    first one afterwards, must still equal lb_fill."""
    import torch
    w, h, chart, cov, rng = _tile(7)
    channels, rings = 4, 6
    values = rng.uniform(0, 4, size=(w * h, channels)).astype(np.float32)
    valid = (cov & (rng.uniform(size=w * h) > 0.5)).astype(np.uint8)
    d_chart = torch.from_numpy(chart.view(np.int32)).cuda()
    a_v, a_k = torch.from_numpy(values).cuda(), torch.from_numpy(valid).cuda()
    torch.cuda.synchronize()
    N.check(N.lib().lb_fill(gpu.handle, w, h, d_chart.data_ptr(), a_v.data_ptr(), channels, a_k.data_ptr(), rings),
            "lb_fill")
    gpu.sync()
    want_v, want_k = a_v.cpu().numpy(), a_k.cpu().numpy()

    cu = _driver()
    dev, ctx = C.c_int(), C.c_void_p()
    _ok(cu.cuDeviceGet(C.byref(dev), 0), "cuDeviceGet")
    _ok(cu.cuCtxCreate_v2(C.byref(ctx), 0, dev), "cuCtxCreate")  # current on this thread from here
    bufs = []
    try:
        def upload(a):
            p = C.c_uint64()
            _ok(cu.cuMemAlloc_v2(C.byref(p), C.c_size_t(a.nbytes)), "cuMemAlloc")
            bufs.append(p)
            _ok(cu.cuMemcpyHtoD_v2(p, a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)), "cuMemcpyHtoD")
            return p.value
        p_chart, p_v, p_k = upload(np.ascontiguousarray(chart)), upload(values.copy()), upload(valid.copy())
        # the context's own default stream (null handle)
        N.check(N.lib().lb_fill_fixed(None, w, h, p_chart, p_v, channels, p_k, rings), "lb_fill_fixed (context 2)")
        _ok(cu.cuCtxSynchronize(), "cuCtxSynchronize")
        got_v, got_k = np.empty_like(values), np.empty_like(valid)
        _ok(cu.cuMemcpyDtoH_v2(got_v.ctypes.data_as(C.c_void_p), C.c_uint64(p_v), C.c_size_t(got_v.nbytes)), "DtoH")
        _ok(cu.cuMemcpyDtoH_v2(got_k.ctypes.data_as(C.c_void_p), C.c_uint64(p_k), C.c_size_t(got_k.nbytes)), "DtoH")
    finally:
        for p in bufs:
            cu.cuMemFree_v2(p)
        popped = C.c_void_p()
        cu.cuCtxPopCurrent_v2(C.byref(popped))
        cu.cuCtxDestroy_v2(ctx)
    assert np.array_equal(want_k, got_k)
    assert np.array_equal(want_v.view(np.uint32), got_v.view(np.uint32))

    # back in the primary context: its own address again
    b_v, b_k = torch.from_numpy(values).cuda(), torch.from_numpy(valid).cuda()
    torch.cuda.synchronize()
    N.check(N.lib().lb_fill_fixed(C.c_void_p(gpu.stream), w, h, d_chart.data_ptr(), b_v.data_ptr(), channels,
                                  b_k.data_ptr(), rings), "lb_fill_fixed (primary context)")
    gpu.sync()
    assert np.array_equal(want_k, b_k.cpu().numpy())
    assert np.array_equal(want_v.view(np.uint32), b_v.cpu().numpy().view(np.uint32))


def test_fixed_scratch_first_call_refused_under_capture():
    """The first call in a context looks up the array's address, which may load the library into that
    context; during a stream capture it is refused with a clear message instead, and nothing is launched."""
    cu = _driver()
    dev, ctx, stream, graph = C.c_int(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    _ok(cu.cuDeviceGet(C.byref(dev), 0), "cuDeviceGet")
    _ok(cu.cuCtxCreate_v2(C.byref(ctx), 0, dev), "cuCtxCreate")
    try:
        _ok(cu.cuStreamCreate(C.byref(stream), 1), "cuStreamCreate")  # non-blocking
        _ok(cu.cuStreamBeginCapture_v2(stream, 2), "cuStreamBeginCapture")  # relaxed mode
        # no pointer is dereferenced: the call is refused before any launch
        rc = N.lib().lb_fill_fixed(stream, 16, 16, C.c_void_p(256), C.c_void_p(256), 1, C.c_void_p(256), 1)
        msg = N.last_error()
        _ok(cu.cuStreamEndCapture(stream, C.byref(graph)), "cuStreamEndCapture")
        if graph.value:
            cu.cuGraphDestroy(graph)
        assert rc == -1 and "before any stream capture" in msg
    finally:
        if stream.value:
            cu.cuStreamDestroy_v2(stream)
        popped = C.c_void_p()
        cu.cuCtxPopCurrent_v2(C.byref(popped))
        cu.cuCtxDestroy_v2(ctx)
