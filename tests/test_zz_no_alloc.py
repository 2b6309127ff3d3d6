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
