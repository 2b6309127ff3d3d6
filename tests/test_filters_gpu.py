"""The texel filters on the device (lb_smooth, lb_fill, lb_sun_field: crates/lightbaker/src/filter.rs)
against the oracle's restatement on the same tiles: bit-identical. Tiles come from the rasteriser of a
real map (charts, normals, covered texels), values and hard-bit masks are seeded random."""
import ctypes as C

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import _native as N
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


def tiles(n=4):
    P = lb.prepare(scenes.small_map())
    for t in range(min(n, len(P.tiles))):
        tex = P.rasterize(t)
        h, w = tex.shape
        cov = (tex["pos"][:, :, 3] > 0.5).reshape(-1)
        chart = np.where(cov, tex["normal"][:, :, 3].reshape(-1).view(np.uint32), np.uint32(0xffffffff)).astype(np.uint32)
        normal = np.ascontiguousarray(tex["normal"][:, :, :3].reshape(-1, 3), np.float32)
        yield w, h, chart, normal, cov


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t, dtype, shape):
    return t.cpu().numpy().view(dtype).reshape(shape)


@pytest.mark.parametrize("channels,radius", [(1, 1), (3, 2), (4, 1), (2, 0)])
def test_smooth(gpu, channels, radius):
    import oracle
    rng = np.random.default_rng(channels * 10 + radius)
    for w, h, chart, normal, cov in tiles():
        v = rng.uniform(0, 4, size=(w * h, channels)).astype(np.float32)
        valid = (cov & (rng.uniform(size=w * h) > 0.2)).astype(np.uint8)
        want = oracle.smooth(w, h, chart, normal, v, valid, radius)
        dc, dn, dv, dvalid = dev(chart.view(np.int32)), dev(normal), dev(v), dev(valid)
        import torch
        out = torch.empty_like(dv)
        N.check(N.lib().lb_smooth(gpu.handle, w, h, dc.data_ptr(), dn.data_ptr(), dv.data_ptr(), channels,
                                  dvalid.data_ptr(), radius, out.data_ptr()), "lb_smooth")
        gpu.sync()
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("channels,rings", [(1, 6), (3, 8), (4, 3)])
def test_fill(gpu, channels, rings):
    import oracle
    rng = np.random.default_rng(channels * 100 + rings)
    for w, h, chart, normal, cov in tiles():
        v = rng.uniform(0, 4, size=(w * h, channels)).astype(np.float32)
        valid = (cov & (rng.uniform(size=w * h) > 0.5)).astype(np.uint8)
        want_v, want_k = oracle.fill(w, h, chart, v, valid, rings)
        dc, dv, dk = dev(chart.view(np.int32)), dev(v), dev(valid)
        N.check(N.lib().lb_fill(gpu.handle, w, h, dc.data_ptr(), dv.data_ptr(), channels, dk.data_ptr(), rings),
                "lb_fill")
        gpu.sync()
        assert np.array_equal(dk.cpu().numpy(), want_k)
        assert np.array_equal(dv.cpu().numpy().view(np.uint32), want_v.view(np.uint32))


@pytest.mark.parametrize("g,radius", [(4, 2.0), (3, 1.5), (2, 3.0)])
def test_sun_field(gpu, g, radius):
    import oracle
    rng = np.random.default_rng(g)
    for w, h, chart, normal, cov in tiles():
        # shadow edges: a half-plane of lit cells per tile with noise
        yy, xx = np.mgrid[0:h, 0:w]
        lit = ((xx + 0.3 * yy) < w * 0.5).reshape(-1)
        bits = np.where(lit, (1 << (g * g)) - 1, 0).astype(np.uint32)
        flip = rng.integers(0, 1 << (g * g), size=w * h, dtype=np.uint32) & rng.integers(0, 1 << (g * g), size=w * h,
                                                                                          dtype=np.uint32)
        hard = bits ^ flip
        covered = cov.astype(np.uint8)
        want = oracle.sun_field(w, h, chart, normal, hard, covered, g, radius)
        import torch
        out = torch.empty(w * h, dtype=torch.float32, device="cuda")
        dc, dn, dh, dcov = dev(chart.view(np.int32)), dev(normal), dev(hard.view(np.int32)), dev(covered)
        N.check(N.lib().lb_sun_field(gpu.handle, w, h, dc.data_ptr(), dn.data_ptr(), dh.data_ptr(), dcov.data_ptr(), g,
                                     C.c_float(radius), out.data_ptr()), "lb_sun_field")
        gpu.sync()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want.view(np.uint32))
