"""The float64 transport restatement (oracle/transport_ref.py) checked on the CPU: its smooth and fill
operators against the oracle's filter.rs restatement, and its gradient against central differences on a
synthetic texel layout."""
import numpy as np
import pytest

import oracle
from oracle import transport_ref as T


def _tile(rng, w, h, charts=3):
    chart = rng.integers(0, charts, size=w * h).astype(np.uint32)
    chart[rng.uniform(size=w * h) < 0.15] = 0xFFFFFFFF
    normal = np.tile(np.array([0.0, 1.0, 0.0], np.float32), (w * h, 1))
    tilt = rng.uniform(size=w * h) < 0.2
    normal[tilt] = np.array([0.6, 0.0, 0.8], np.float32)
    return chart, normal


@pytest.mark.parametrize("r", [1, 2])
def test_smooth_matrix_is_filter_smooth(r):
    rng = np.random.default_rng(r)
    w, h = 13, 9
    chart, normal = _tile(rng, w, h)
    valid = (rng.uniform(size=w * h) < 0.7) & (chart != 0xFFFFFFFF)
    v = rng.uniform(0, 2, size=(w * h, 3)).astype(np.float32)
    tiles = np.array([[0, 0, w, h, 0]], np.uint32)
    L = T.Layout(tiles, w * h, w)
    q = float(r) * 0.75
    sigma2 = np.float32(2.0) * np.float32(q * q)
    wts = np.array([np.exp(-np.float32(dx * dx + dy * dy) / sigma2) for dy in range(-r, r + 1) for dx in range(-r, r + 1)],
                   np.float32)
    m = T.smooth_matrix(L, chart.astype(np.int64), normal, valid, r, wts)
    got = m @ v.astype(np.float64)
    want = oracle.smooth(w, h, chart, normal, v, valid.astype(np.uint8), r)
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-6)


def test_fill_rings_are_filter_fill():
    rng = np.random.default_rng(5)
    w, h = 11, 12
    chart, _ = _tile(rng, w, h)
    valid = rng.uniform(size=w * h) < 0.3
    v = rng.uniform(0, 2, size=(w * h, 3)).astype(np.float32)
    tiles = np.array([[0, 0, w, h, 0]], np.uint32)
    L = T.Layout(tiles, w * h, w)
    x = v.astype(np.float64)
    was = valid.copy()
    for _ in range(4):
        m, was = T.fill_ring(L, chart.astype(np.int64), was)
        x = m @ x
    want, known = oracle.fill(w, h, chart, v, valid.astype(np.uint8), 4)
    np.testing.assert_array_equal(was, known.astype(bool))
    np.testing.assert_allclose(x, want, rtol=2e-6, atol=1e-6)


def _synthetic(seed=0):
    """Two tiles in a 16 x 8 atlas, two bounces, 8 rays a gathered texel, 3 materials."""
    rng = np.random.default_rng(seed)
    aw, ah, ds = 16, 8, 2
    tiles = np.array([[0, 0, 8, 8, 0], [8, 0, 6, 5, 64]], np.uint32)
    n_tex = 64 + 30
    chart = np.concatenate([rng.integers(0, 2, 64), rng.integers(2, 4, 30)]).astype(np.uint32)
    covered = rng.uniform(size=n_tex) < 0.85
    chart[~covered] = 0xFFFFFFFF
    texels = np.zeros((n_tex, 16), np.float32)
    texels[:, 5] = 1.0
    texels[:, 0] = covered
    gathered = (covered & (rng.uniform(size=n_tex) < 0.6)).astype(np.uint8)
    known = np.where(covered, np.where(rng.uniform(size=n_tex) < 0.8, 2, 1), 0).astype(np.uint8)
    state = np.zeros(n_tex, np.uint8)
    fb_tex = np.nonzero(known == 0)[0][:2]
    state[fb_tex] = 5
    known[fb_tex] = 1
    kb = np.where(state == 5, 0, known).astype(np.uint8)
    owner = np.full(aw * ah, 0xFFFFFFFF, np.uint32)
    for x, y, w, h, off in tiles:
        for yy in range(h):
            for xx in range(w):
                owner[(y + yy) * aw + x + xx] = off + yy * w + xx
    idx = np.nonzero(gathered)[0].astype(np.uint32)
    rays, M = 8, 3
    n_rec = len(idx) * rays
    kind = rng.choice([0, 1, 2], size=n_rec, p=[0.3, 0.1, 0.6])
    mat = rng.integers(0, M, n_rec)
    li = rng.integers(0, aw * ah, n_rec).astype(np.uint32)
    li[rng.uniform(size=n_rec) < 0.1] = 0xFFFFFFFF
    ybits = rng.uniform(-0.3, 1.0, n_rec).astype(np.float32).view(np.uint32)
    rec = np.zeros((n_rec, 2), np.uint32)
    rec[:, 0] = (kind.astype(np.uint32) << 30) | np.where(kind == 2, mat, 0).astype(np.uint32)
    rec[:, 1] = np.where(kind == 0, ybits, np.where(kind == 2, li, 0))
    r = 1
    wts = np.array([np.exp(-(dx * dx + dy * dy) / 1.125) for dy in (-1, 0, 1) for dx in (-1, 0, 1)], np.float32)
    return {
        "shape": np.array([aw, ah, aw // ds, ah // ds, ds, r, 3, 2, rays, len(idx), n_tex, M], np.uint32),
        "tiles": tiles, "texels": texels, "chart": chart, "gathered": gathered, "known": known,
        "known_bounce": kb, "state": state,
        "direct_light": np.concatenate([rng.uniform(0, 3, (n_tex, 3)), np.zeros((n_tex, 1))], 1).astype(np.float32),
        "fixed_indirect": np.concatenate([rng.uniform(0, 1, (n_tex, 3)), np.zeros((n_tex, 1))], 1).astype(np.float32),
        "owner": owner, "gathered_index": idx, "records": rec, "smooth_weights": wts,
    }


def test_reference_gradient_is_central_differences():
    arrays = _synthetic()
    ref = T.TransportRef(arrays)
    rng = np.random.default_rng(1)
    theta = np.concatenate([rng.uniform(0.2, 0.8, 9), [0.3, 0.4, 0.5, 0.2, 0.2, 0.3, 0.1, 0.1, 0.1, 1.0]])
    g = rng.normal(size=(ref.iw * ref.ih, 3))
    _, grad = ref.gradient(theta, g)
    import torch
    h = 1e-3
    for j in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[j] += h
        tm[j] -= h
        fp = (ref.forward(torch.from_numpy(tp)).numpy() * g).sum()
        fm = (ref.forward(torch.from_numpy(tm)).numpy() * g).sum()
        fd = (fp - fm) / (2 * h)
        assert abs(fd - grad[j]) <= 1e-6 * max(1.0, abs(grad[j])), (j, fd, grad[j])
    # theta enters: every slot has a nonzero gradient in this layout
    assert np.count_nonzero(grad) == len(theta)
