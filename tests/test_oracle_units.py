"""The oracle's sample sequence and helpers against independent Python restatements of
crates/lightbaker/src/gpu/trace.wgsl:41-61."""
import math

import numpy as np
import pytest

import oracle


def pcg_py(v):
    # trace.wgsl:41-45 in Python integers, u32 wraparound
    s = (v * 747796405 + 2891336453) & 0xffffffff
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xffffffff
    return ((w >> 22) ^ w) & 0xffffffff


def test_pcg_and_rand():
    rng = np.random.default_rng(0)
    for v in list(rng.integers(0, 2**32, size=2000, dtype=np.uint64)) + [0, 1, 0xffffffff, 7919 * 123456]:
        v = int(v)
        assert oracle.pcg(v) == pcg_py(v)
    for a, b in [(0, 3), (7919, 5), (0xffffffff, 17), (123456789, 2000)]:
        want = np.float32(np.float32(pcg_py(a ^ pcg_py((b + 0) & 0xffffffff))) * np.float32(2.0**-32))
        assert oracle.rand(a, b, 0) == want


def test_radical():
    for i in [0, 1, 2, 3, 255, 1000, 2**31, 0xffffffff]:
        rev = int(f"{i:032b}"[::-1], 2)
        assert oracle.radical(i) == np.float32(np.float32(rev) * np.float32(2.0**-32))


def test_sincos_accuracy():
    xs = np.concatenate([np.linspace(0, 2 * math.pi, 5001), np.arange(256) * 2.399963])
    worst = 0.0
    for x in xs.astype(np.float32):
        s, c = oracle.sincos(float(x))
        worst = max(worst, abs(s - math.sin(float(x))), abs(c - math.cos(float(x))))
    assert worst < 3e-7, worst


def test_item_rays_are_unit_and_keyed():
    import lightbaker_b200 as lb
    from lightbaker_b200 import scenes
    P = lb.prepare(scenes.small_map())
    items = P.covered_texels()[:50]
    for i, it in enumerate(items):
        r = oracle.item_rays(0, P.params, it, i)
        n = np.linalg.norm(r["d"].astype(np.float64), axis=1)
        assert np.all(np.abs(n - 1) < 1e-5)
        ao = r["kind"] == 3
        assert ao.sum() == P.params.counts[1]
        assert np.array_equal(r["key"][ao], (i * 7919 + 2000 + np.arange(ao.sum())) & 0xffffffff)
        # occlusion rays leave the surface's front (cosine hemisphere about the normal)
        nrm = it["normal"][:3]
        assert np.all(r["d"][ao] @ nrm > -1e-6)


def test_fp64_twin_agrees_away_from_edges():
    """The FP32 walk and its FP64 twin agree on rays that pass no edge within 1e-4."""
    import lightbaker_b200 as lb
    from lightbaker_b200 import scenes
    P = lb.prepare(scenes.small_map())
    sc = oracle.Scene.of(P)
    items = P.covered_texels()[::97][:200]
    n_cmp = n_amb = 0
    for i, it in enumerate(items):
        r = oracle.item_rays(0, P.params, it, i)
        for k in range(0, len(r["d"]), 7):
            o, d, tm, an, key = r["o"][k], r["d"][k], r["tmax"][k], r["any"][k], r["key"][k]
            t32, tri32, b32 = oracle.trace(sc, P.params, o, d, tm, an, key, 32)
            t64, tri64, b64 = oracle.trace(sc, P.params, o, d, tm, an, key, 64)
            if oracle.ray_ambiguous(sc, P.params, o, d, tm, key, 1e-4):
                n_amb += 1
                continue
            n_cmp += 1
            assert (tri32 == 0xffffffff) == (tri64 == 0xffffffff)
            if not an and tri32 != 0xffffffff:
                assert tri32 == tri64 and b32 == b64
                assert abs(t32 - t64) <= 1e-4 * max(1.0, t64)
    assert n_cmp > 1000 and n_amb < n_cmp // 10
