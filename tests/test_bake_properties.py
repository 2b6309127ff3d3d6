"""The reference's own integration test restated (crates/lightbaker/tests/bake.rs:95-154): bake its
hand-built scene and check what the light must show (a box's shadow, darker corners at its foot, a red
wall's colour bounced onto the ground, the volume's sun, light along a strip narrower than a texel),
then bake again from the cache (nothing baked, identical atlas) and with the box moved (only the tiles
it reaches).

The CPU run bakes through the product's host pipeline with the oracle's passes: it pins the oracle by
the reference's own assertions. The gpu run bakes with the CUDA passes.
"""
import math
import shutil
import tempfile

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes
from helpers import affine_texel


def ground_texel(b, positions_ground, x, z):
    """tests/bake.rs:74-89: the atlas texel a ground point falls in."""
    tri = None
    for t in range(len(positions_ground) // 3):
        p = positions_ground[t * 3:t * 3 + 3]
        lo, hi = p.min(axis=0), p.max(axis=0)
        if lo[0] <= x <= hi[0] and lo[2] <= z <= hi[2]:
            tri = t
            break
    c = b.tri_charts[tri]
    ax, ay = affine_texel(b.charts[c], (x, 0.0, z))
    return ay, ax


def ground_positions():
    out = []
    for i in range(16):
        for j in range(16):
            x, z = i * 4.0, j * 4.0
            out += scenes.quad((x, 0, z), (x, 0, z + 4), (x + 4, 0, z + 4), (x + 4, 0, z))
    return np.array(out, np.float32)


def check_properties(b):
    g = ground_positions()
    assert b.stats.tiles_baked == b.stats.tiles
    shade = b.direct[ground_texel(b, g, 11.0, 11.0)]
    open_ = b.direct[ground_texel(b, g, 4.0, 11.0)]
    assert shade[0] < 0.4, f"in the box's shadow: field {shade[0]}"
    assert open_[0] > 0.6, f"in the sun: field {open_[0]}"
    foot = b.direct[ground_texel(b, g, 7.85, 11.0)]
    assert foot[1] < open_[1] - 0.1, f"occlusion at the box's foot {foot[1]} vs open {open_[1]}"

    def small(yx):
        return (yx[0] // 2, yx[1] // 2)
    near = b.indirect[small(ground_texel(b, g, 38.5, 40.0))]
    far = b.indirect[small(ground_texel(b, g, 20.0, 40.0))]
    assert near[0] / near[1] > far[0] / far[1] * 1.15, f"bounced red near the wall {near} vs far {far}"
    assert far[2] > 0.0

    nx, ny, nz = b.volume_size
    o, st = b.volume_origin, b.volume_step

    def probe(x, y, z):
        i, j, k = int((x - o[0]) / st), int((y - o[1]) / st), int((z - o[2]) / st)
        return b.volume[(j * nz + k) * nx + i]
    assert probe(20.0, 0.5, 40.0)[0][3] > 0.9
    assert probe(42.0, 0.5, 40.0)[0][3] < 0.1

    ds = b.width // b.indirect_size[0]
    # the strip is mesh 3: its first triangle's chart (tests/bake.rs:133-144)
    n_ground, n_box, n_wall = 16 * 16 * 2, 12, 12
    c = b.tri_charts[n_ground + n_box + n_wall]
    for k in range(12):
        y = 0.3 + k * 0.19
        ax, ay = affine_texel(b.charts[c], (30.0, y, 20.025))
        e = b.indirect[ay // ds, ax // ds]
        assert e.sum() > 0.1, f"strip at {y} m: {e}"


def bake_twice_and_move(bake_fn):
    d = tempfile.mkdtemp(prefix="lightbaker-test-")
    try:
        b = bake_fn(scenes.reference_test(8.0), d)
        check_properties(b)
        again = bake_fn(scenes.reference_test(8.0), d)
        assert again.stats.tiles_baked == 0
        assert again.stats.chunks_baked == 0
        assert np.array_equal(again.direct, b.direct)
        moved = bake_fn(scenes.reference_test(6.0), d)
        assert 0 < moved.stats.tiles_baked < moved.stats.tiles, (moved.stats.tiles_baked, moved.stats.tiles)
        return b
    finally:
        shutil.rmtree(d, ignore_errors=True)


def test_reference_properties_on_oracle():
    import oracle
    t, keep = oracle.tracer()
    bake_twice_and_move(lambda s, d: lb.bake_with(s, t, cache=d))


@pytest.mark.gpu
def test_reference_properties_on_gpu(gpu):
    bake_twice_and_move(lambda s, d: lb.bake(s, gpu, cache=d))
