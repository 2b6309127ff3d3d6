"""The ray query (lb_trace) and the watertight triangle test on the GPU, through the C ABI.

- lb_trace with the shader's test equals the oracle's FP32 walk bit for bit (t, triangle, face) on the
  passes' own rays; with the watertight test (lb_scene_set_vertices) it equals the oracle's FP32
  watertight walk bit for bit.
- Hit/miss masks of the two tests agree on every ray not within 1e-4 of a triangle edge; the rays that
  are within it are counted and reported. The watertight masks agree with the FP64 walk the same way.
- On rays crossing the surface exactly at shared edges, the watertight walk never lets a ray through.
- The passes with the watertight test equal the oracle's passes with it, record for record, and a bake
  with it stays within 1e-3 of the shader-test bake on all but the texels whose edge rays flipped.
"""
import numpy as np
import pytest

import lightbaker_b200 as lb
from helpers import edge_crossing_rays
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu
NONE = 0xffffffff


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    return oracle


def _pass_rays(oracle, P, items):
    rays = []
    for pass_, its in ((0, items), (1, items[::4]), (2, [])):
        for i, it in enumerate(its):
            rays.append(oracle.rays_of(oracle.item_rays(pass_, P.params, it, i)))
    return np.concatenate(rays)


def _seed(P):
    return int(np.float32(P.params.reach[3]).view(np.uint32))


def _bits(h):
    return np.stack([h["t"].view(np.uint32), h["tri"], h["back"]], axis=1)


def _oracle_bits(o):
    t, tri, back = o
    return np.stack([t.astype(np.float32).view(np.uint32), tri, back.astype(np.uint32)], axis=1)


@pytest.mark.parametrize("name", ["small_map", "map_100m"])
def test_trace_matches_oracle_both_tests(gpu, oracle_mod, name):
    P = lb.prepare(scenes.WORKLOADS[name]())
    rng = np.random.default_rng(3)
    items = P.covered_texels()
    items = items[np.sort(rng.choice(len(items), size=min(400, len(items)), replace=False))]
    rays = _pass_rays(oracle_mod, P, items)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    gpu.set_bvh(2)
    for any_hit in (False, True):
        g = gpu.trace(buffers, rays, any_hit, _seed(P))
        c = oracle_mod.trace_rays(oracle_mod.Scene.of(P), P.params, rays, any_hit)
        bad = np.nonzero((_bits(g) != _oracle_bits(c)).any(axis=1))[0]
        assert len(bad) == 0, f"shader test, any={any_hit}: {len(bad)} of {len(rays)} rays differ"
    buffers.set_vertices(P.verts)
    for any_hit in (False, True):
        g = gpu.trace(buffers, rays, any_hit, _seed(P))
        c = oracle_mod.trace_rays(oracle_mod.Scene.of(P, watertight=True), P.params, rays, any_hit)
        bad = np.nonzero((_bits(g) != _oracle_bits(c)).any(axis=1))[0]
        assert len(bad) == 0, f"watertight, any={any_hit}: {len(bad)} of {len(rays)} rays differ"
    buffers.set_vertices(None)
    g = gpu.trace(buffers, rays, False, _seed(P))
    c = oracle_mod.trace_rays(oracle_mod.Scene.of(P), P.params, rays, False)
    assert np.array_equal(_bits(g), _oracle_bits(c)), "dropping the vertices restores the shader's test"


@pytest.mark.parametrize("name", ["small_map", "map_100m"])
def test_masks_agree_except_near_edges(gpu, oracle_mod, name):
    """Shadow, occlusion, inside-test and gather hit/miss masks: the watertight walk against the shader's
    test and against FP64, on the GPU; differences only on rays within 1e-4 of an edge (counted)."""
    P = lb.prepare(scenes.WORKLOADS[name]())
    rng = np.random.default_rng(5)
    items = P.covered_texels()
    items = items[np.sort(rng.choice(len(items), size=min(600, len(items)), replace=False))]
    rays = _pass_rays(oracle_mod, P, items)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    gpu.set_bvh(2)
    mt = gpu.trace(buffers, rays, False, _seed(P))
    buffers.set_vertices(P.verts)
    wt = gpu.trace(buffers, rays, False, _seed(P))
    f64 = oracle_mod.trace_rays(oracle_mod.Scene.of(P), P.params, rays, False, precision=64)
    amb = oracle_mod.rays_ambiguous(oracle_mod.Scene.of(P), P.params, rays, 1e-4)
    m_mt, m_wt, m_64 = mt["tri"] != NONE, wt["tri"] != NONE, f64[1] != NONE
    flips = m_mt != m_wt
    print(f"{name}: {len(rays)} rays, {int(amb.sum())} within 1e-4 of an edge; hit/miss flips between the "
          f"tests {int(flips.sum())} (all within it: {not np.any(flips & ~amb)}); watertight vs FP64 "
          f"{int((m_wt != m_64).sum())}")
    assert not np.any(flips & ~amb)
    assert not np.any((m_wt != m_64) & ~amb)


def test_watertight_closes_edges_on_gpu(gpu):
    P = lb.prepare(scenes.small_map())
    rays, pairs = edge_crossing_rays(P.verts)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    res = {}
    for bvh in (2, 8):
        gpu.set_bvh(bvh)
        buffers.set_vertices(None)
        mt = gpu.trace(buffers, rays, False, _seed(P))
        buffers.set_vertices(P.verts)
        wt = gpu.trace(buffers, rays, False, _seed(P))

        def through(h):
            on_edge = (h["tri"] == pairs[:, 0]) | (h["tri"] == pairs[:, 1])
            return (h["tri"] == NONE) | (~on_edge & (h["t"] > 3.01))

        res[bvh] = (int(through(mt).sum()), int(through(wt).sum()))
    gpu.set_bvh(2)
    print(f"edge-crossing rays {len(rays)}: through the edge (shader test, watertight): BVH2 {res[2]}, "
          f"8-wide {res[8]}")
    assert res[2][1] == 0 and res[8][1] == 0


@pytest.mark.parametrize("kernel,near", [(0, 0), (1, 0), (1, 1)], ids=["thread_per_item", "warp", "warp_leaf_lists"])
def test_passes_watertight_bit_exact(gpu, oracle_mod, kernel, near):
    P = lb.prepare(scenes.small_map())
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    buffers.set_vertices(P.verts)
    sc = oracle_mod.Scene.of(P, watertight=True)
    rng = np.random.default_rng(7)
    items = P.covered_texels()
    items = items[np.sort(rng.choice(len(items), size=min(6000, len(items)), replace=False))]
    aw, ah = P.info.atlas_width, P.info.atlas_height
    light = rng.uniform(0.0, 3.0, size=(aw * ah, 4)).astype(np.float32)
    light[:, 3] = (rng.uniform(size=aw * ah) > 0.3).astype(np.float32)
    gpu.set_pass_kernel(kernel)
    gpu.set_ray_order(0, 0)
    gpu.set_bvh(2)
    gpu.set_near(near)
    try:
        for pass_, its in ((lb.Pass.DIRECT, items), (lb.Pass.GATHER, items[:2000])):
            g = gpu.run(pass_, buffers, P.params, its, light)
            c, _ = oracle_mod.run(int(pass_), sc, P.params, its, light)
            bad = np.nonzero((g.view(np.uint32) != c.view(np.uint32)).any(axis=1))[0]
            assert len(bad) == 0, f"{pass_.name}: {len(bad)} of {len(its)} records differ"
    finally:
        gpu.set_pass_kernel(0)
        gpu.set_near(1)


def test_bake_watertight(gpu):
    """The device bake with the watertight test: equal to the host pipeline's watertight bake, and within
    1e-3 of the shader-test bake on all but a few texels (those whose rays through edges flipped)."""
    scene = scenes.small_map()
    wt_dev = lb.bake_device(scene, gpu, watertight=True)
    wt_host = lb.bake(scene, gpu, watertight=True)
    assert np.array_equal(wt_dev.direct, wt_host.direct)
    assert np.array_equal(wt_dev.indirect, wt_host.indirect)
    mt = lb.bake_device(scene, gpu)
    for name in ("direct", "indirect"):
        a, b = getattr(mt, name), getattr(wt_dev, name)
        off = np.abs(a - b) > 1e-3 * np.maximum(1.0, np.abs(a))
        texels = off.reshape(off.shape[0], off.shape[1], -1).any(axis=2)
        print(f"{name}: {int(texels.sum())} of {texels.size} texels beyond 1e-3 of the shader-test bake")
        assert texels.mean() < 0.01
