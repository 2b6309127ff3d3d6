"""Parity of the CUDA passes with the oracle, through the C ABI (lb_run): the direct, gather and volume
records must be bit-identical (the kernels and the oracle perform the same float operations in the
same order; shadow and occlusion masks, picks and shares are integer or exact). The walk's work counters
(rays, nodes fetched, triangles tested, materials read) must match the oracle's exactly too.
"""
import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    return oracle


def _light_for(P, rng):
    aw, ah = P.info.atlas_width, P.info.atlas_height
    light = rng.uniform(0.0, 3.0, size=(aw * ah, 4)).astype(np.float32)
    light[:, 3] = (rng.uniform(size=aw * ah) > 0.3).astype(np.float32)
    return light


def _compare(gpu_out, cpu_out, what):
    a = gpu_out.view(np.uint32)
    b = cpu_out.view(np.uint32)
    bad = np.nonzero((a != b).any(axis=1))[0]
    assert len(bad) == 0, f"{what}: {len(bad)} of {len(a)} records differ, first {bad[:5]}: " \
                          f"gpu {gpu_out[bad[:3]]} oracle {cpu_out[bad[:3]]}"


@pytest.mark.parametrize("kernel,order,bvh,refill,near",
                         [(0, 8, 2, 0, 0), (1, 8, 2, 0, 0), (1, 0, 2, 0, 0), (1, 1, 2, 1, 0), (1, 8, 2, 1, 0),
                          (1, 8, 8, 0, 0), (1, 0, 8, 0, 0), (1, 8, 2, 0, 1), (1, 0, 2, 0, 1)],
                         ids=["thread_per_item", "warp_shader_order", "warp_azimuth_wedges", "warp_patches_refill",
                              "warp_refill", "warp_bvh8", "warp_bvh8_wedges", "warp_leaf_lists",
                              "warp_leaf_lists_wedges"])
@pytest.mark.parametrize("name,limit", [("reference_test", 20000), ("small_map", 20000), ("map_100m", 3000)])
def test_passes_bit_exact(gpu, oracle_mod, name, limit, kernel, order, bvh, refill, near):
    scene = scenes.WORKLOADS[name]()
    P = lb.prepare(scene)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    sc = oracle_mod.Scene.of(P)
    rng = np.random.default_rng(1)
    items = P.covered_texels()
    # a spread sample across the map, in list order (keys follow the index)
    idx = np.sort(rng.choice(len(items), size=min(limit, len(items)), replace=False))
    items = items[idx]
    gpu.set_pass_kernel(kernel)
    gpu.set_ray_order(order, order)
    gpu.set_bvh(bvh)
    gpu.set_refill(refill)
    gpu.set_near(near)
    gpu.set_counting(True)
    g = gpu.run(lb.Pass.DIRECT, buffers, P.params, items)
    gc = gpu.counters()
    c, cc = oracle_mod.run(0, sc, P.params, items)
    _compare(g, c, f"{name} direct")
    # the BVH2 walks fetch, test and read exactly what the oracle does; the 8-wide walk its own amounts
    for k in ("rays", "nodes", "tris", "mats") if bvh == 2 and not near else ("rays",):
        assert gc[k] == cc[k], f"direct {k}: gpu {gc[k]} oracle {cc[k]}"
    assert cc["overflows"] == 0
    light = _light_for(P, rng)
    gi = items[: limit // 4]
    g = gpu.run(lb.Pass.GATHER, buffers, P.params, gi, light)
    gc = gpu.counters()
    c, cc = oracle_mod.run(1, sc, P.params, gi, light)
    _compare(g, c, f"{name} gather")
    # (with leaf lists a gather ray that finds its hit nearby never walks the tree)
    for k in ("rays", "nodes", "tris", "mats") if bvh == 2 and not (near and kernel == 1) else ("rays",):
        assert gc[k] == cc[k], f"gather {k}: gpu {gc[k]} oracle {cc[k]}"
    probes = np.zeros(500, lb.TEXEL)
    probes["pos"][:, :3] = rng.uniform(0, 1, size=(500, 3)) * np.array([P.nodes[0]["max"] - P.nodes[0]["min"]]) + \
        P.nodes[0]["min"]
    probes["pos"][:, 3] = 1.0
    probes["normal"][:, 1] = 1.0
    probes["normal"][:, 3] = np.arange(500, dtype=np.uint32).view(np.float32)
    g = gpu.run(lb.Pass.VOLUME, buffers, P.params, probes, light)
    c, _ = oracle_mod.run(2, sc, P.params, probes, light)
    _compare(g, c, f"{name} volume")
    gpu.set_counting(False)
    gpu.set_pass_kernel(0)
    gpu.set_ray_order(8, 8)
    gpu.set_bvh(2)
    gpu.set_refill(0)
    gpu.set_near(1)


@pytest.mark.parametrize("cap,near", [(3, 1), (4, 1), (3, 0), (4, 0)])
@pytest.mark.parametrize("name,limit", [("small_map", 12000), ("map_100m", 3000)])
def test_register_capped_passes_bit_exact(gpu, oracle_mod, name, limit, cap, near):
    """The register-capped warp kernels (their own instantiations, used without counting) give the oracle's
    records too."""
    scene = scenes.WORKLOADS[name]()
    P = lb.prepare(scene)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    sc = oracle_mod.Scene.of(P)
    rng = np.random.default_rng(2)
    items = P.covered_texels()
    items = items[np.sort(rng.choice(len(items), size=min(limit, len(items)), replace=False))]
    gpu.set_pass_kernel(1)
    gpu.set_ray_order(0, 0)
    gpu.set_near(near)
    gpu.set_register_cap(cap)
    try:
        g = gpu.run(lb.Pass.DIRECT, buffers, P.params, items)
        c, _ = oracle_mod.run(0, sc, P.params, items)
        _compare(g, c, f"{name} direct, cap {cap}")
        light = _light_for(P, rng)
        gi = items[: limit // 4]
        g = gpu.run(lb.Pass.GATHER, buffers, P.params, gi, light)
        c, _ = oracle_mod.run(1, sc, P.params, gi, light)
        _compare(g, c, f"{name} gather, cap {cap}")
    finally:
        gpu.set_register_cap(0)
        gpu.set_pass_kernel(0)
        gpu.set_ray_order(8, 8)
        gpu.set_near(1)


def test_empty_and_edge_cases(gpu, oracle_mod):
    P = lb.prepare(scenes.small_map())
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    # no items: an empty result (gpu/mod.rs:143-145)
    assert gpu.run(lb.Pass.DIRECT, buffers, P.params, np.zeros(0, lb.TEXEL)).shape == (0, 4)
    # one item, and a list whose keys wrap u32 (index * 7919)
    items = P.covered_texels()[:3]
    g = gpu.run(lb.Pass.DIRECT, buffers, P.params, items[:1])
    c, _ = oracle_mod.run(0, oracle_mod.Scene.of(P), P.params, items[:1])
    _compare(g, c, "one item")
    # a scene with no casting triangle: the reference's one-node BVH; every ray escapes
    nodes = np.zeros(1, lb.NODE)
    nodes[0]["min"] = np.finfo(np.float32).max
    nodes[0]["max"] = -np.finfo(np.float32).max
    tris = np.zeros(1, lb.TRI)
    empty = gpu.scene(nodes, tris, P.materials, np.zeros((0, 8), np.float32))
    g = gpu.run(lb.Pass.DIRECT, empty, P.params, items)
    c, _ = oracle_mod.run(0, oracle_mod.Scene(nodes, tris, P.materials, np.zeros((0, 8), np.float32)), P.params, items)
    _compare(g, c, "empty scene")
    assert np.all(g[:, 2] == 0.0)  # no occlusion


def test_opacity_coin(gpu, oracle_mod):
    """Materials that stop only part of the light (trace.wgsl:69-72): the coin per (triangle, ray)."""
    P = lb.prepare(scenes.small_map())
    mats = P.materials.copy()
    mats[1:, 3] = np.linspace(0.1, 0.9, len(mats) - 1)
    buffers = gpu.scene(P.nodes, P.tris, mats, P.charts)
    items = P.covered_texels()[::7][:5000]
    g = gpu.run(lb.Pass.DIRECT, buffers, P.params, items)
    c, _ = oracle_mod.run(0, oracle_mod.Scene(P.nodes, P.tris, mats, P.charts), P.params, items)
    _compare(g, c, "opacity")


def test_bake_matches_oracle_bake(gpu, oracle_mod):
    """The whole drop-in bake: CUDA passes vs the oracle's, same host pipeline: identical atlases."""
    s = scenes.small_map()
    t, keep = oracle_mod.tracer()
    a = lb.bake(s, gpu)
    b = lb.bake_with(s, t)
    assert np.array_equal(a.direct.view(np.uint32), b.direct.view(np.uint32))
    assert np.array_equal(a.indirect.view(np.uint32), b.indirect.view(np.uint32))
    assert np.array_equal(a.validity, b.validity)
    assert np.array_equal(a.volume.view(np.uint32), b.volume.view(np.uint32))
    assert a.stats.rays == b.stats.rays
    assert a.write()[64:] != b""


@pytest.mark.parametrize("near", [0, 1])
@pytest.mark.parametrize("name,limit", [("small_map", 12000), ("map_100m", 3000)])
def test_dynamic_fetch_bit_exact(gpu, oracle_mod, name, limit, near):
    """Warps taking their next item from a work counter (lb_set_fetch) give the same records: an item's
    keys are its index in the list, whichever warp takes it."""
    scene = scenes.WORKLOADS[name]()
    P = lb.prepare(scene)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    sc = oracle_mod.Scene.of(P)
    rng = np.random.default_rng(5)
    items = P.covered_texels()
    items = items[np.sort(rng.choice(len(items), size=min(limit, len(items)), replace=False))]
    gpu.set_pass_kernel(1)
    gpu.set_near(near)
    gpu.set_fetch(True)
    try:
        for rep in range(2):  # the counter starts again from zero at every launch
            g = gpu.run(lb.Pass.DIRECT, buffers, P.params, items)
            c, _ = oracle_mod.run(0, sc, P.params, items)
            _compare(g, c, f"{name} direct, fetch")
            light = _light_for(P, rng)
            gi = items[: limit // 4]
            g = gpu.run(lb.Pass.GATHER, buffers, P.params, gi, light)
            c, _ = oracle_mod.run(1, sc, P.params, gi, light)
            _compare(g, c, f"{name} gather, fetch")
    finally:
        gpu.set_fetch(False)
        gpu.set_pass_kernel(0)
        gpu.set_near(1)
        buffers.close()


@pytest.mark.parametrize("watertight", [False, True])
@pytest.mark.parametrize("name,limit", [("small_map", 12000), ("map_100m", 4000), ("uneven_tiles", 4000)])
def test_warp_walk_sun_rays_bit_exact(gpu, oracle_mod, name, limit, watertight):
    """A texel's sun rays walked together by the warp (lb_set_warp_walk) give the same shadow bits as their own
    walks: the direct records equal the oracle's, with the shader's triangle test and the watertight one."""
    scene = scenes.WORKLOADS[name]() if name != "uneven_tiles" else scenes.uneven_tiles(seed=2, tiles=3)
    P = lb.prepare(scene)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    if watertight:
        buffers.set_vertices(P.verts)
    sc = oracle_mod.Scene.of(P, watertight=watertight)
    rng = np.random.default_rng(9)
    items = P.covered_texels()
    items = items[np.sort(rng.choice(len(items), size=min(limit, len(items)), replace=False))]
    gpu.set_pass_kernel(1)
    try:
        for near in (0, 1):
            gpu.set_near(near)
            for ww in (True, False):
                gpu.set_warp_walk(ww)
                g = gpu.run(lb.Pass.DIRECT, buffers, P.params, items)
                c, _ = oracle_mod.run(0, sc, P.params, items)
                _compare(g, c, f"{name} direct, warp walk {ww}, near {near}")
    finally:
        gpu.set_warp_walk(True)
        gpu.set_near(1)
        gpu.set_pass_kernel(0)
        buffers.close()
