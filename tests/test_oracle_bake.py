"""The oracle's whole bake (oracle/bake_ref.py + bake_ref.cpp: the reference's bake.rs, raster.rs and
volume.rs restated independently of the product) against the product's host pipeline (csrc/host, the
drop-in bake) running the same oracle tracer, on the CPU: the Params, the charts' affines, every
tile's texels, and the finished atlases and volume must be the same bits."""
import numpy as np
import pytest

import lightbaker_b200 as lb
import oracle
from lightbaker_b200 import scenes
from oracle.bake_ref import OracleBake, chart_affines, make_params, raster_tile, read_scene


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_same(name, a, b):
    d = np.nonzero(bits(a) != bits(b))
    assert len(d[0]) == 0, f"{name}: {len(d[0])} values differ, first at {[x[:3] for x in d]}"


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_params_affines_and_raster(name):
    s = scenes.WORKLOADS[name]()
    P = lb.prepare(s)
    header, positions = read_scene(s)
    p = make_params(header, int(P.info.atlas_width), int(P.info.atlas_height))
    assert bytes(memoryview(p)) == bytes(memoryview(P.params))
    lm = header["lightmap"]
    layout = P.layout()
    assert_same("affines", chart_affines(layout, P.tiles, np.float32(lm["texelsPerMeter"]), int(lm["padding"])),
                P.charts)
    tiles = range(len(P.tiles)) if name != "map_100m" else range(0, len(P.tiles), 7)
    for t in tiles:
        mine = raster_tile(layout, P.tiles[t], t, positions, np.float32(lm["texelsPerMeter"]), int(lm["padding"]))
        assert_same(f"tile {t} texels", mine.view(np.uint32), P.rasterize(t).reshape(-1).view(np.uint32))
        if name == "reference_test":
            assert (mine["pos"][:, 3] > 0.5).any()


@pytest.mark.parametrize("name", ["reference_test", "small_map"])
def test_oracle_bake_equals_host_pipeline(name):
    s = scenes.WORKLOADS[name]()
    P = lb.prepare(s)
    ob = OracleBake(s, P)
    t, keep = oracle.tracer()
    hb = lb.bake_with(s, t)
    assert_same("direct atlas", ob.direct, hb.direct)
    assert_same("validity", ob.validity, hb.validity)
    assert_same("indirect atlas", ob.indirect, hb.indirect)
    assert_same("volume", ob.volume, hb.volume)
    assert (ob.rays["direct"], ob.rays["gather"], ob.rays["volume"]) == (
        hb.stats.rays_direct, hb.stats.rays_gather, hb.stats.rays_volume)
    # every validity code the bake writes is exercised on the small map (offset, pushed, filled, volume)
    if name == "small_map":
        counts = np.bincount(ob.validity.reshape(-1), minlength=6)
        assert (counts[1:] > 0).all(), counts


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m", "uneven_tiles"])
def test_bvh_equals_oracle_build(name):
    """bvh.rs:50-162 restated independently (oracle/bvh_ref.cpp, serial): the product's parallel build gives
    the same nodes and triangles byte for byte."""
    from oracle.bake_ref import build_bvh
    s = scenes.WORKLOADS[name]() if name != "uneven_tiles" else scenes.uneven_tiles(seed=1, tiles=4,
                                                                                     tri_range=(2_000, 40_000))
    P = lb.prepare(s)
    nodes, tris = build_bvh(s, P.layout())
    assert_same("nodes", nodes.reshape(-1), P.nodes.view(np.uint32).reshape(-1))
    assert_same("triangles", tris.reshape(-1), P.tris.view(np.uint32).reshape(-1))


@pytest.mark.parametrize("name", ["opacity", "casts_only", "degenerate", "no_bounce", "night", "inside",
                                  "nothing_received", "nothing_casts"])
def test_edge_scenes_equal_oracle_bake(name):
    """The edge scenes (tests/edge_scenes.py): the opacity coin, casters that are not laid out and receivers
    that cast nothing, degenerate and sub-texel triangles, no bounce, no sun, texels inside solids. The host
    pipeline on the oracle's tracer equals the oracle's whole bake, BVH included."""
    from edge_scenes import EDGE_SCENES
    from oracle.bake_ref import build_bvh
    s = EDGE_SCENES[name]()
    P = lb.prepare(s)
    nodes, tris = build_bvh(s, P.layout())
    assert_same("nodes", nodes.reshape(-1), P.nodes.view(np.uint32).reshape(-1))
    assert_same("triangles", tris.reshape(-1), P.tris.view(np.uint32).reshape(-1))
    ob = OracleBake(s, P)
    t, keep = oracle.tracer()
    hb = lb.bake_with(s, t)
    assert_same("direct atlas", ob.direct, hb.direct)
    assert_same("validity", ob.validity, hb.validity)
    assert_same("indirect atlas", ob.indirect, hb.indirect)
    if ob.volume is not None or hb.volume is not None:
        assert_same("volume", ob.volume, hb.volume)
    assert ob.rays["direct"] == hb.stats.rays_direct and ob.rays["gather"] == hb.stats.rays_gather
