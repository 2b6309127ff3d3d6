"""The device-resident bake (one CUDA graph over every dirty tile) against the drop-in bake (the CUDA
passes with the host's texel passes between them, already checked against the oracle): every output
must be bit-identical — atlases, validity, the volume — and the ray counts equal. The cache must work
the same (a second bake bakes nothing; a moved box rebakes only the tiles it reaches), and a bake that
reads some tiles from the cache must match one that bakes them all."""
import shutil
import tempfile

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


def same(a, b):
    assert np.array_equal(a.direct.view(np.uint32), b.direct.view(np.uint32)), "direct atlas"
    assert np.array_equal(a.validity, b.validity), "validity"
    d = np.nonzero((a.indirect.view(np.uint32) != b.indirect.view(np.uint32)).any(axis=2))
    assert len(d[0]) == 0, f"indirect atlas: {len(d[0])} texels differ, e.g. {a.indirect[d][:3]} vs {b.indirect[d][:3]}"
    if a.volume is not None:
        assert np.array_equal(a.volume.view(np.uint32), b.volume.view(np.uint32)), "volume"


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_device_bake_equals_drop_in(gpu, name):
    s = scenes.WORKLOADS[name]()
    plain = lb.bake(s, gpu)
    dev = lb.bake_device(s, gpu)
    same(dev, plain)
    assert dev.stats.rays_direct == plain.stats.rays_direct
    # later bounces evaluate the first bounce's records: only its gather rays are traced
    bounces = lb.prepare(s).info.gi_bounces
    assert dev.stats.rays_gather * bounces == plain.stats.rays_gather
    assert dev.stats.rays_volume == plain.stats.rays_volume
    assert dev.stats.tiles_baked == plain.stats.tiles_baked
    # tracing every bounce again gives the same bits and the drop-in's ray count
    again = lb.bake_device(s, gpu, trace_every_bounce=True)
    same(again, plain)
    assert again.stats.rays_gather == plain.stats.rays_gather


def test_uneven_tiles_in_one_graph(gpu):
    """Tiles whose triangle counts (lognormal, 2k to 40k) and atlas regions differ by an order of magnitude,
    all rebaked in one graph with the autotuner on: the same bits as the drop-in bake."""
    s = scenes.uneven_tiles(seed=1, tiles=4, tri_range=(2_000, 40_000), bounces=2)
    P = lb.prepare(s)
    areas = [int(t["w"]) * int(t["h"]) for t in P.tiles]
    assert max(areas) >= 8 * min(areas)
    plain = lb.bake(s, gpu)
    dev = lb.bake_device(s, gpu, autotune=True)
    same(dev, plain)
    assert dev.stats.rays_gather * 2 == plain.stats.rays_gather and dev.stats.tiles_baked == len(areas)


def test_autotuned_device_bake_equals_drop_in(gpu):
    s = scenes.small_map()
    logs = []
    dev = lb.bake_device(s, gpu, autotune=True, log=logs.append)
    assert any(l.startswith("autotune:") for l in logs), logs
    same(dev, lb.bake(s, gpu))


def test_plan_replays_identically(gpu):
    s = scenes.small_map()
    p = lb.Plan(s, gpu)
    p.launch()
    a = p.result()
    rays = p.rays()
    p.launch()
    p.launch()
    b = p.result()
    assert p.rays() == rays
    same(a, b)
    p.close()


def test_device_bake_cache(gpu):
    d = tempfile.mkdtemp(prefix="lightbaker-dev-")
    try:
        full = lb.bake_device(scenes.reference_test(8.0), gpu, cache=d)
        again = lb.bake_device(scenes.reference_test(8.0), gpu, cache=d)
        assert again.stats.tiles_baked == 0 and again.stats.chunks_baked == 0
        same(again, full)
        moved = lb.bake_device(scenes.reference_test(6.0), gpu, cache=d)
        assert 0 < moved.stats.tiles_baked < moved.stats.tiles
        # the drop-in bake of the moved scene from the same cache state gives the same atlas
        d2 = tempfile.mkdtemp(prefix="lightbaker-plain-")
        try:
            lb.bake(scenes.reference_test(8.0), gpu, cache=d2)
            moved_plain = lb.bake(scenes.reference_test(6.0), gpu, cache=d2)
            same(moved, moved_plain)
        finally:
            shutil.rmtree(d2, ignore_errors=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_device_raster_equals_host(gpu, name):
    """The device bake rasterises its tiles on the GPU (raster.cu): every texel record, covered or not,
    equals the host rasteriser's (raster.rs:39-114) bit for bit, tile after tile in the plan's order."""
    scene = scenes.WORKLOADS[name]()
    P = lb.prepare(scene)
    tr = lb.Transport(scene, gpu)
    try:
        dev = tr.export("texels").reshape(-1, 16).view(np.uint32)
    finally:
        tr.close()
    host = np.concatenate([P.rasterize(t).reshape(-1) for t in range(len(P.tiles))])
    host = host.view(np.float32).reshape(-1, 16).view(np.uint32)
    assert dev.shape == host.shape
    bad = np.nonzero((dev != host).any(axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} of {len(host)} texels differ, first {bad[:5]}"
    assert (host.view(np.float32)[:, 3] > 0.5).sum() > 0
