"""The 8-wide BVH built on the device at scene upload (bvh8_build.cu) against the host collapse
(lb_bvh8_collapse) of the same BVH2: equal byte for byte, nodes and triangles, on the workloads, the
reference's empty BVH and a leaf of 70 triangles. The walks over it (lb_set_bvh 8) are checked against
the oracle in test_passes_gpu.py and test_watertight_gpu.py."""
import time

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


def _upload(gpu, nodes, tris):
    return gpu.scene(nodes, tris, np.zeros((1, 4), np.float32), np.zeros((0, 8), np.float32))


def _check(gpu, nodes, tris, label):
    t0 = time.perf_counter()
    buffers = _upload(gpu, nodes, tris)
    t1 = time.perf_counter()
    dn, dt = buffers.bvh8()
    t2 = time.perf_counter()
    hn, ht = lb.bvh8_collapse(nodes, tris)
    t3 = time.perf_counter()
    print(f"{label}: {len(nodes)} BVH2 nodes -> {len(hn)} 8-wide nodes, {len(ht)} triangles; upload with the "
          f"device build {t1 - t0:.3f} s, host collapse {t3 - t2:.3f} s")
    assert dn.shape == hn.shape and dt.shape == ht.shape, label
    bad = np.nonzero((dn != hn).any(axis=1))[0]
    assert len(bad) == 0, f"{label}: {len(bad)} of {len(hn)} nodes differ, first {bad[:5]}"
    assert np.array_equal(dt, ht), f"{label}: triangles differ"
    buffers.close()


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m", "uneven_tiles"])
def test_device_bvh8_equals_host(gpu, name):
    P = lb.prepare(scenes.WORKLOADS[name]())
    _check(gpu, P.nodes, P.tris, name)


def test_device_bvh8_empty_and_big_leaf(gpu):
    nodes = np.zeros(1, lb.NODE)
    nodes[0]["min"] = np.finfo(np.float32).max
    nodes[0]["max"] = -np.finfo(np.float32).max
    _check(gpu, nodes, np.zeros(1, lb.TRI), "empty")
    rng = np.random.default_rng(0)
    for count in (3, 70, 300):
        tris = np.zeros(count, lb.TRI)
        tris["v0"][:, :3] = rng.uniform(0, 1, (count, 3))
        tris["e1"][:, :3] = rng.uniform(0, 0.1, (count, 3))
        tris["e2"][:, :3] = rng.uniform(0, 0.1, (count, 3))
        v = np.concatenate([tris["v0"][:, :3], tris["v0"][:, :3] + tris["e1"][:, :3],
                            tris["v0"][:, :3] + tris["e2"][:, :3]])
        nodes = np.zeros(1, lb.NODE)
        nodes[0]["min"], nodes[0]["max"] = v.min(0), v.max(0)
        nodes[0]["first"], nodes[0]["count"] = 0, count
        _check(gpu, nodes, tris, f"one leaf of {count}")


def test_upload_rejects_leaf_past_triangles(gpu):
    nodes = np.zeros(1, lb.NODE)
    nodes[0]["first"], nodes[0]["count"] = 0, 5
    with pytest.raises(lb.LightbakerError, match="leaf 0 reaches past the triangle array"):
        _upload(gpu, nodes, np.zeros(4, lb.TRI))


def test_upload_rejects_cyclic_bvh(gpu):
    """An inner node whose child points back at it would make every walk loop: refused before the upload."""
    nodes = np.zeros(3, lb.NODE)
    nodes[0]["first"], nodes[0]["count"] = 1, 0
    nodes[1]["first"], nodes[1]["count"] = 0, 0
    nodes[2]["first"], nodes[2]["count"] = 0, 2
    with pytest.raises(lb.LightbakerError, match="not a tree node"):
        _upload(gpu, nodes, np.zeros(4, lb.TRI))
