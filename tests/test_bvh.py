"""The BVHs: the reference's BVH2 as the host builds it (crates/lightbaker/src/bvh.rs:50-106) and the
8-wide BVH collapsed from it for the device."""
import ctypes as C

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import _native as N
from lightbaker_b200 import scenes


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_bvh2_structure(name):
    P = lb.prepare(scenes.WORKLOADS[name]())
    n, t = P.nodes, P.tris
    seen = np.zeros(len(t), int)
    stack = [0]
    while stack:
        i = stack.pop()
        if n["count"][i] > 0:
            f, c = n["first"][i], n["count"][i]
            seen[f:f + c] += 1
            v0 = t["v0"][f:f + c, :3]
            for corner in (v0, v0 + t["e1"][f:f + c, :3], v0 + t["e2"][f:f + c, :3]):
                assert np.all(corner >= n["min"][i] - 1e-4) and np.all(corner <= n["max"][i] + 1e-4)
        else:
            for ch in (n["first"][i], n["first"][i] + 1):
                assert np.all(n["min"][ch] >= n["min"][i]) and np.all(n["max"][ch] <= n["max"][i])
                stack.append(ch)
    assert np.all(seen == 1)
    # leaves of at most 4 (bvh.rs:10) unless no split beats a leaf
    assert n["count"].max() <= 4


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_bvh2_bytes_are_the_serial_builds(name):
    """The BVH2's bytes (node order, triangle order: the opacity coin and the hit indices depend on them)
    equal those of the serial build the golden hashes were made with (tests/golden/make_bvh_hashes.py)."""
    import json
    from pathlib import Path
    want = json.loads((Path(__file__).parent / "golden" / "bvh_hashes.json").read_text())[name]
    P = lb.prepare(scenes.WORKLOADS[name]())
    assert (len(P.nodes), len(P.tris)) == (want["nodes"], want["tris"])
    assert lb.blake3(P.nodes.tobytes() + P.tris.tobytes()).hex() == want["blake3"]


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_bvh8_collapse(name):
    P = lb.prepare(scenes.WORKLOADS[name]())
    n8, depth = C.c_uint64(), C.c_uint64()
    N.check(N.lib().lb_bvh8_check(N.ptr(P.nodes), len(P.nodes), N.ptr(P.tris), len(P.tris), C.byref(n8),
                                  C.byref(depth)), "bvh8")
    # fewer, shallower nodes: about a seventh of the BVH2's
    assert n8.value < len(P.nodes) / 3
    assert depth.value * 7 < 96


def test_bvh8_empty_and_big_leaves():
    nodes = np.zeros(1, lb.NODE)
    nodes[0]["min"] = np.finfo(np.float32).max
    nodes[0]["max"] = -np.finfo(np.float32).max
    tris = np.zeros(1, lb.TRI)
    N.check(N.lib().lb_bvh8_check(N.ptr(nodes), 1, N.ptr(tris), 1, None, None), "empty")
    # one leaf of 70 triangles (no split beat a leaf): split into slots of 4 over extra nodes
    rng = np.random.default_rng(0)
    tris = np.zeros(70, lb.TRI)
    tris["v0"][:, :3] = rng.uniform(0, 1, (70, 3))
    tris["e1"][:, :3] = rng.uniform(0, 0.1, (70, 3))
    tris["e2"][:, :3] = rng.uniform(0, 0.1, (70, 3))
    v = np.concatenate([tris["v0"][:, :3], tris["v0"][:, :3] + tris["e1"][:, :3], tris["v0"][:, :3] + tris["e2"][:, :3]])
    nodes = np.zeros(1, lb.NODE)
    nodes[0]["min"], nodes[0]["max"] = v.min(0), v.max(0)
    nodes[0]["first"], nodes[0]["count"] = 0, 70
    N.check(N.lib().lb_bvh8_check(N.ptr(nodes), 1, N.ptr(tris), 70, None, None), "big leaf")


@pytest.mark.parametrize("name", ["reference_test", "small_map"])
def test_bvh8_collapse_export(name):
    """lb_bvh8_collapse (the host collapse the device build is checked against): the node count of
    lb_bvh8_check, every triangle once (e2.w a permutation of the BVH2's triangle indices, the triangle
    otherwise unchanged), and the root's inner children numbered from 1."""
    P = lb.prepare(scenes.WORKLOADS[name]())
    n8 = C.c_uint64()
    N.check(N.lib().lb_bvh8_check(N.ptr(P.nodes), len(P.nodes), N.ptr(P.tris), len(P.tris), C.byref(n8), None), "bvh8")
    nodes, tris = lb.bvh8_collapse(P.nodes, P.tris)
    assert len(nodes) == n8.value and len(tris) == len(P.tris)
    orig = tris[:, 11]
    assert np.array_equal(np.sort(orig), np.arange(len(P.tris)))
    src = P.tris.view(np.uint32).reshape(-1, 12)[orig]
    assert np.array_equal(tris[:, :11], src[:, :11])
    assert nodes[0, 4] == 1 and (nodes[0, 3] >> 24) != 0
