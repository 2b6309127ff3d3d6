"""The watertight triangle test in the oracle (the CPU restatement the kernels are checked against): it
closes the edges two triangles share, and away from edges it decides every ray as the shader's test does."""
import numpy as np

import lightbaker_b200 as lb
import oracle
from helpers import edge_crossing_rays
from lightbaker_b200 import scenes

NONE = 0xffffffff


def test_prepared_vertices_are_the_triangles():
    """Prepared.verts holds each BVH triangle's vertices: v0 as the record's, e1 and e2 their differences."""
    P = lb.prepare(scenes.small_map())
    V = P.verts.reshape(-1, 3, 3)
    assert len(V) == len(P.tris)
    assert np.array_equal(V[:, 0], P.tris["v0"][:, :3])
    assert np.array_equal((V[:, 1] - V[:, 0]).astype(np.float32), P.tris["e1"][:, :3])
    assert np.array_equal((V[:, 2] - V[:, 0]).astype(np.float32), P.tris["e2"][:, :3])


def test_watertight_closes_shared_edges():
    """Rays through points of shared edges, crossing the surface there: the watertight test meets one of
    the two triangles every time; the shader's Moller-Trumbore lets some through (counted)."""
    P = lb.prepare(scenes.small_map())
    rays, pairs = edge_crossing_rays(P.verts)
    assert len(rays) > 3000
    mt = oracle.trace_rays(oracle.Scene.of(P), P.params, rays, False)
    wt = oracle.trace_rays(oracle.Scene.of(P, watertight=True), P.params, rays, False)
    # the edge point lies 3 along each ray: a ray that gets through the edge misses, or meets neither of the
    # edge's triangles but a surface behind it
    def through(h):
        on_edge = (h[1] == pairs[:, 0]) | (h[1] == pairs[:, 1])
        return (h[1] == NONE) | (~on_edge & (h[0] > 3.01))
    mt_leaks, wt_leaks = int(through(mt).sum()), int(through(wt).sum())
    print(f"edge-crossing rays: {len(rays)}; through the edge: shader test {mt_leaks}, watertight {wt_leaks}")
    assert wt_leaks == 0


def test_watertight_agrees_with_the_shader_test_away_from_edges():
    """On the direct pass's rays (inside tests, sun, occlusion) of a sample of texels, the two tests agree
    on hit/miss for every ray not within 1e-4 of an edge (or_ray_ambiguous); where both hit, on the face
    and on t to 1e-5 relative, and on the triangle but between coincident ones (coplanar overlaps, where
    either test may pick either at the same t)."""
    P = lb.prepare(scenes.small_map())
    items = P.covered_texels()[::53][:300]
    rays = np.concatenate([oracle.rays_of(oracle.item_rays(0, P.params, it, i)) for i, it in enumerate(items)])
    mt = oracle.trace_rays(oracle.Scene.of(P), P.params, rays, False)
    wt = oracle.trace_rays(oracle.Scene.of(P, watertight=True), P.params, rays, False)
    amb = oracle.rays_ambiguous(oracle.Scene.of(P), P.params, rays, 1e-4)
    differ = (mt[1] == NONE) != (wt[1] == NONE)
    print(f"{len(rays)} rays, {int(amb.sum())} within 1e-4 of an edge, {int(differ.sum())} hit/miss differences")
    assert not np.any(differ & ~amb)
    both = (mt[1] != NONE) & (wt[1] != NONE) & ~amb
    assert np.array_equal(mt[2][both], wt[2][both])
    assert np.all(np.abs(mt[0][both] - wt[0][both]) <= 1e-5 * np.maximum(1.0, wt[0][both]))
    # another triangle only where two coincide (coplanar overlaps: the same t to rounding)
    other = both & (mt[1] != wt[1])
    assert np.all(np.abs(mt[0][other] - wt[0][other]) <= 1e-6 * np.maximum(1.0, wt[0][other]))
    # and with the FP64 walk
    f64 = oracle.trace_rays(oracle.Scene.of(P), P.params, rays, False, precision=64)
    assert not np.any(((f64[1] == NONE) != (wt[1] == NONE)) & ~amb)
