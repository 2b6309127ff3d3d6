"""Shared helpers for the tests: the reference test's lookups (crates/lightbaker/tests/bake.rs:74-89)."""
import math

import numpy as np


def affine_texel(chart_rows, p):
    """floor of a chart's affine rows applied to a world point: (atlas x, atlas y)."""
    r0, r1 = chart_rows[:4], chart_rows[4:]
    q = np.array([p[0], p[1], p[2], 1.0], np.float32)
    x = np.float32(0)
    y = np.float32(0)
    for k in range(4):
        x = np.float32(x + np.float32(r0[k] * q[k]))
        y = np.float32(y + np.float32(r1[k] * q[k]))
    return int(math.floor(x)), int(math.floor(y))


def edge_crossing_rays(verts, seed=0, fractions=(0.5, 0.25, 1.0 / 3.0), length=3.0):
    """Rays through points of the edges two triangles share, crossing the surface there: for each shared
    edge (a, b) and fraction f, the float point a (1 - f) + b f, a downward direction tilted at random,
    starting `length` before the point. Kept only where the ray sees both triangles from the same side
    (the surface really crosses the ray at the edge; at a fold the ray only touches the edge line).
    Returns a RAY array (oracle.RAY layout) and the pairs of triangles."""
    import oracle
    V = np.asarray(verts, np.float32).reshape(-1, 3, 3)
    edges = {}
    for i, tri in enumerate(V):
        for a, b in ((0, 1), (1, 2), (2, 0)):
            ka, kb = tuple(tri[a].tolist()), tuple(tri[b].tolist())
            edges.setdefault((min(ka, kb), max(ka, kb)), []).append(i)
    shared = [(k, v) for k, v in edges.items() if len(v) == 2]
    normals = np.cross((V[:, 1] - V[:, 0]).astype(np.float64), (V[:, 2] - V[:, 0]).astype(np.float64))
    rng = np.random.default_rng(seed)
    rays, pairs = [], []
    for (a, b), ts in shared:
        a = np.array(a, np.float32)
        b = np.array(b, np.float32)
        for f in fractions:
            p = (a * np.float32(1.0 - f) + b * np.float32(f)).astype(np.float32)
            d = np.array([rng.normal() * 0.3, -1.0, rng.normal() * 0.3])
            d = (d / np.linalg.norm(d)).astype(np.float32)
            s0, s1 = np.sign(normals[ts[0]] @ d), np.sign(normals[ts[1]] @ d)
            if s0 == 0 or s0 != s1:
                continue
            rays.append(((p - d * np.float32(length)).astype(np.float32), d))
            pairs.append(ts)
    out = np.zeros(len(rays), oracle.RAY)
    for i, (o, d) in enumerate(rays):
        out[i]["o"], out[i]["d"], out[i]["tmax"], out[i]["key"] = o, d, np.float32(2 * length), i
    return out, np.array(pairs, np.int64).reshape(-1, 2)
