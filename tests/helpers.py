"""Shared helpers for the tests: the reference test's lookups (crates/lightbaker/tests/bake.rs:74-89)."""
import math

import numpy as np


def ground_texel(scene_positions_ground, prepared_charts, tri_chart_ground, tiles_of_chart, width, x, z):
    raise NotImplementedError


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
