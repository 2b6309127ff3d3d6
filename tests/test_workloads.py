"""The synthetic workloads hold the shapes their configurations state."""
import json
import struct

import numpy as np

import lightbaker_b200 as lb
from lightbaker_b200 import scenes


def header(scene: bytes) -> dict:
    n = struct.unpack_from("<I", scene, 8)[0]
    return json.loads(scene[12:12 + n])


def test_uneven_tiles_is_the_batching_configuration():
    """64 tiles whose triangle counts are lognormal over 5k-500k and whose atlas regions run from 64^2 to
    512^2 texels; the small plain bake's rays: 64 occlusion rays at 2 m, one bounce of 64 gather rays."""
    s = scenes.uneven_tiles()
    h = header(s)
    tris = np.array(h["user"]["tile_triangles"])
    assert len(tris) == 64 and tris.min() >= 5_000 and tris.max() <= 500_000
    assert tris.max() / tris.min() > 20
    b = h["bake"]
    assert (b["aoRays"], b["aoReach"], b["giRays"], b["giBounces"]) == (64, 2.0, 64, 1)
    P = lb.prepare(s)
    areas = np.array([t["w"] * t["h"] for t in P.tiles])
    assert len(areas) == 64
    assert areas.min() >= 64 * 64 and areas.max() <= 512 * 512 and areas.max() / areas.min() > 20
