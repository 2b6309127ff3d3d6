"""Small scenes at the edges of the bake's behaviour, for parity tests (each a few thousand rays):

  opacity        a leafy canopy of material opacity 0.5 over the ground: the opacity coin
                 (trace.wgsl:69-72) decides each hit
  casts_only     a caster that is not laid out (receives false) and a receiver that casts nothing
  degenerate     zero-area and sliver triangles, and triangles far smaller than a texel (the rasteriser's
                 conservative pass, raster.rs:49-51)
  no_bounce      giBounces 0 (no gather pass), no volume
  night          the sun below the horizon (no sun ray is cast), one bounce from the sky alone
  nothing_received / nothing_casts   no chart at all; the empty BVH
  inside         boxes sunk into each other and into the ground, and a plate just under a box's top: texels
                 inside solids, sample points moved and pushed, the volume's fallback
"""
import numpy as np

from lightbaker_b200 import scenes as S


def _lightmap(width=256, tpm=8.0):
    return {"texelsPerMeter": tpm, "tileSize": 16.0, "chartAngleDeg": 40.0, "padding": 2, "atlasWidth": width,
            "indirectDownscale": 2}


SKY = {"zenith": [0.5, 0.6, 0.8], "horizon": [0.4, 0.45, 0.5], "ground": [0.2, 0.2, 0.2]}
SUN = {"direction": S.sun_direction(40.0, 130.0), "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}


def ground(size=12.0, step=1.0, seed=0):
    rng = np.random.default_rng(seed)
    h = rng.uniform(0.0, 0.2, size=(64, 64))
    return S.heightfield(0.0, 0.0, size, size, step,
                         lambda X, Z: h[np.clip(X.astype(int), 0, 63), np.clip(Z.astype(int), 0, 63)])


def opacity():
    mats = [S._material("ground", [0.5, 0.5, 0.5]), S._material("leaves", [0.2, 0.6, 0.2], opacity=0.5)]
    canopy = S.heightfield(2.0, 2.0, 8.0, 8.0, 0.5, lambda X, Z: 3.0 + 0.0 * X)
    bake = S._defaults_bake(aoRays=64, giRays=64, giBounces=1)
    vol = {"min": [0.5, 0.5, 0.5], "max": [11.5, 4.5, 11.5], "step": 1.0, "rays": 32}
    return S._assemble([("ground", 0, ground()), ("canopy", 1, canopy)], mats, SUN, SKY, _lightmap(), bake, vol)


def casts_only():
    mats = [S._material("ground", [0.5, 0.5, 0.5], casts=False), S._material("blocker", [0.8, 0.2, 0.2], receives=False),
            S._material("box", [0.3, 0.3, 0.9])]
    bake = S._defaults_bake(aoRays=32, giRays=32, giBounces=2)
    groups = [("ground", 0, ground()), ("blocker", 1, S.cube((3, 0, 3), (5, 3, 5))),
              ("box", 2, S.cube((7, 0, 6), (9, 2, 8)))]
    return S._assemble(groups, mats, SUN, SKY, _lightmap(), bake, None)


def degenerate():
    mats = [S._material("ground", [0.5, 0.5, 0.5]), S._material("bits", [0.7, 0.7, 0.2])]
    bits = []
    rng = np.random.default_rng(3)
    for k in range(40):
        c = rng.uniform(1.0, 11.0, 3) * np.array([1, 0.1, 1]) + np.array([0, 0.3, 0])
        e = rng.uniform(-1, 1, (2, 3)) * (0.02 if k % 2 else 0.3)
        bits += [tuple(c), tuple(c + e[0]), tuple(c + e[1])]
    bits += [(4.0, 1.0, 4.0), (5.0, 1.0, 4.0), (6.0, 1.0, 4.0)]          # zero area (collinear)
    bits += [(4.0, 1.5, 6.0), (4.0, 1.5, 6.0), (4.5, 1.5, 6.2)]          # a repeated vertex
    bits += [(8.0, 2.0, 2.0), (8.0 + 1e-4, 2.0, 2.0), (8.0, 3.0, 2.0)]   # a sliver
    bake = S._defaults_bake(aoRays=32, giRays=32, giBounces=1)
    return S._assemble([("ground", 0, ground()), ("bits", 1, bits)], mats, SUN, SKY, _lightmap(), bake, None)


def no_bounce():
    mats = [S._material("ground", [0.5, 0.5, 0.5]), S._material("box", [0.6, 0.3, 0.2])]
    bake = S._defaults_bake(aoRays=32, giRays=32, giBounces=0)
    groups = [("ground", 0, ground()), ("box", 1, S.cube((4, 0, 4), (6, 2.5, 7)))]
    return S._assemble(groups, mats, SUN, SKY, _lightmap(), bake, None)


def night():
    mats = [S._material("ground", [0.5, 0.5, 0.5]), S._material("box", [0.6, 0.3, 0.2])]
    sun = {"direction": [0.3, -0.5, 0.2], "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}
    bake = S._defaults_bake(aoRays=32, giRays=32, giBounces=1)
    vol = {"min": [0.5, 0.5, 0.5], "max": [11.5, 3.5, 11.5], "step": 1.5, "rays": 32}
    groups = [("ground", 0, ground()), ("box", 1, S.cube((4, 0, 4), (6, 2.5, 7)))]
    return S._assemble(groups, mats, sun, SKY, _lightmap(), bake, vol)


def inside():
    mats = [S._material("ground", [0.5, 0.5, 0.5]), S._material("a", [0.8, 0.4, 0.1]), S._material("b", [0.1, 0.4, 0.8])]
    groups = [("ground", 0, ground()), ("a", 1, S.cube((3, -0.5, 3), (6, 2, 6))), ("b", 2, S.cube((4, 0.5, 4), (8, 3, 7))),
              ("c", 2, S.cube((5.5, 1.0, 5.5), (5.9, 1.4, 5.9))),
              # a plate 2 cm under box a's top: its texels lie inside a, within reach of the push out
              ("plate", 1, S.quad((3.5, 1.98, 3.2), (3.5, 1.98, 3.9), (4.2, 1.98, 3.9), (4.2, 1.98, 3.2)))]
    bake = S._defaults_bake(aoRays=32, giRays=32, giBounces=2)
    vol = {"min": [0.5, 0.5, 0.5], "max": [11.5, 3.5, 11.5], "step": 1.0, "rays": 32}
    return S._assemble(groups, mats, SUN, SKY, _lightmap(), bake, vol)


def nothing_received():
    """No material receives: no chart, no tile, an atlas of padding only (every texel its default)."""
    mats = [S._material("ground", [0.5, 0.5, 0.5], receives=False)]
    return S._assemble([("ground", 0, ground())], mats, SUN, SKY, _lightmap(), S._defaults_bake(), None)


def nothing_casts():
    """No material casts: the reference's empty BVH (one leaf nothing reaches); every ray escapes."""
    mats = [S._material("ground", [0.5, 0.5, 0.5], casts=False)]
    vol = {"min": [0.5, 0.5, 0.5], "max": [11.5, 2.5, 11.5], "step": 2.0, "rays": 16}
    return S._assemble([("ground", 0, ground())], mats, SUN, SKY, _lightmap(), S._defaults_bake(aoRays=16, giRays=16),
                       vol)


EDGE_SCENES = {"opacity": opacity, "casts_only": casts_only, "degenerate": degenerate, "no_bounce": no_bounce,
               "night": night, "inside": inside, "nothing_received": nothing_received, "nothing_casts": nothing_casts}
