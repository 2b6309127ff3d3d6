"""Seeded synthetic scenes (.lbscene) for the bake workloads, and the reference's own test scene.

Nothing here is read from a dataset: every scene is generated from a seed. Geometry follows the
reference's conventions (Y up, metres, three vertices a triangle, faces counter-clockwise seen from
outside: crates/lightbaker/tests/bake.rs:11-26).

  small_map      20 x 20 m heightfield on a 1 m grid (800 triangles, heights U[0, 0.3]), 16 boxes
                 (sides U[1, 4]), sun at elevation 40 deg / azimuth 130 deg, constant sky (0.5, 0.6, 0.8),
                 8 texels/m, atlas width 256, 64 AO rays (2 m), 1 bounce x 64 rays, 20 x 20 x 8 probes at 1 m
  map_100m       100 x 100 m heightfield on a 0.5 m grid (80k triangles), 4-octave value noise of 2 m
                 amplitude, 400 boxes (sides U[2, 15]), 2000 open 32-segment cylinders (r U[0.2, 1],
                 h U[1, 6], random yaw), 16 materials (albedo U[0.15, 0.85]), 4 texels/m, atlas width 2048,
                 256 AO rays (2 m), 3 bounces x 128 rays, 50 x 50 x 16 probes at 2 m
  reference_test the scene of crates/lightbaker/tests/bake.rs:29-72 (ground, a box, a red wall, a strip)

Settings a workload leaves open take the reference test's values (tests/bake.rs:52-66): sunSamples 16,
sunRadius 0.5 deg, tileSize 16 m, chartAngle 40 deg, padding 2, indirectDownscale 2, aoStrength 1,
aoFloor 0.25, aoContrast 1, sdfRadius 2, giReach 12, insideShare 0.25, giFilter 1; volume rays = gi rays.
"""
from __future__ import annotations

import math

import numpy as np

from . import encode_scene


def quad(a, b, c, d):
    """tests/bake.rs:11-13: two triangles (a, b, c) and (a, c, d)."""
    return [a, b, c, a, c, d]


def cube(mn, mx):
    """A closed box, faces outward (tests/bake.rs:15-26)."""
    def p(x, y, z):
        return (mx[0] if x > 0 else mn[0], mx[1] if y > 0 else mn[1], mx[2] if z > 0 else mn[2])
    out = []
    out += quad(p(0, 1, 0), p(0, 1, 1), p(1, 1, 1), p(1, 1, 0))
    out += quad(p(0, 0, 0), p(1, 0, 0), p(1, 0, 1), p(0, 0, 1))
    out += quad(p(0, 0, 1), p(1, 0, 1), p(1, 1, 1), p(0, 1, 1))
    out += quad(p(1, 0, 0), p(0, 0, 0), p(0, 1, 0), p(1, 1, 0))
    out += quad(p(1, 0, 1), p(1, 0, 0), p(1, 1, 0), p(1, 1, 1))
    out += quad(p(0, 0, 0), p(0, 0, 1), p(0, 1, 1), p(0, 1, 0))
    return out


def heightfield(x0, z0, size_x, size_z, step, height):
    """A grid of quads (two triangles a cell, facing up); height(x, z) -> y (vectorised)."""
    nx, nz = int(round(size_x / step)), int(round(size_z / step))
    xs = x0 + np.arange(nx + 1, dtype=np.float64) * step
    zs = z0 + np.arange(nz + 1, dtype=np.float64) * step
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    Y = height(X, Z)
    P = np.stack([X, Y, Z], axis=-1).astype(np.float32)
    a = P[:-1, :-1]
    b = P[:-1, 1:]
    c = P[1:, 1:]
    d = P[1:, :-1]
    tris = np.stack([a, b, c, a, c, d], axis=2)  # (nx, nz, 6, 3)
    return tris.reshape(-1, 3)


def cylinder(cx, cy, cz, r, h, yaw, segments=32):
    """An open cylinder's side, 2 triangles a segment, facing out."""
    ang = yaw + np.arange(segments + 1) * (2 * math.pi / segments)
    x = cx + r * np.cos(ang)
    z = cz + r * np.sin(ang)
    out = np.zeros((segments, 6, 3), np.float64)
    for k in range(segments):
        b0 = (x[k], cy, z[k])
        b1 = (x[k + 1], cy, z[k + 1])
        t0 = (x[k], cy + h, z[k])
        t1 = (x[k + 1], cy + h, z[k + 1])
        # counter-clockwise seen from outside
        out[k] = [b0, t0, t1, b0, t1, b1]
    return out.reshape(-1, 3).astype(np.float32)


def _value_noise(rng, octaves, amplitude, extent):
    """Fractal value noise (bilinear lattice noise, octave k at 2^k times the base frequency)."""
    lattices = []
    for k in range(octaves):
        n = 4 * (2 ** k) + 2
        lattices.append((rng.uniform(-1, 1, size=(n, n)), n))

    def f(X, Z):
        y = np.zeros_like(X)
        amp = amplitude
        norm = 0.0
        for lat, n in lattices:
            u = (X / extent) * (n - 2)
            v = (Z / extent) * (n - 2)
            i = np.clip(np.floor(u).astype(int), 0, n - 2)
            j = np.clip(np.floor(v).astype(int), 0, n - 2)
            fu, fv = u - i, v - j
            fu = fu * fu * (3 - 2 * fu)
            fv = fv * fv * (3 - 2 * fv)
            val = (lat[i, j] * (1 - fu) * (1 - fv) + lat[i + 1, j] * fu * (1 - fv) +
                   lat[i, j + 1] * (1 - fu) * fv + lat[i + 1, j + 1] * fu * fv)
            y = y + amp * val
            norm += amp
            amp *= 0.5
        return y * (amplitude / norm)
    return f


def sun_direction(elevation_deg, azimuth_deg):
    """Towards the sun: elevation above the horizon, azimuth from +x towards +z."""
    e, a = math.radians(elevation_deg), math.radians(azimuth_deg)
    return [math.cos(e) * math.cos(a), math.sin(e), math.cos(e) * math.sin(a)]


def _header(materials, meshes, sun, sky, lightmap, bake, volume, user=None):
    return {"sun": sun, "sky": sky, "materials": materials, "meshes": meshes, "lightmap": lightmap,
            "bake": bake, "volume": volume, "user": user if user is not None else {}}


def _material(name, albedo, receives=True, casts=True, opacity=1.0):
    return {"name": name, "albedo": [float(a) for a in albedo], "receives": receives, "casts": casts,
            "opacity": float(opacity)}


def _defaults_bake(**kw):
    b = {"sunSamples": 16, "aoRays": 64, "aoReach": 2.0, "aoStrength": 1.0, "aoFloor": 0.25, "aoContrast": 1.0,
         "sdfRadius": 2.0, "giRays": 64, "giBounces": 1, "giReach": 12.0, "insideShare": 0.25, "giFilter": 1}
    b.update(kw)
    return b


def _assemble(groups, materials, sun, sky, lightmap, bake, volume, user=None):
    """groups: list of (name, material index, positions (n*3, 3))."""
    meshes, positions = [], []
    for name, m, p in groups:
        p = np.asarray(p, np.float32).reshape(-1, 3)
        if len(p) == 0:
            continue
        meshes.append({"name": name, "material": int(m), "triangles": int(len(p) // 3)})
        positions.append(p)
    return encode_scene(_header(materials, meshes, sun, sky, lightmap, bake, volume, user), positions)


def small_map(seed: int = 0, bounces: int = 1) -> bytes:
    """The small plain bake: 20 x 20 m heightfield (800 triangles) and 16 boxes."""
    rng = np.random.default_rng(seed)
    hts = rng.uniform(0.0, 0.3, size=(21, 21))

    def height(X, Z):
        return hts[np.clip(np.round(X).astype(int), 0, 20), np.clip(np.round(Z).astype(int), 0, 20)]
    ground = heightfield(0.0, 0.0, 20.0, 20.0, 1.0, height)
    materials = [_material("ground", [0.5, 0.5, 0.5])]
    groups = [("ground", 0, ground)]
    for k in range(16):
        sx, sy, sz = rng.uniform(1.0, 4.0, size=3)
        x, z = rng.uniform(0.0, 20.0 - sx), rng.uniform(0.0, 20.0 - sz)
        albedo = rng.uniform(0.2, 0.8, size=3)
        materials.append(_material(f"box{k}", albedo))
        groups.append((f"box{k}", k + 1, cube((x, 0.0, z), (x + sx, sy, z + sz))))
    sky = {"zenith": [0.5, 0.6, 0.8], "horizon": [0.5, 0.6, 0.8], "ground": [0.5, 0.6, 0.8]}
    sun = {"direction": sun_direction(40.0, 130.0), "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}
    lightmap = {"texelsPerMeter": 8.0, "tileSize": 16.0, "chartAngleDeg": 40.0, "padding": 2, "atlasWidth": 256,
                "indirectDownscale": 2}
    bake = _defaults_bake(aoRays=64, aoReach=2.0, giRays=64, giBounces=bounces)
    # 20 x 20 x 8 probes at 1 m: min/max chosen to give exactly that grid
    volume = {"min": [0.5, 0.5, 0.5], "max": [19.5, 7.5, 19.5], "step": 1.0, "rays": 64}
    return _assemble(groups, materials, sun, sky, lightmap, bake, volume, {"workload": "small_map", "seed": seed})


def map_100m(seed: int = 0, boxes: int = 400, cylinders: int = 2000) -> bytes:
    """The 100 x 100 m map (about 200k triangles)."""
    rng = np.random.default_rng(seed)
    noise = _value_noise(rng, 4, 2.0, 100.0)
    ground = heightfield(0.0, 0.0, 100.0, 100.0, 0.5, noise)
    materials = [_material(f"m{k}", rng.uniform(0.15, 0.85, size=3)) for k in range(16)]
    per_mat_boxes = [[] for _ in range(16)]
    per_mat_cyl = [[] for _ in range(16)]
    for _ in range(boxes):
        sx, sy, sz = rng.uniform(2.0, 15.0, size=3)
        x, z = rng.uniform(0.0, 100.0 - sx), rng.uniform(0.0, 100.0 - sz)
        base = float(noise(np.array(x + sx / 2), np.array(z + sz / 2))) - 0.5
        m = int(rng.integers(0, 16))
        per_mat_boxes[m].extend(cube((x, base, z), (x + sx, base + sy, z + sz)))
    for _ in range(cylinders):
        r, h = rng.uniform(0.2, 1.0), rng.uniform(1.0, 6.0)
        x, z = rng.uniform(1.0, 99.0), rng.uniform(1.0, 99.0)
        yaw = rng.uniform(0.0, 2 * math.pi)
        base = float(noise(np.array(x), np.array(z))) - 0.2
        m = int(rng.integers(0, 16))
        per_mat_cyl[m].append(cylinder(x, base, z, r, h, yaw))
    groups = [("ground", 0, ground)]
    for m in range(16):
        if per_mat_boxes[m]:
            groups.append((f"boxes{m}", m, np.array(per_mat_boxes[m], np.float32)))
        if per_mat_cyl[m]:
            groups.append((f"props{m}", m, np.concatenate(per_mat_cyl[m])))
    sky = {"zenith": [0.5, 0.6, 0.8], "horizon": [0.5, 0.6, 0.8], "ground": [0.5, 0.6, 0.8]}
    sun = {"direction": sun_direction(40.0, 130.0), "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}
    lightmap = {"texelsPerMeter": 4.0, "tileSize": 16.0, "chartAngleDeg": 40.0, "padding": 2, "atlasWidth": 2048,
                "indirectDownscale": 2}
    bake = _defaults_bake(aoRays=256, aoReach=2.0, giRays=128, giBounces=3)
    # 50 x 50 x 16 probes at 2 m
    volume = {"min": [1.0, 0.5, 1.0], "max": [99.0, 30.5, 99.0], "step": 2.0, "rays": 128}
    return _assemble(groups, materials, sun, sky, lightmap, bake, volume, {"workload": "map_100m", "seed": seed})


def reference_test(box_x: float = 8.0) -> bytes:
    """crates/lightbaker/tests/bake.rs:29-72: 64 x 64 m ground of 4 m quads, a grey box at (box_x, 0, 10),
    a red wall along x = 40, a strip narrower than a texel standing at x = 30."""
    ground = []
    for i in range(16):
        for j in range(16):
            x, z = i * 4.0, j * 4.0
            ground += quad((x, 0, z), (x, 0, z + 4), (x + 4, 0, z + 4), (x + 4, 0, z))
    box = cube((box_x, 0, 10), (box_x + 2, 2, 12))
    wall = cube((40, 0, 30), (40.5, 4, 50))
    strip = quad((30, 0.2, 20), (30, 2.6, 20), (30, 2.6, 20.05), (30, 0.2, 20.05))
    materials = [_material("ground", [0.5, 0.5, 0.5]), _material("grey", [0.5, 0.5, 0.5]),
                 _material("red", [0.9, 0.05, 0.05])]
    groups = [("ground", 0, ground), ("box", 1, box), ("wall", 2, wall), ("strip", 1, strip)]
    sun = {"direction": [-1.0, 0.8, 0.0], "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}
    sky = {"zenith": [0.2, 0.25, 0.35], "horizon": [0.3, 0.3, 0.32], "ground": [0.1, 0.1, 0.1]}
    lightmap = {"texelsPerMeter": 4.0, "tileSize": 16.0, "chartAngleDeg": 40.0, "padding": 2, "atlasWidth": 1024,
                "indirectDownscale": 2}
    bake = {"sunSamples": 16, "aoRays": 64, "aoReach": 0.8, "aoStrength": 1.0, "aoFloor": 0.25, "aoContrast": 1.0,
            "sdfRadius": 2.0, "giRays": 256, "giBounces": 2, "giReach": 12.0, "insideShare": 0.25, "giFilter": 1}
    volume = {"min": [0.0, 0.5, 0.0], "max": [64.0, 4.5, 64.0], "step": 2.0, "rays": 128}
    return _assemble(groups, materials, sun, sky, lightmap, bake, volume, {"test": True})


def uneven_tiles(seed: int = 0, tiles: int = 8, tri_range=(5_000, 500_000), region_range=(64, 512),
                 bounces: int = 1) -> bytes:
    """Tiles of uneven weight for the batched bake, with the small plain bake's generators (a heightfield and
    boxes): a tiles x tiles grid of 16 m tiles (the layout's tile size). Each tile draws two things of its
    own: a triangle count, lognormal clipped to tri_range, made up by its own patch of heightfield
    tessellated that finely (one chart: the patch is gently rolling); and an atlas region, log-uniform
    between region_range[0]^2 and region_range[1]^2 texels at 4 texels/m, made up by boxes (sides U[1, 4]
    m, six charts each) standing on the patch. So the texels a tile holds and the triangles its rays meet
    both vary by orders of magnitude, independently. The small plain bake's ray counts and bounce: 64
    occlusion rays reaching 2 m, one bounce of 64 gather rays; 16 materials; no volume."""
    rng = np.random.default_rng(seed)
    extent = 16.0 * tiles
    noise = _value_noise(rng, 3, 0.5, extent)
    lo, hi = np.log(tri_range[0]), np.log(tri_range[1])
    counts = np.exp(np.clip(rng.normal((lo + hi) / 2, (hi - lo) / 4, size=tiles * tiles), lo, hi)).astype(int)
    side = np.exp(rng.uniform(np.log(region_range[0]), np.log(region_range[1]), size=tiles * tiles))
    materials = [_material(f"m{k}", rng.uniform(0.15, 0.85, size=3)) for k in range(16)]
    per_mat = [[] for _ in range(16)]
    ground = []
    density, pad = 4.0, 2
    for t in range(tiles * tiles):
        tx, tz = (t % tiles) * 16.0, (t // tiles) * 16.0
        # boxes until the tile's charts fill about side^2 texels (its ground chart takes 68^2)
        budget = side[t] ** 2 - (16 * density + 2 * pad) ** 2
        boxes = []
        while budget > 0 and len(boxes) < 2000:
            sx, sy, sz = rng.uniform(1.0, 4.0, size=3)
            faces = [(sx, sy), (sx, sy), (sz, sy), (sz, sy), (sx, sz), (sx, sz)]
            budget -= sum((a * density + 2 * pad + 1) * (b * density + 2 * pad + 1) for a, b in faces) * 1.15
            x, z = tx + rng.uniform(0.2, 15.8 - sx), tz + rng.uniform(0.2, 15.8 - sz)
            base = float(noise(np.array(x + sx / 2), np.array(z + sz / 2))) - 0.3
            boxes.append((x, base, z, sx, sy, sz))
        for (x, base, z, sx, sy, sz) in boxes:
            per_mat[int(rng.integers(0, 16))].append(np.asarray(cube((x, base, z), (x + sx, base + sy, z + sz)),
                                                                np.float32))
        # the rest of the triangles in the tile's own ground patch, 2 a cell
        cells = max(1, int(round(math.sqrt(max(2, counts[t] - 12 * len(boxes)) / 2))))
        ground.append(heightfield(tx, tz, 16.0, 16.0, 16.0 / cells, noise))
    groups = [("ground", 0, np.concatenate(ground))]
    for k in range(16):
        if per_mat[k]:
            groups.append((f"boxes{k}", k, np.concatenate(per_mat[k])))
    sky = {"zenith": [0.5, 0.6, 0.8], "horizon": [0.5, 0.6, 0.8], "ground": [0.5, 0.6, 0.8]}
    sun = {"direction": sun_direction(40.0, 130.0), "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}
    lightmap = {"texelsPerMeter": density, "tileSize": 16.0, "chartAngleDeg": 40.0, "padding": pad,
                "atlasWidth": 4096, "indirectDownscale": 2}
    bake = _defaults_bake(aoRays=64, aoReach=2.0, giRays=64, giBounces=bounces)
    return _assemble(groups, materials, sun, sky, lightmap, bake, None,
                     {"workload": "uneven_tiles", "seed": seed, "tile_triangles": [int(c) for c in counts],
                      "tile_region_side": [float(v) for v in side]})


def stress_map(seed: int = 0, size: float = 400.0, boxes: int = 6000, cylinders: int = 30000, bounces: int = 4,
               segments: int = 16) -> bytes:
    """The stress map: size x size m, 0.5 m fractal heightfield (4 octaves, 2 m), boxes (sides 2-15 m) and
    open cylinder props (r 0.2-1 m, h 1-6 m, `segments` sides), 16 materials; 50 m tiles at 4 texels/m,
    256 AO rays, `bounces` x 128 gather rays, an L1 SH volume at 2 m (200 x 200 x 32 probes at 400 m).
    At 400 m: 1.28 M ground triangles + 72 k box + 0.96 M prop triangles."""
    rng = np.random.default_rng(seed)
    noise = _value_noise(rng, 4, 2.0, size)
    ground = heightfield(0.0, 0.0, size, size, 0.5, noise)
    materials = [_material(f"m{k}", rng.uniform(0.15, 0.85, size=3)) for k in range(16)]
    per_mat = [[] for _ in range(16)]
    for _ in range(boxes):
        sx, sy, sz = rng.uniform(2.0, 15.0, size=3)
        x, z = rng.uniform(0.0, size - sx), rng.uniform(0.0, size - sz)
        base = float(noise(np.array(x + sx / 2), np.array(z + sz / 2))) - 0.5
        per_mat[int(rng.integers(0, 16))].append(np.asarray(cube((x, base, z), (x + sx, base + sy, z + sz)), np.float32))
    r = rng.uniform(0.2, 1.0, cylinders)
    h = rng.uniform(1.0, 6.0, cylinders)
    x = rng.uniform(1.0, size - 1.0, cylinders)
    z = rng.uniform(1.0, size - 1.0, cylinders)
    yaw = rng.uniform(0.0, 2 * math.pi, cylinders)
    m = rng.integers(0, 16, cylinders)
    base = noise(x, z) - 0.2
    for k in range(cylinders):
        per_mat[int(m[k])].append(cylinder(x[k], base[k], z[k], r[k], h[k], yaw[k], segments))
    groups = [("ground", 0, ground)]
    for k in range(16):
        if per_mat[k]:
            groups.append((f"objects{k}", k, np.concatenate(per_mat[k])))
    sky = {"zenith": [0.5, 0.6, 0.8], "horizon": [0.5, 0.6, 0.8], "ground": [0.5, 0.6, 0.8]}
    sun = {"direction": sun_direction(40.0, 130.0), "radiusDeg": 0.5, "irradiance": [3.0, 3.0, 3.0]}
    lightmap = {"texelsPerMeter": 4.0, "tileSize": 50.0, "chartAngleDeg": 40.0, "padding": 2,
                "atlasWidth": 8192 if size > 200 else 2048, "indirectDownscale": 2}
    bake = _defaults_bake(aoRays=256, aoReach=2.0, giRays=128, giBounces=bounces)
    ny = 32 if size >= 400 else 16
    volume = {"min": [1.0, 0.5, 1.0], "max": [size - 1.0, 0.5 + 2.0 * (ny - 1), size - 1.0], "step": 2.0, "rays": 128}
    return _assemble(groups, materials, sun, sky, lightmap, bake, volume, {"workload": "stress_map", "seed": seed})


def with_light(scene: bytes, albedo=None, zenith=None, horizon=None, ground=None, irradiance=None) -> bytes:
    """The same scene with other light parameters: materials' albedos (one rgb a material), the sky's
    colours, the sun's irradiance. Only the header changes (scene.rs:164-181: "LBSC", version, header
    length, header JSON padded to 4 bytes, then the meshes)."""
    import json
    import struct
    hl = struct.unpack_from("<I", scene, 8)[0]
    h = json.loads(scene[12:12 + hl])
    if albedo is not None:
        for m, a in zip(h["materials"], np.asarray(albedo, np.float32).reshape(-1, 3)):
            m["albedo"] = [float(v) for v in a]
    for key, v in (("zenith", zenith), ("horizon", horizon), ("ground", ground)):
        if v is not None:
            h["sky"][key] = [float(c) for c in np.asarray(v, np.float32)]
    if irradiance is not None:
        h["sun"]["irradiance"] = [float(c) for c in np.asarray(irradiance, np.float32)]
    head = json.dumps(h, separators=(",", ":")).encode()
    pad = lambda n: (n + 3) & ~3  # noqa: E731
    rest = scene[pad(12 + hl):]
    body = scene[:8] + struct.pack("<I", len(head)) + head
    return body + b"\0" * (pad(len(body)) - len(body)) + rest


WORKLOADS = {"small_map": small_map, "map_100m": map_100m, "reference_test": reference_test,
             "uneven_tiles": uneven_tiles, "stress_map": stress_map}
