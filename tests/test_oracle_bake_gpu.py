"""The device-resident bake (csrc/raster.cu, post.cu, bake_device.cu) against the oracle's independent
restatement of the reference's CPU work (oracle/bake_ref.cpp: raster.rs:39-114, bake.rs:197-421,
volume.rs:86-147), which shares no code with the product.

Whole bakes (reference_test, small_map): every atlas, the validity and the volume equal the oracle's
whole CPU bake bit for bit. map_100m is too large for the oracle's tracer, so its stages are checked one
at a time on the device's own inputs: the raster of every tile; on a subset of tiles the per-tile post
from the device's direct records, the gather selection, and the last bounce's filters from the device's
gather results; over the whole map the light atlas, the volume fallback and the composite."""
import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes
from oracle import bake_ref as R
from oracle.bake_ref import OracleBake

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_same(name, a, b):
    d = np.nonzero(bits(a) != bits(b))
    assert len(d[0]) == 0, f"{name}: {len(d[0])} values differ, first at {[x[:3] for x in d]}"


@pytest.mark.parametrize("name", ["reference_test", "small_map"])
def test_device_bake_equals_oracle_bake(gpu, name):
    s = scenes.WORKLOADS[name]()
    ob = OracleBake(s, lb.prepare(s))
    dev = lb.bake_device(s, gpu)
    assert_same("direct atlas", dev.direct, ob.direct)
    assert_same("validity", dev.validity, ob.validity)
    assert_same("indirect atlas", dev.indirect, ob.indirect)
    assert_same("volume", dev.volume, ob.volume)
    assert dev.stats.rays_direct == ob.rays["direct"] and dev.stats.rays_volume == ob.rays["volume"]


EXPORTS = ("tiles", "texels", "sample_points", "chart", "valid", "known", "state", "gathered", "field", "ao", "direct",
           "indirect_light", "direct_records", "gather_out", "light", "probes")


class Stages:
    """A scene's layout and settings, the device bake's own arrays (lb_transport_export) and its atlases."""

    def __init__(self, scene: bytes, x: dict, atlases):
        self.P = lb.prepare(scene)
        self.header, self.positions = R.read_scene(scene)
        self.x = x
        self.tiles = x["tiles"]
        self.texels = np.ascontiguousarray(x["texels"], np.float32).reshape(-1).copy().view(R.TEXEL)
        self.atlases = atlases

    @staticmethod
    def of_device(scene: bytes, gpu) -> "Stages":
        tr = lb.Transport(scene, gpu)
        try:
            x = {k: tr.export(k) for k in EXPORTS}
        finally:
            tr.close()
        return Stages(scene, x, lb.bake_device(scene, gpu))


def post_settings(S):
    b, lm = S.header["bake"], S.header["lightmap"]
    st = R.PostSettings()
    st.inside_share, st.ao_strength = R.f32(b["insideShare"]), R.f32(b["aoStrength"])
    st.ao_floor, st.ao_contrast, st.sdf_radius = R.f32(b["aoFloor"]), R.f32(b["aoContrast"]), R.f32(b["sdfRadius"])
    st.sun_irradiance[:] = [R.f32(v) for v in S.header["sun"]["irradiance"]]
    st.sun_dir[:] = list(S.P.params.sun_dir)[:3]
    st.grid, st.padding = int(S.P.params.counts[0]), int(lm["padding"])
    return st


def check_post_and_selection(S, every=5):
    """bake.rs:197-298 on every `every`-th tile: from the device's direct records, the oracle's valid, state,
    known, moved sample points, field, occlusion and direct light, and its gather selection."""
    x, l, lm = S.x, R._declare(), S.header["lightmap"]
    st = post_settings(S)
    cov_before = checked = 0
    for t, (tx, ty, w, h, off) in enumerate(S.tiles.tolist()):
        n = w * h
        sl = slice(off, off + n)
        tex = S.texels[sl].copy()
        ncov = int((tex["pos"][:, 3] > 0.5).sum())
        if t % every == 0:
            va, kn, sa = (np.zeros(n, np.uint8) for _ in range(3))
            fi, ao, dl = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
            rec = np.ascontiguousarray(x["direct_records"][cov_before:cov_before + ncov], np.float32)
            used = l.or_tile_post(w, h, R._p(tex), R._p(rec), R.C.byref(st), R._p(va), R._p(kn), R._p(sa), R._p(fi),
                                  R._p(ao), R._p(dl))
            assert used == ncov
            assert_same(f"tile {t} valid", x["valid"][sl], va)
            # texels the volume lit later (state 5) were without light here
            vol = x["state"][sl] == 5
            assert ((kn == 0) | ~vol).all()
            keep = ~vol
            assert_same(f"tile {t} state", x["state"][sl][keep], sa[keep])
            assert_same(f"tile {t} known", x["known"][sl][keep], kn[keep])
            assert_same(f"tile {t} field", x["field"][sl][keep], fi[keep])
            assert_same(f"tile {t} ao", x["ao"][sl][keep], ao[keep])
            assert_same(f"tile {t} direct light", x["direct"][sl][keep, :3], dl[keep])
            moved = va != 0
            assert_same(f"tile {t} sample points", x["sample_points"][sl][moved, :3], tex["pos"][moved, :3])
            g = np.zeros(n, np.uint8)
            l.or_gather_select(w, h, R._p(va), R._p(np.ascontiguousarray(x["chart"][sl])), int(lm["indirectDownscale"]),
                               R._p(g))
            assert_same(f"tile {t} gathered", x["gathered"][sl], g)
            checked += 1
        cov_before += ncov
    assert cov_before == len(x["direct_records"]) and checked >= 1
    return checked


def check_last_bounce_filters(S, every=5):
    """bake.rs:303-322 on every `every`-th tile: the device's last-bounce gather results scattered, smoothed
    and filled by the oracle give the device's indirect light."""
    x, l, b, lm = S.x, R._declare(), S.header["bake"], S.header["lightmap"]
    ds = int(lm["indirectDownscale"])
    radius, rings = int(b["giFilter"]) * ds, int(lm["padding"]) + 2 * ds + 2
    g_before = checked = 0
    for t, (tx, ty, w, h, off) in enumerate(S.tiles.tolist()):
        sl = slice(off, off + w * h)
        gathered = np.ascontiguousarray(x["gathered"][sl])
        ng = int(gathered.sum())
        if t % every == 0:
            normal = np.ascontiguousarray(S.texels[sl]["normal"][:, :3])
            e = np.zeros((w * h, 3), np.float32)
            res = np.ascontiguousarray(x["gather_out"][g_before:g_before + ng], np.float32)
            used = l.or_bounce_tile(w, h, R._p(np.ascontiguousarray(x["chart"][sl])), R._p(normal), R._p(gathered),
                                    R._p(res), radius, rings, R._p(e))
            assert used == ng
            keep = x["state"][sl] != 5
            assert_same(f"tile {t} indirect light", x["indirect_light"][sl][keep, :3], e[keep])
            checked += 1
        g_before += ng
    assert g_before == len(x["gather_out"]) and checked >= 1
    return checked


def check_light_fallback_composite(S):
    """Over every tile: write_light (bake.rs:435-445) of the last bounce, the volume fallback (bake.rs:337-359
    with volume.rs:125-147) from the device's probes, and the composite with its dilations
    (bake.rs:364-421) of the device's final texel arrays, against the device's atlases."""
    x, l, P = S.x, R._declare(), S.P
    aw, ah, ds = int(P.info.atlas_width), int(P.info.atlas_height), int(P.info.indirect_downscale)
    vs = S.header["volume"]
    light = np.zeros((aw * ah, 4), np.float32)
    known, state, field, ao, ind = [], [], [], [], []
    (nx, ny, nz), _, _ = R.volume_probes(vs, S.header["lightmap"]["tileSize"])
    probes = np.ascontiguousarray(x["probes"], np.float32).reshape(-1, 16)
    assert probes.shape == (nx * ny * nz, 16)
    fallback = 0
    C = R.C
    for t, (tx, ty, w, h, off) in enumerate(S.tiles.tolist()):
        n = w * h
        sl = slice(off, off + n)
        vol = x["state"][sl] == 5
        k = np.ascontiguousarray(x["known"][sl]).copy()
        k[vol] = 0  # as the last bounce wrote its light
        d3 = np.ascontiguousarray(x["direct"][sl][:, :3], np.float32)
        i3 = np.ascontiguousarray(x["indirect_light"][sl][:, :3], np.float32)
        l.or_write_light(tx, ty, w, h, aw, R._p(k), R._p(d3), R._p(i3), R._p(light))
        s2, f2, a2 = np.zeros(n, np.uint8), np.zeros(n, np.float32), np.zeros(n, np.float32)
        d2, e2 = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
        fallback += l.or_volume_fallback(
            w, h, R._p(S.texels[sl].copy()), R._p(probes), nx, ny, nz, (C.c_float * 3)(*[R.f32(v) for v in vs["min"]]),
            float(R.f32(vs["step"])), (C.c_float * 3)(*[R.f32(v) for v in S.header["sun"]["irradiance"]]),
            (C.c_float * 3)(*list(P.params.sun_dir)[:3]), R._p(k), R._p(s2), R._p(f2), R._p(a2), R._p(d2), R._p(e2))
        assert_same(f"tile {t} fallback texels", s2 == 5, vol)
        assert_same(f"tile {t} fallback field", f2[vol], x["field"][sl][vol])
        assert_same(f"tile {t} fallback ao", a2[vol], x["ao"][sl][vol])
        assert_same(f"tile {t} fallback direct", d2[vol], x["direct"][sl][vol, :3])
        assert_same(f"tile {t} fallback indirect", e2[vol], x["indirect_light"][sl][vol, :3])
        for lst, a in zip((known, state, field, ao, ind), (x["known"][sl], x["state"][sl], x["field"][sl], x["ao"][sl], i3)):
            lst.append(np.ascontiguousarray(a))
    assert_same("light atlas", x["light"].reshape(-1, 4), light)
    T = len(S.tiles)
    rects = np.ascontiguousarray(S.tiles[:, :4], np.uint32).reshape(-1)
    ptrs = lambda arrs: (C.c_void_p * T)(*[a.ctypes.data for a in arrs])
    iw, ih = (aw + ds - 1) // ds, (ah + ds - 1) // ds
    d_out, v_out = np.zeros((ah, aw, 2), np.float32), np.zeros((ah, aw), np.uint8)
    i_out = np.zeros((ih, iw, 3), np.float32)
    l.or_composite(aw, ah, ds, T, R._p(rects), ptrs(known), ptrs(state), ptrs(field), ptrs(ao), ptrs(ind),
                   R._p(d_out), R._p(v_out), R._p(i_out))
    assert_same("direct atlas", S.atlases.direct, d_out)
    assert_same("validity", S.atlases.validity, v_out)
    assert_same("indirect atlas", S.atlases.indirect, i_out)
    return fallback


@pytest.fixture(scope="module")
def map100(gpu):
    return Stages.of_device(scenes.map_100m(), gpu)


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_device_raster_equals_oracle(gpu, name):
    s = scenes.WORKLOADS[name]()
    P = lb.prepare(s)
    header, positions = R.read_scene(s)
    lm = header["lightmap"]
    layout = P.layout()
    tr = lb.Transport(s, gpu)
    try:
        dev = tr.export("texels").reshape(-1).view(np.uint32)
        tiles = tr.export("tiles")
    finally:
        tr.close()
    for t, (x, y, w, h, off) in enumerate(tiles.tolist()):
        mine = R.raster_tile(layout, P.tiles[t], t, positions, R.f32(lm["texelsPerMeter"]), int(lm["padding"]))
        assert_same(f"tile {t}", dev[off * 16:(off + w * h) * 16], mine.view(np.uint32))


def test_map_100m_post_and_selection_per_tile(map100):
    assert check_post_and_selection(map100) >= 5


def test_map_100m_last_bounce_filters_per_tile(map100):
    assert check_last_bounce_filters(map100) >= 5


def test_map_100m_light_fallback_and_composite(map100):
    assert check_light_fallback_composite(map100) > 0


@pytest.mark.parametrize("name", ["opacity", "casts_only", "degenerate", "no_bounce", "night", "inside",
                                  "nothing_received", "nothing_casts"])
def test_device_bake_edge_scenes_equal_oracle_bake(gpu, name):
    """The edge scenes (tests/edge_scenes.py) through the device-resident bake and through the drop-in bake on
    the GPU: both equal the oracle's whole bake bit for bit."""
    from edge_scenes import EDGE_SCENES
    s = EDGE_SCENES[name]()
    ob = OracleBake(s, lb.prepare(s))
    for b in (lb.bake_device(s, gpu), lb.bake(s, gpu)):
        assert_same("direct atlas", b.direct, ob.direct)
        assert_same("validity", b.validity, ob.validity)
        assert_same("indirect atlas", b.indirect, ob.indirect)
        if ob.volume is not None:
            assert_same("volume", b.volume, ob.volume)
