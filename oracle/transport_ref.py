"""ORACLE — test infrastructure only: the checker, never the product.

The bounce transport of a bake restated in float64 with torch autograd, as the reference gradient for
the product's adjoint (lb_transport_backward). The forward follows the reference's bake step by step:

  direct light into the atlas   crates/lightbaker/src/bake.rs:268-275, write_light :434-444
  each gather result            crates/lightbaker/src/gpu/trace.wgsl:245-270 (bounced :133-148, sky :63-66)
  the bounce's texel work       crates/lightbaker/src/bake.rs:303-328 with filter.rs:20-53 (smooth) and
                                filter.rs:58-94 (fill)
  the volume's probes           crates/lightbaker/src/gpu/trace.wgsl:272-324 (L1 projection of the recorded
                                volume rays against the last bounce's light), volume.rs:88-121 (the fill)
  the fallback texels           crates/lightbaker/src/bake.rs:335-359 with volume.rs:125-147 (irradiance)
  the indirect atlas            crates/lightbaker/src/bake.rs:364-421 (block average, two dilations)

Every linear step is a scipy sparse matrix built from the fixed arrays the transport exports (texel
layout, charts, normals, flags, records); the records' evaluation runs in torch, so the gradient comes
from torch's autograd and owes nothing to the product's transposes. theta: albedo (3 a material),
zenith, horizon, ground (3 each), the sun's scale.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

NONE = 0xFFFFFFFF


class Layout:
    """Texel i's tile, its place in the tile and in the atlas."""

    def __init__(self, tiles: np.ndarray, n_tex: int, aw: int):
        tiles = np.asarray(tiles, np.int64).reshape(-1, 5)
        self.tiles = tiles
        i = np.arange(n_tex, dtype=np.int64)
        k = np.searchsorted(tiles[:, 4], i, side="right") - 1
        self.tx, self.ty, self.w, self.h, self.off = (tiles[k, c] for c in range(5))
        li = i - self.off
        self.x = li % self.w
        self.y = li // self.w
        self.atlas = (self.ty + self.y) * aw + self.tx + self.x
        self.n = n_tex

    def neighbour(self, dx: int, dy: int):
        """(valid, j): the texel at (x + dx, y + dy) in the same tile."""
        nx, ny = self.x + dx, self.y + dy
        ok = (nx >= 0) & (nx < self.w) & (ny >= 0) & (ny < self.h)
        j = np.where(ok, self.off + ny * self.w + nx, 0)
        return ok, j


def same_surface(chart, normal, i, j):
    """filter.rs:13-18 in float32, summed as the shader orders it."""
    a, b = normal[i].astype(np.float32), normal[j].astype(np.float32)
    d = (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]
    return (chart[i] == chart[j]) & (d >= np.float32(0.9))


def smooth_matrix(L: Layout, chart, normal, valid, r: int, w: np.ndarray):
    """filter.rs:20-53: a valid texel becomes the weighted mean of its valid, same-surface neighbours
    within r; others are kept."""
    rows, cols, vals = [], [], []
    valid = valid.astype(bool)
    i = np.arange(L.n)
    if r == 0:
        return sp.identity(L.n, format="csr")
    wsum = np.zeros(L.n)
    entries = []
    for dy in range(-r, r + 1):
        for dx in range(-r, r + 1):
            ok, j = L.neighbour(dx, dy)
            ok &= valid & valid[j]
            ok[ok] = same_surface(chart, normal, i[ok], j[ok])
            wk = float(w[(dy + r) * (2 * r + 1) + (dx + r)])
            wsum[ok] += wk
            entries.append((i[ok], j[ok], wk))
    for a, b, wk in entries:
        rows.append(a)
        cols.append(b)
        vals.append(np.full(len(a), wk) / wsum[a])
    keep = ~valid
    rows.append(i[keep])
    cols.append(i[keep])
    vals.append(np.ones(int(keep.sum())))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(L.n, L.n))


def fill_ring(L: Layout, chart, was: np.ndarray):
    """filter.rs:58-94, one ring: (matrix, flags after). A texel not yet known takes the mean of its known
    neighbours of its own chart, else (a texel of no chart) of any known neighbour."""
    was = was.astype(bool)
    i = np.arange(L.n)
    no = np.zeros(L.n, np.int64)
    na = np.zeros(L.n, np.int64)
    pairs = []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            ok, j = L.neighbour(dx, dy)
            ok &= was[j]
            own = ok & (chart != NONE) & (chart[j] == chart)
            other = ok & ~own
            no += own
            na += other
            pairs.append((ok, j, own))
    mode = np.where(~was & (no > 0), 1, np.where(~was & (na > 0) & (chart == NONE), 2, 0))
    rows, cols, vals = [], [], []
    for ok, j, own in pairs:
        take = ((mode == 1) & own) | ((mode == 2) & ok)
        n = np.where(mode == 1, no, na)
        rows.append(i[take])
        cols.append(j[take])
        vals.append(1.0 / n[take])
    keep = mode == 0
    rows.append(i[keep])
    cols.append(i[keep])
    vals.append(np.ones(int(keep.sum())))
    m = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(L.n, L.n))
    return m, was | (mode > 0)


def composite_matrix(owner, known, aw, ah, iw, ih, ds):
    """bake.rs:364-391: each smaller texel's weighted mean of its known texels (weight 1 for a texel's own
    light, 1e-3 for a filled one) and whether it has any."""
    ax = np.arange(aw * ah) % aw
    ay = np.arange(aw * ah) // aw
    t = owner.astype(np.int64)
    ok = owner != NONE
    ok[ok] = known[t[ok]] != 0
    k = np.where(ok, np.where(known[np.where(ok, t, 0)] == 2, 1.0, 1e-3), 0.0)
    b = (ay // ds) * iw + (ax // ds)
    inside = (ax // ds < iw) & (ay // ds < ih)
    ok &= inside
    s3 = np.zeros(iw * ih)
    np.add.at(s3, b[ok], k[ok])
    m = sp.csr_matrix((k[ok] / s3[b[ok]], (b[ok], t[ok])), shape=(iw * ih, len(known)))
    return m, s3 > 0


def dilate_pass(has: np.ndarray, iw: int, ih: int):
    """bake.rs:394-421, one pass: (matrix, flags after)."""
    n = iw * ih
    i = np.arange(n)
    x, y = i % iw, i // iw
    cnt = np.zeros(n, np.int64)
    pairs = []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            nx, ny = x + dx, y + dy
            ok = (nx >= 0) & (nx < iw) & (ny >= 0) & (ny < ih)
            j = np.where(ok, ny * iw + nx, 0)
            ok &= has[j]
            cnt += ok
            pairs.append((ok, j))
    fill = ~has & (cnt > 0)
    rows, cols, vals = [], [], []
    for ok, j in pairs:
        take = fill & ok
        rows.append(i[take])
        cols.append(j[take])
        vals.append(1.0 / cnt[take])
    keep = ~fill
    rows.append(i[keep])
    cols.append(i[keep])
    vals.append(np.ones(int(keep.sum())))
    m = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return m, has | fill


def _pcg(v):
    """trace.wgsl:41-45 on uint32 arrays."""
    v = np.asarray(v, np.uint64) & 0xFFFFFFFF
    s = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
    return ((w >> 22) ^ w) & 0xFFFFFFFF


def _rnd(a, b, seed):
    """trace.wgsl:46: a uniform float in [0, 1) from two keys and the seed."""
    return _pcg(np.asarray(a, np.uint64) ^ _pcg(np.uint64(b) + np.uint64(seed))).astype(np.float32) * np.float32(2.0 ** -32)


def _radical(i):
    """trace.wgsl:49: the bits of i reversed, over 2^32."""
    i = np.asarray(i, np.uint64)
    r = np.zeros_like(i)
    for k in range(32):
        r |= ((i >> k) & 1) << (31 - k)
    return r.astype(np.float32) * np.float32(2.0 ** -32)


def fill_probe_rings(known, nx, ny, nz, rings):
    """volume.rs:88-121: each ring, an unknown probe with known neighbours becomes their mean (and known);
    the others keep their values. Returns the rings' matrices, first first."""
    n = nx * ny * nz
    k = np.arange(n)
    x, z, y = k % nx, (k // nx) % nz, k // (nx * nz)
    out = []
    was = known.copy()
    for _ in range(rings):
        rows, cols, vals = [], [], []
        cnt = np.zeros(n, np.int64)
        nb = []
        for dx, dy, dz in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            xx, yy, zz = x + dx, y + dy, z + dz
            ok = (xx >= 0) & (yy >= 0) & (zz >= 0) & (xx < nx) & (yy < ny) & (zz < nz)
            j = np.where(ok, (yy * nz + zz) * nx + xx, 0)
            ok &= was[j]
            nb.append((ok, j))
            cnt += ok
        filled = ~was & (cnt > 0)
        keep = ~filled
        rows.append(k[keep]), cols.append(k[keep]), vals.append(np.ones(keep.sum()))
        for ok, j in nb:
            m = filled & ok
            rows.append(k[m]), cols.append(j[m]), vals.append(1.0 / cnt[m])
        out.append(sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)))
        was = was | filled
    return out


def _torch_sparse(m):
    import torch
    m = m.tocoo()
    idx = torch.from_numpy(np.vstack([m.row, m.col]).astype(np.int64))
    return torch.sparse_coo_tensor(idx, torch.from_numpy(m.data.astype(np.float64)), m.shape,
                                   check_invariants=True).coalesce()


class TransportRef:
    """The transport of one bake in float64, from the arrays lightbaker_b200.Transport.export gives."""

    def __init__(self, arrays: dict):
        shape = arrays["shape"]
        self.aw, self.ah, self.iw, self.ih, self.ds, self.r, self.rings, self.B, self.rays, self.n_gath, n_tex, self.M = \
            (int(v) for v in shape)
        self.n_light = self.aw * self.ah
        L = Layout(arrays["tiles"], n_tex, self.aw)
        self.layout = L
        chart = arrays["chart"].astype(np.int64)
        normal = arrays["texels"][:, 4:7]
        gathered = arrays["gathered"].astype(bool)
        self.kb = arrays["known_bounce"] >= 1
        known = arrays["known"]
        self.state = arrays["state"]
        self.dl0 = arrays["direct_light"][:, :3].astype(np.float64)
        self.fixed = arrays["fixed_indirect"][:, :3].astype(np.float64)
        idx = arrays["gathered_index"].astype(np.int64)
        # bake.rs:309-323: scatter, smooth (radius giFilter * ds over the gathered texels), fill
        scatter = sp.csr_matrix((np.ones(len(idx)), (idx, np.arange(len(idx)))), shape=(n_tex, len(idx)))
        chart_u = np.where(chart == NONE, NONE, chart)
        sm = smooth_matrix(L, chart_u, normal, gathered, self.r, arrays["smooth_weights"])
        m = sm @ scatter
        was = gathered.copy()
        for _ in range(self.rings):
            f, was = fill_ring(L, chart_u, was)
            m = f @ m
        self.bounce = _torch_sparse(m)
        # write_light (bake.rs:434-444): a known texel's light into its atlas texel
        kt = np.nonzero(self.kb)[0]
        self.write = _torch_sparse(sp.csr_matrix((np.ones(len(kt)), (L.atlas[kt], kt)), shape=(self.n_light, n_tex)))
        self.light_flag = np.zeros(self.n_light, bool)
        self.light_flag[L.atlas[kt]] = True
        # the atlas (bake.rs:364-421)
        cm, has0 = composite_matrix(arrays["owner"], known, self.aw, self.ah, self.iw, self.ih, self.ds)
        d1, has1 = dilate_pass(has0, self.iw, self.ih)
        d2, _ = dilate_pass(has1, self.iw, self.ih)
        self.atlas = _torch_sparse(d2 @ d1 @ cm)
        # the records, as eval reads them
        rec = arrays["records"].reshape(self.n_gath, self.rays, 2)
        kind = rec[:, :, 0] >> 30
        self.kind = kind
        self.mat = (rec[:, :, 0] & 0x3FFFFFFF).astype(np.int64)
        self.li = rec[:, :, 1].astype(np.int64)
        self.y = np.where(kind == 0, rec[:, :, 1].view(np.float32).astype(np.float64), 0.0)
        surf = (kind == 2) & (self.mat < self.M)
        lit = surf & (rec[:, :, 1] != NONE)
        lit[lit] = self.light_flag[self.li[lit]]
        self.surf, self.lit = surf, lit
        self.sky_up = (kind == 0) & (self.y >= 0)
        self.sky_down = (kind == 0) & (self.y < 0)
        # the volume's share, when the transport has one (some texel takes the fallback)
        grid = arrays.get("volume_grid")
        self.vol = grid is not None and len(grid) == 10
        if self.vol:
            self._volume(arrays, grid, n_tex)

    def _volume(self, arrays, grid, n_tex):
        nx, ny, nz, vrays, nv, seed = (int(v) for v in grid[:6])
        origin = grid[6:9].astype(np.uint32).view(np.float32)
        step = grid[9:10].astype(np.uint32).view(np.float32)[0]
        items = arrays["volume_items"].reshape(nv, 16)
        self.vslots = arrays["volume_slots"].astype(np.int64)
        raw = arrays["volume_raw"].reshape(-1, 4, 4)
        self.n_probes = nx * ny * nz
        # every ray's direction (trace.wgsl:278-295), in float64 from the float32 seeds
        key = (items[:, 7].view(np.uint32).astype(np.uint64) * 7919 + 77) & 0xFFFFFFFF
        s1, s2 = _rnd(key, 29, seed).astype(np.float64), _rnd(key, 31, seed).astype(np.float64)
        r = np.arange(vrays, dtype=np.float64)
        u = (r[None, :] + 0.5) / vrays + s1[:, None]
        u -= np.floor(u)
        v = _radical(np.arange(vrays)).astype(np.float64)[None, :] + s2[:, None]
        v -= np.floor(v)
        zc = 1.0 - 2.0 * u
        rr = np.sqrt(np.maximum(0.0, 1.0 - zc * zc))
        a = v * 2.0 * math.pi
        self.vdir = np.stack([rr * np.cos(a), zc, rr * np.sin(a)], axis=-1)
        self.vw = 4.0 * math.pi / vrays
        rec = arrays["volume_records"].reshape(nv, vrays, 2)
        kind = rec[:, :, 0] >> 30
        self.vmat = (rec[:, :, 0] & 0x3FFFFFFF).astype(np.int64)
        self.vli = rec[:, :, 1].astype(np.int64)
        self.vy = np.where(kind == 0, rec[:, :, 1].view(np.float32).astype(np.float64), 0.0)
        surf = (kind == 2) & (self.vmat < self.M)
        lit = surf & (rec[:, :, 1] != NONE)
        lit[lit] = self.light_flag[self.vli[lit]]
        self.vsurf, self.vlit = surf, lit
        self.vsky_up = (kind == 0) & (self.vy >= 0)
        self.vsky_down = (kind == 0) & (self.vy < 0)
        # the fill (volume.rs:88-121), its known flags from the back-face share
        self.vfill = [_torch_sparse(m) for m in fill_probe_rings(raw[:, 1, 3] <= np.float32(0.5), nx, ny, nz, 8)]
        # the fallback texels' trilinear corners (volume.rs:125-137, in float32 as the bake computes them)
        f5 = np.nonzero(self.state == 5)[0]
        self.f5 = f5
        pos = arrays["sample_points"][f5, :3].astype(np.float32)
        nrm = arrays["texels"][f5, 4:7].astype(np.float32)
        q = pos + nrm * np.float32(0.15)
        f = (q - origin[None, :]) / step
        dims = np.array([nx, ny, nz])
        f = np.minimum(np.maximum(f, np.float32(0.0)), (dims - 1).astype(np.float32)[None, :])
        c0 = np.minimum(f.astype(np.int64), dims[None, :] - 2)
        t = (f - c0.astype(np.float32)).astype(np.float32)
        rows, cols, vals = [], [], []
        for k in range(8):
            dx, dy, dz = k & 1, (k >> 1) & 1, (k >> 2) & 1
            w = ((t[:, 0] if dx else 1 - t[:, 0]) * (t[:, 1] if dy else 1 - t[:, 1])) * (t[:, 2] if dz else 1 - t[:, 2])
            j = ((c0[:, 1] + dy) * nz + (c0[:, 2] + dz)) * nx + (c0[:, 0] + dx)
            rows.append(np.arange(len(f5))), cols.append(j), vals.append(w.astype(np.float64))
        self.vinterp = _torch_sparse(sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                                                   shape=(len(f5), self.n_probes)))
        self.vnormal = nrm.astype(np.float64)

    def forward(self, theta):
        """theta: a float64 torch tensor (3 M + 10) -> the indirect atlas (ih * iw, 3)."""
        import torch
        M = self.M
        al = theta[:3 * M].reshape(M, 3) if M else theta.new_zeros((0, 3))
        zen, hor, gro = theta[3 * M:3 * M + 3], theta[3 * M + 3:3 * M + 6], theta[3 * M + 6:3 * M + 9]
        s = theta[3 * M + 9]
        fb = (zen + hor) * 0.5 * math.pi  # bake.rs:150-152
        dl = s * torch.from_numpy(self.dl0)
        y = torch.from_numpy(self.y)[..., None]
        sky = torch.where(torch.from_numpy(self.sky_down)[..., None], gro.expand(*y.shape[:2], 3),
                          hor * (1.0 - y) + zen * y)
        sky = sky * torch.from_numpy(self.sky_up | self.sky_down)[..., None]
        mat = torch.from_numpy(np.where(self.surf, self.mat, 0))
        li = torch.from_numpy(np.where(self.lit, self.li, 0))
        surf = torch.from_numpy(self.surf)[..., None]
        lit = torch.from_numpy(self.lit)[..., None]
        light = torch.sparse.mm(self.write, dl)
        e = None
        for b in range(self.B):
            # trace.wgsl:258-269: (pi * the mean of the terms), a term al / pi * (the hit's light or the
            # fallback) or the sky's colour
            hit = torch.where(lit, light[li], fb.expand(*li.shape, 3))
            term = torch.where(surf, al[mat] / math.pi * hit, sky) if M else sky
            res = term.sum(dim=1) * math.pi / self.rays
            e = torch.sparse.mm(self.bounce, res)
            if b + 1 < self.B:
                light = torch.sparse.mm(self.write, dl + e)
        fallback = torch.from_numpy(self.state == 5)[:, None]
        fixed = torch.from_numpy(self.fixed)
        ind = torch.where(fallback, fixed, e if e is not None else torch.zeros_like(fixed))
        if self.vol:
            # the light the volume reads: the last bounce's (trace.wgsl:296-306 reads the atlas after it)
            last = torch.sparse.mm(self.write, dl + e) if self.B > 0 else light
            vy = torch.from_numpy(self.vy)[..., None]
            vsky = torch.where(torch.from_numpy(self.vsky_down)[..., None], gro.expand(*vy.shape[:2], 3),
                               hor * (1.0 - vy) + zen * vy)
            vsky = vsky * torch.from_numpy(self.vsky_up | self.vsky_down)[..., None]
            vmat = torch.from_numpy(np.where(self.vsurf, self.vmat, 0))
            vli = torch.from_numpy(np.where(self.vlit, self.vli, 0))
            vhit = torch.where(torch.from_numpy(self.vlit)[..., None], last[vli], fb.expand(*vli.shape, 3))
            l = torch.where(torch.from_numpy(self.vsurf)[..., None], al[vmat] / math.pi * vhit, vsky) if M else vsky
            d = torch.from_numpy(self.vdir)
            coef = torch.stack([(l * 0.282095).sum(1)] + [(l * 0.488603 * d[..., a:a + 1]).sum(1) for a in range(3)],
                               dim=1) * self.vw  # (items, 4, 3)
            probes = torch.zeros((self.n_probes, 4, 3), dtype=torch.float64)
            probes = probes.index_put((torch.from_numpy(self.vslots),), coef)
            p = probes.reshape(self.n_probes, 12)
            for f in self.vfill:
                p = torch.sparse.mm(f, p)
            p4 = torch.sparse.mm(self.vinterp, p).reshape(-1, 4, 3)
            n = torch.from_numpy(self.vnormal)
            a0, a1 = math.pi * 0.282095, 2.0 * math.pi / 3.0 * 0.488603
            arg = a0 * p4[:, 0] + a1 * (p4[:, 1] * n[:, 0:1] + p4[:, 2] * n[:, 1:2] + p4[:, 3] * n[:, 2:3])
            e5 = 0.5 * a0 * p4[:, 0] + 0.5 * torch.relu(arg)
            ind = ind.index_put((torch.from_numpy(self.f5),), e5)
        return torch.sparse.mm(self.atlas, ind)

    def gradient(self, theta: np.ndarray, g_indirect: np.ndarray):
        """(the atlas at theta, d(sum g * atlas)/d(theta)), both float64."""
        import torch
        th = torch.tensor(np.asarray(theta, np.float64), requires_grad=True)
        out = self.forward(th)
        g = torch.from_numpy(np.asarray(g_indirect, np.float64).reshape(-1, 3))
        (out * g).sum().backward()
        return out.detach().numpy(), th.grad.numpy()
