"""Dense numpy restatement of the viscosity level-0 construction, written
independently of the oracle's leaf-by-leaf C code, for small domains:

  L_with_level::calculate_subcell_sdf_volume   (simd_viscosity3d.cpp:258-330)
  volume_fraction                               (volume_fractions.cpp:82-120)
  calculate_matrix_coefficients_volume         (simd_viscosity3d.cpp:332-406)
  mark_dof                                      (simd_viscosity3d.cpp:408-498)
  finest_level_matrix_setter                    (simd_viscosity3d.cpp:541-878)

Every float32 operation is issued in the reference's order, so the results are
compared bit for bit.  Leaf sets come from voxel-level dilations
(scipy.ndimage) rather than the oracle's per-leaf boundary test.  Viscosity is
constant (a grid without leaves), as in the viscosity call site of FLIP_vdb.
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage

F32 = np.float32


class Box:
    """Dense index box [lo, lo + size)^3, lo a multiple of 16."""

    def __init__(self, lo: int, size: int):
        self.lo = lo
        self.size = size


def dense(grid, box: Box, scale: int = 1):
    """Values of a leaf grid over the box (getValue semantics: background
    outside the leaves), plus the active mask and the leaf-block mask."""
    n = box.size * scale
    vals = np.full((n, n, n), F32(grid.background[0]), F32)
    act = np.zeros((n, n, n), bool)
    blocks = np.zeros((n // 8,) * 3, bool)
    off = np.arange(512)
    lx, ly, lz = off >> 6, (off >> 3) & 7, off & 7
    masks = ((grid.masks[:, :, None] >> np.arange(64, dtype=np.uint64)[None, None, :]) & np.uint64(1)).reshape(-1, 512)
    for i in range(grid.leaf_count):
        o = grid.origins[i] - box.lo * scale
        vals[o[0] + lx, o[1] + ly, o[2] + lz] = grid.values[i].reshape(512)
        act[o[0] + lx, o[1] + ly, o[2] + lz] = masks[i].astype(bool)
        blocks[o[0] // 8, o[1] // 8, o[2] // 8] = True
    return vals, act, blocks


def block_dilate(active, blocks, r, face_only=False):
    """Leaves of dilateActiveValues(r): original leaves plus leaves that the
    dilated active voxels enter."""
    st = ndimage.generate_binary_structure(3, 1 if face_only else 3)
    d = ndimage.binary_dilation(active, structure=st, iterations=r) if active.any() else active
    n = d.shape[0] // 8
    occ = d.reshape(n, 8, n, 8, n, 8).any(axis=(1, 3, 5))
    return occ | blocks


def expand(blocks):
    return np.repeat(np.repeat(np.repeat(blocks, 8, 0), 8, 1), 8, 2)


def lerp(a, b, w):
    d = (b - a).astype(F32)
    return (a + (d.astype(np.float64) * w).astype(F32)).astype(F32)


def trilinear(vals, bg, px, py, pz):
    """BoxSampler::sample over a dense array (index 0 = array origin);
    coordinates outside read bg."""
    fx, fy, fz = np.floor(px), np.floor(py), np.floor(pz)
    u, v, w = px - fx, py - fy, pz - fz
    ix, iy, iz = fx.astype(np.int64), fy.astype(np.int64), fz.astype(np.int64)
    n = vals.shape

    def get(a, b, c):
        ok = (a >= 0) & (a < n[0]) & (b >= 0) & (b < n[1]) & (c >= 0) & (c < n[2])
        out = np.full(a.shape, F32(bg), F32)
        out[ok] = vals[a[ok], b[ok], c[ok]]
        return out

    d = {}
    for i in (0, 1):
        for j in (0, 1):
            for k in (0, 1):
                d[i, j, k] = get(ix + i, iy + j, iz + k)
    a0 = lerp(lerp(d[0, 0, 0], d[0, 0, 1], w), lerp(d[0, 1, 0], d[0, 1, 1], w), v)
    a1 = lerp(lerp(d[1, 0, 0], d[1, 0, 1], w), lerp(d[1, 1, 0], d[1, 1, 1], w), v)
    return lerp(a0, a1, u)


def tet_fraction(p0, p1, p2, p3):
    s = np.sort(np.stack([p0, p1, p2, p3], -1), axis=-1)
    q0, q1, q2, q3 = (s[..., k] for k in range(4))
    with np.errstate(all="ignore"):
        def stet(a, b, c, d):
            return (a * a * a / ((a - b) * (a - c) * (a - d))).astype(F32)

        def sprism(a0, a1, a2, a3):
            a = a0 / (a0 - a2); b = a0 / (a0 - a3); c = a1 / (a1 - a3); d = a1 / (a1 - a2)
            return (a * b * (F32(1) - d) + b * (F32(1) - c) * d + c * d).astype(F32)

        r = np.zeros(q0.shape, F32)
        r = np.where(q0 <= 0, stet(q0, q1, q2, q3), r)
        r = np.where(q1 <= 0, sprism(q0, q1, q2, q3), r)
        r = np.where(q2 <= 0, F32(1) - stet(q3, q2, q1, q0), r)
        r = np.where(q3 <= 0, F32(1), r)
    return r.astype(F32)


def cube_fraction(p000, p100, p010, p110, p001, p101, p011, p111):
    t = [tet_fraction(p000, p001, p101, p011), tet_fraction(p000, p101, p100, p110),
         tet_fraction(p000, p010, p011, p110), tet_fraction(p101, p011, p111, p110),
         F32(2) * tet_fraction(p000, p011, p101, p110), tet_fraction(p100, p101, p001, p111),
         tet_fraction(p100, p001, p000, p010), tet_fraction(p100, p110, p111, p010),
         tet_fraction(p001, p111, p011, p010), F32(2) * tet_fraction(p100, p111, p001, p010)]
    s = t[0]
    for x in t[1:]:
        s = (s + x).astype(F32)
    s = (s / F32(12)).astype(F32)
    allneg = ((p000 < 0) & (p100 < 0) & (p010 < 0) & (p110 < 0) & (p001 < 0) & (p101 < 0) &
              (p011 < 0) & (p111 < 0))
    return np.where(allneg, F32(1), s).astype(F32)


def shift(a, d, fill=0):
    """out[g] = a[g + d] (fill outside)."""
    out = np.full(a.shape, fill, a.dtype)
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    for ax in range(3):
        k = d[ax]
        if k > 0:
            src[ax] = slice(k, None); dst[ax] = slice(0, -k)
        elif k < 0:
            src[ax] = slice(0, k); dst[ax] = slice(-k, None)
    out[tuple(dst)] = a[tuple(src)]
    return out


def e(ax, s=1):
    v = [0, 0, 0]
    v[ax] = s
    return v


def level0(scene, box: Box):
    """Returns dict with DOF masks, pattern blocks, coefficient arrays (dense,
    untrimmed), face volumes and the defaults."""
    dx = F32(scene.dx)
    liq, act, lblocks = dense(scene.liquid_phi, box)
    lbg = F32(scene.liquid_phi.background[0])
    sol, _, _ = dense(scene.solid_phi, box)
    sbg = F32(scene.solid_phi.background[0])
    mu = F32(scene.viscosity.background[0])
    assert scene.viscosity.leaf_count == 0

    a1 = block_dilate(act, lblocks, 1)
    a2 = block_dilate(act, lblocks, 2)
    a1f = block_dilate(act, lblocks, 1, face_only=True)

    # subcell SDF over 2 * box
    ns = 2 * box.size
    s = np.arange(ns) + 2 * box.lo
    S0, S1, S2 = np.meshgrid(s, s, s, indexing="ij")
    member = np.repeat(np.repeat(np.repeat(a1, 16, 0), 16, 1), 16, 2)
    sub_bg = F32(F32(1.5) * dx)
    p = lambda S: 0.5 * S - 0.5 - box.lo
    v = trilinear(liq, lbg, p(S0), p(S1), p(S2))
    sdf = np.where(member, np.where(v < sub_bg, v, sub_bg), sub_bg).astype(F32)
    sp = np.full((ns + 1,) * 3, sub_bg, F32)
    sp[:ns, :ns, :ns] = sdf
    c = lambda a, b, k: sp[a:a + ns, b:b + ns, k:k + ns]
    frac = cube_fraction(c(0, 0, 0), c(1, 0, 0), c(0, 1, 0), c(1, 1, 0), c(0, 0, 1), c(1, 0, 1),
                         c(0, 1, 1), c(1, 1, 1))
    svol = np.where(member & (frac > 0), frac, F32(0)).astype(F32)

    # control volumes: padded subcell volume indexed at 2g + offsets in [-1, 1]
    n = box.size
    spad = np.zeros((ns + 2,) * 3, F32)
    spad[1:-1, 1:-1, 1:-1] = svol

    def sv(ox, oy, oz):
        return spad[1 + ox:1 + ox + ns:2, 1 + oy:1 + oy + ns:2, 1 + oz:1 + oz + ns:2]

    vol_c = np.zeros((n,) * 3, F32)
    vol_f = [np.zeros((n,) * 3, F32) for _ in range(3)]
    vol_e = [np.zeros((n,) * 3, F32) for _ in range(3)]
    for i in (0, 1):
        for j in (0, 1):
            for k in (0, 1):
                vol_c = (vol_c + sv(i, j, k)).astype(F32)
                for ax in range(3):
                    f = [i, j, k]; f[ax] -= 1
                    vol_f[ax] = (vol_f[ax] + sv(*f)).astype(F32)
                    g = [i - 1, j - 1, k - 1]; g[ax] += 1
                    vol_e[ax] = (vol_e[ax] + sv(*g)).astype(F32)
    m2 = expand(a2)
    fin = lambda x: np.where(m2 & (x > 0), (x * F32(0.125)).astype(F32), F32(0)).astype(F32)
    V = fin(vol_c)
    FV = [fin(x) for x in vol_f]
    EV = [fin(x) for x in vol_e]

    # is_solid and DOF over the face-dilated liquid leaves
    m1f = expand(a1f)
    g = np.arange(n) + box.lo
    G0, G1, G2 = np.meshgrid(g, g, g, indexing="ij")
    dof = []
    for ch in range(3):
        P = [G0.astype(np.float64), G1.astype(np.float64), G2.astype(np.float64)]
        P[ch] = P[ch] - 0.5
        ssamp = trilinear(sol, sbg, P[0] - box.lo, P[1] - box.lo, P[2] - box.lo)
        solid = m1f & (ssamp < 0)
        d1, d2 = (ch + 1) % 3, (ch + 2) % 3
        on = (FV[ch] > 0) | (V > 0) | (shift(V, e(ch, -1)) > 0)
        on |= (EV[d1] > 0) | (shift(EV[d1], e(d2)) > 0) | (EV[d2] > 0) | (shift(EV[d2], e(d1)) > 0)
        dof.append(m1f & ~solid & on)
    union = dof[0] | dof[1] | dof[2]
    nb = n // 8
    dblocks = union.reshape(nb, 8, nb, 8, nb, 8).any(axis=(1, 3, 5))
    pattern = block_dilate(union, dblocks, 2)

    factor = F32(F32(scene.dt) / (F32(scene.rho) * dx * dx))
    doff = F32(factor * mu)
    ddiag = F32(F32(1) + F32(8) * doff)
    coef = np.zeros((3, 9, n, n, n), F32)
    for ch in range(3):
        d0, d1, d2 = ch, (ch + 1) % 3, (ch + 2) % 3
        D = dof[ch]
        fv = np.where(FV[d0] < F32(0.1), F32(0.1), FV[d0]).astype(F32)
        diag = (F32(0) + fv).astype(F32)
        two_f = F32(F32(2) * factor)
        t = ((two_f * V).astype(F32) * mu).astype(F32)
        diag = (diag + t).astype(F32)
        t = ((two_f * shift(V, e(d0, -1))).astype(F32) * mu).astype(F32)
        diag = (diag + t).astype(F32)
        neg = {d0: np.where(shift(D, e(d0, -1), False), -t, F32(0))}
        t = ((factor * shift(EV[d2], e(d1))).astype(F32) * mu).astype(F32)
        diag = (diag + t).astype(F32)
        t = ((factor * EV[d2]).astype(F32) * mu).astype(F32)
        diag = (diag + t).astype(F32)
        neg[d1] = np.where(shift(D, e(d1, -1), False), -t, F32(0))
        t = ((factor * shift(EV[d1], e(d2))).astype(F32) * mu).astype(F32)
        diag = (diag + t).astype(F32)
        t = ((factor * EV[d1]).astype(F32) * mu).astype(F32)
        diag = (diag + t).astype(F32)
        neg[d2] = np.where(shift(D, e(d2, -1), False), -t, F32(0))
        with np.errstate(divide="ignore"):
            inv = np.where(diag != 0, (F32(1) / diag).astype(F32), F32(0))
        coef[ch, 0] = np.where(D, diag, ddiag)
        coef[ch, 1] = np.where(D, inv, F32(0))
        for ax in range(3):
            coef[ch, 2 + ax] = np.where(D, neg[ax], F32(0))
        for jk in range(4):
            j, k = jk >> 1, jk & 1
            pair = shift(dof[d1], e(d1, j), False) & shift(dof[d2], e(d2, k), False)
            ev = shift(EV[d0], [a + b for a, b in zip(e(d1, j), e(d2, k))])
            f = factor if j == k else F32(-factor)
            coef[ch, 5 + jk] = np.where(pair, ((f * ev).astype(F32) * mu).astype(F32), F32(0))
    return dict(dof=dof, pattern=pattern, coef=coef, face_vol=FV, ddiag=ddiag, doff=doff, factor=factor)
