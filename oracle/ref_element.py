"""Independent restatement of the refined reference element (TEST
INFRASTRUCTURE): build_patch_ref_r64 with ref_square_regroup and the cc level
(src/patch_refine_mod.f90:100-262, 264-311, 313-421), written in numpy from
the algorithm, not from the C++ of the library or of oracle/orc_levels.cpp,
so that the library's tables are checked against a separate derivation.

Level 1 is the Vioreanu-Rokhlin rule of degree order-1 (n1 nodes).  Level l
>= 2 is the 4-split of level l-1: every node (u, v), with (a, b) = 2(u, v) -
1, has the four images (a, b), (-a, -b), (a, b+2), (a+2, b), each mapped by
x -> ((x - 1)/2 + 1)/2 and weighted a quarter, image-major.  With four levels
the last is the cc level: 39 of the 64 sub-patches of the 4-split of level 3
(CC_KEEP, cc_subidx_at :264-311) and the 4 sub-patches of level 2 scaled by
0.625 about (0.4375, 0.4375) with weights times 0.625^2.  In square mode every
level >= 2 then pairs the sub-patches whose centroids share a cell of a
2^(l-1) x 2^(l-1) grid (8 x 8 at the cc level, whose last 4 sub-patches stay
single) into one qg x qg Gauss-Legendre square of the cell (weights scaled by
twice the level-1 weight sum), pairs first in cell order (row by row), then
the single sub-patches in their order.  qg = korder + 1, or korder + 3 below 8.

Only tests/ import this module.
"""
import numpy as np

CC_KEEP = (1, 2, 3, 4, 7, 8, 9, 10, 11, 13, 14, 16, 17, 27, 32, 33, 34, 35, 37, 40, 41, 42, 43, 44, 46, 47, 48, 49,
           50, 52, 53, 55, 58, 59, 60, 61, 62, 63, 64)  # 1-based sub-triangles of the split kept at the cc level
CC_SCALE, CC_SHIFT = 0.625, 0.4375


def _images(uv, wt):
    a = 2.0 * uv - 1.0
    imgs = [a, -a, a + np.array([0.0, 2.0]), a + np.array([2.0, 0.0])]
    out = np.concatenate(imgs)
    return ((out - 1.0) * 0.5 + 1.0) * 0.5, np.tile(0.25 * wt, 4)


def _squares(uv, wt, n1, ncell, npair_max, qg, fac):
    """(uv, wt, suboff, subtyp) after pairing sub-patches 0..npair_max-1 by cell"""
    nsub = uv.shape[0] // n1
    cen = uv.reshape(nsub, n1, 2).mean(axis=1)
    side = 1.0 / ncell
    cell = np.clip(np.floor(cen / side).astype(np.int64), 0, ncell - 1)
    key = cell[:, 0] + ncell * cell[:, 1]
    pairable = np.arange(nsub) < npair_max
    count = np.bincount(key[pairable], minlength=ncell * ncell)
    assert count.max() <= 2, "more than two sub-patches in a cell"
    t, w = np.polynomial.legendre.leggauss(qg)
    t, w = 0.5 * (t + 1.0), 0.5 * w
    parts_uv, parts_wt, sizes, typ = [], [], [], []
    for c in np.flatnonzero(count == 2):  # cells in row-major order: jc outer, ic inner
        ic, jc = c % ncell, c // ncell
        uu = (ic + t[None, :]) * side * np.ones((qg, 1))
        vv = (jc + t[:, None]) * side * np.ones((1, qg))
        parts_uv.append(np.stack([uu.ravel(), vv.ravel()], axis=1))
        parts_wt.append((w[None, :] * w[:, None]).ravel() * side * side * fac)
        sizes.append(qg * qg)
        typ.append(1)
    single = [q for q in range(nsub) if not pairable[q] or count[key[q]] == 1]
    for q in single:
        parts_uv.append(uv[q * n1:(q + 1) * n1])
        parts_wt.append(wt[q * n1:(q + 1) * n1])
        sizes.append(n1)
        typ.append(0)
    return (np.concatenate(parts_uv), np.concatenate(parts_wt), np.concatenate([[0], np.cumsum(sizes)]),
            np.array(typ, np.int64))


def reference_element(korder, order, vr_uv, vr_wt, nlevel=4, square=True):
    """levels as dicts (uv (n, 2), wt, suboff, subtyp); vr_uv/vr_wt: the
    Vioreanu-Rokhlin rule of degree order-1 (the published table)"""
    n1 = order * (order + 1) // 2
    uv1, wt1 = np.asarray(vr_uv, float).reshape(n1, 2), np.asarray(vr_wt, float)
    raw = [(uv1, wt1)]
    for il in range(2, nlevel + 1):
        uv, wt = _images(*raw[-1])
        if il == nlevel == 4:
            idx = np.concatenate([np.arange((k - 1) * n1, k * n1) for k in CC_KEEP])
            uv2, wt2 = raw[1]
            uv = np.concatenate([uv[idx], (uv2[:4 * n1] - 0.5) * CC_SCALE + CC_SHIFT])
            wt = np.concatenate([wt[idx], CC_SCALE * CC_SCALE * wt2[:4 * n1]])
        raw.append((uv, wt))
    qg = korder + 1 if korder + 1 >= 8 else korder + 3
    fac = 2.0 * wt1.sum()
    out = []
    for il, (uv, wt) in enumerate(raw, start=1):
        nsub = uv.shape[0] // n1
        if square and il >= 2:
            cc = il == nlevel == 4
            uv, wt, so, st = _squares(uv, wt, n1, 8 if cc else 2 ** (il - 1), nsub - 4 if cc else nsub, qg, fac)
        else:
            so, st = np.arange(nsub + 1) * n1, np.zeros(nsub, np.int64)
        out.append(dict(uv=uv, wt=wt, suboff=so, subtyp=st))
    return out
