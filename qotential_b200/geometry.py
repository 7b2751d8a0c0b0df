"""Synthetic inputs for the near-field path: triangulated Fourier surfaces and
near-target lists.

Surfaces follow the reference's geometry generator
(``utils/stellarator_geo_mex.c``): a (toroidal t, poloidal p) grid of
mp x np charts (aspect split at 1.65, ``build_charts`` :125-160), each chart
sampled on a p x p Gauss-Legendre tensor grid, derivatives by the spectral
differentiation matrix, and two Vioreanu-Rokhlin triangles per chart by 1D
polynomial interpolation (``geo_core`` :636-750).  Boundary modes use the VMEC
convention of ``surf_eval`` (:91-102):
    R = sum rc cos(m p - nfp n t),  Z = sum zs sin(m p - nfp n t).
This is input preparation (host numpy), not part of the measured path.
"""
import ctypes as C
import math

import numpy as np

ASPECT = 1.65


def gauss(n):
    """Gauss-Legendre nodes (ascending), weights and differentiation matrix
    D[i,k] (restated from utils/gauss.m)."""
    x, w = np.polynomial.legendre.leggauss(n)
    D = np.zeros((n, n))
    a = np.array([np.prod([x[k] - x[i] for i in range(n) if i != k]) for k in range(n)])
    for k in range(n):
        for i in range(n):
            if i != k:
                D[i, k] = (a[i] / a[k]) / (x[i] - x[k])
        D[k, k] = sum(1.0 / (x[k] - x[i]) for i in range(n) if i != k)
    return x, w, D


def vr_nodes(deg):
    """Vioreanu-Rokhlin nodes/weights of degree deg from the library's table."""
    from . import _vrtable
    return _vrtable.nodes(deg)


class Surface:
    """A Fourier boundary: modes = [(m, n, rc, zs), ...], nfp field periods."""

    def __init__(self, modes, nfp=1):
        self.modes = np.array(modes, dtype=np.float64).reshape(-1, 4)
        self.nfp = nfp

    def eval(self, t, p):
        t = np.asarray(t, dtype=np.float64)
        p = np.asarray(p, dtype=np.float64)
        R = np.zeros(np.broadcast(t, p).shape)
        Z = np.zeros_like(R)
        for m, n, rc, zs in self.modes:
            ang = m * p - self.nfp * n * t
            R = R + rc * np.cos(ang)
            Z = Z + zs * np.sin(ang)
        return np.stack([R * np.cos(t), R * np.sin(t), Z], axis=-1)

    def vmec_modes(self):
        """(modes (nmode x 4: m, n, rc, zs), nfp) for the GPU generator."""
        return np.ascontiguousarray(self.modes), self.nfp

    def rz(self, t, p):
        R = 0.0 * t; Z = 0.0 * t
        for m, n, rc, zs in self.modes:
            ang = m * p - self.nfp * n * t
            R = R + rc * np.cos(ang)
            Z = Z + zs * np.sin(ang)
        return R, Z


class BuiltinSurface:
    """The reference's built-in 7-term test surface (stellaratorparam,
    utils/stellarator_geo_mex.c:61-77), t toroidal, p poloidal."""

    nfp = 1

    def vmec_modes(self):
        """The same surface in the VMEC convention (nfp 1): R = sum rc cos(m p -
        n t), Z = sum zs sin(m p - n t), x = (R cos t, R sin t, Z); the cos p and
        sin p terms of the reference's formula combine into one mode (0.75, 1.25)."""
        modes = [(2, 1, 0.17, 0.17), (2, 0, 0.11, 0.11), (1, 0, 0.75, 1.25), (0, 0, 4.5, 0.0),
                 (1, -1, 0.07, 0.07), (1, 1, -0.45, 0.45)]
        return np.ascontiguousarray(np.array(modes, dtype=np.float64)), 1

    def eval(self, t, p):
        t = np.asarray(t, dtype=np.float64); p = np.asarray(p, dtype=np.float64)
        ct, st = np.cos(t), np.sin(t)
        c2pt, s2pt = np.cos(2.0 * p - t), np.sin(2.0 * p - t)
        c2p, s2p = np.cos(2.0 * p), np.sin(2.0 * p)
        cp, sp = np.cos(p), np.sin(p)
        cpt, spt = np.cos(p + t), np.sin(p + t)
        cmpt, smpt = np.cos(-p + t), np.sin(-p + t)
        x = (0.17 * ct * c2pt + 0.11 * ct * c2p + 1.0 * ct * cp + 4.5 * ct
             - 0.25 * ct * cp + 0.07 * ct * cpt - 0.45 * ct * cmpt)
        y = (0.17 * st * c2pt + 0.11 * st * c2p + 1.0 * st * cp + 4.5 * st
             - 0.25 * st * cp + 0.07 * st * cpt - 0.45 * st * cmpt)
        z = (0.17 * s2pt + 0.11 * s2p + 1.0 * sp + 0.0
             + 0.25 * sp + 0.07 * spt - 0.45 * smpt)
        return np.stack([x, y, z], axis=-1)


def torus():
    """R = 2 + cos p, Z = sin p (the order-4 CPU configuration's torus)."""
    return Surface([(0, 0, 2.0, 0.0), (1, 0, 1.0, 1.0)], nfp=1)


def stellarator():
    """R = 5 + cos p + 0.25 cos(p - 5t), Z = sin p - 0.25 sin(p - 5t)."""
    return Surface([(0, 0, 5.0, 0.0), (1, 0, 1.0, 1.0), (1, 1, 0.25, -0.25)], nfp=5)


def _interp_1d(t, s):
    """Lagrange interpolation matrix L[i, j] from nodes s to points t."""
    p = len(s)
    L = np.zeros((len(t), p))
    for j in range(p):
        num = np.ones(len(t))
        den = 1.0
        for k in range(p):
            if k != j:
                num = num * (t - s[k])
                den *= (s[j] - s[k])
        L[:, j] = num / den
    return L


def _charts(surf, mp, np_, x0, split=True):
    ts1, ts2 = math.pi / np_, math.pi / mp
    cl = []
    for j in range(1, np_ + 1):
        for i in range(1, mp + 1):
            def ev(t1, t2):
                return surf.eval((t1 + 2.0 * j) * ts1, (t2 + 2.0 * i) * ts2)
            xll, xul, xlr = ev(x0[0], x0[0]), ev(x0[0], x0[-1]), ev(x0[-1], x0[0])
            dt = np.linalg.norm(xll - xlr); dp = np.linalg.norm(xll - xul)
            base = dict(a1=1.0, b1=0.0, a2=1.0, b2=0.0, jj=float(j), ii=float(i))
            if split and dt / dp > ASPECT:
                cl += [dict(base, a1=0.5, b1=-0.5), dict(base, a1=0.5, b1=0.5)]
            elif split and dp / dt > ASPECT:
                cl += [dict(base, a2=0.5, b2=-0.5), dict(base, a2=0.5, b2=0.5)]
            else:
                cl.append(base)
    return cl


def panels(surf, mp, np_, nterms, split=True):
    """Panel geometry in the reference layout: dict(sx, snx, sw, rts, rps) as
    (nsrc, 3)/(nsrc,) arrays, nsrc = ntri * hdim, hdim = nterms(nterms+1)/2.
    split=False keeps the uniform mp x np grid (no aspect split)."""
    p = nterms
    x0, _, D = gauss(p)
    uvs, wts = vr_nodes(p - 1)
    hd = len(wts)
    ts1, ts2 = math.pi / np_, math.pi / mp
    cl = _charts(surf, mp, np_, x0, split)
    # interpolation from the tensor grid to the four triangle node sets
    u = 2.0 * uvs[:, 0] - 1.0; v = 2.0 * uvs[:, 1] - 1.0
    sets = {"lA": (u, v), "rA": (-u, -v), "lB": (v, -u), "rB": (-v, u)}
    Mt = {}
    for key, (t1, t2) in sets.items():
        L1 = _interp_1d(t1, x0); L2 = _interp_1d(t2, x0)
        # node (a: t2 index, b: t1 index) -> weight L1[i,b] L2[i,a]
        Mt[key] = np.einsum("ib,ia->iba", L1, L2).reshape(hd, p * p)
    b_idx, a_idx = np.meshgrid(np.arange(p), np.arange(p), indexing="ij")  # node m = a + b p
    a_flat = np.zeros(p * p, int); b_flat = np.zeros(p * p, int)
    for b in range(p):
        for a in range(p):
            a_flat[a + b * p] = a; b_flat[a + b * p] = b
    out = {k: [] for k in ("sx", "snx", "sw", "rts", "rps")}
    for c in cl:
        t1 = x0[b_flat]; t2 = x0[a_flat]
        uu = ((c["a1"] * t1 + c["b1"]) + 2.0 * c["jj"]) * ts1
        vv = ((c["a2"] * t2 + c["b2"]) + 2.0 * c["ii"]) * ts2
        sxk = surf.eval(uu, vv)                     # (p*p, 3), node m = a + b p
        G = sxk.reshape(p, p, 3)                    # [b, a, :]
        rts = np.einsum("rk,bkd->brd", D, G).reshape(p * p, 3)   # d/d(a index)
        rps = np.einsum("ck,kad->cad", D, G).reshape(p * p, 3)   # d/d(b index)
        d1 = np.sum((sxk[0] - sxk[p * p - 1]) ** 2)
        d2 = np.sum((sxk[p - 1] - sxk[p * p - p]) ** 2)
        keys = ("lA", "rA") if d1 + 1e-13 > d2 else ("lB", "rB")
        S = np.concatenate([sxk, rts, rps], axis=1)  # (p*p, 9)
        for key in keys:
            acc = Mt[key] @ S
            xt = acc[:, 3:6]; xp = acc[:, 6:9]
            nx = np.cross(xp, xt)
            sp = np.linalg.norm(nx, axis=1)
            out["sx"].append(acc[:, 0:3]); out["snx"].append(nx / sp[:, None])
            out["rts"].append(2.0 * xt); out["rps"].append(2.0 * xp)
            out["sw"].append(sp * wts * 4.0)
    res = {k: np.concatenate(v, axis=0) for k, v in out.items()}
    res["ntri"] = 2 * len(cl)
    res["hdim"] = hd
    return res


def panel_uv2x(surf, mp, np_, nterms, uv, split=True):
    """Surface points at reference-triangle coordinates uv (nuv x 2) of every
    triangle, through the chart map (uv2x_core, stellarator_geo_mex.c:555-584):
    returns (ntri, 3*nuv), x,y,z per point."""
    p = nterms
    x0, _, _ = gauss(p)
    ts1, ts2 = math.pi / np_, math.pi / mp
    cl = _charts(surf, mp, np_, x0, split)
    uv = np.asarray(uv, dtype=np.float64).reshape(-1, 2)
    out = []
    for c in cl:
        def ev(t1, t2):
            return surf.eval(((c["a1"] * t1 + c["b1"]) + 2.0 * c["jj"]) * ts1,
                             ((c["a2"] * t2 + c["b2"]) + 2.0 * c["ii"]) * ts2)
        xll, xur = ev(x0[0], x0[0]), ev(x0[p - 1], x0[p - 1])
        xul, xlr = ev(x0[0], x0[p - 1]), ev(x0[p - 1], x0[0])
        d1 = np.sum((xll - xur) ** 2); d2 = np.sum((xul - xlr) ** 2)
        for side in (0, 1):
            if d1 + 1e-13 > d2:
                V = [(-1, -1), (1, -1), (-1, 1)] if side == 0 else [(1, 1), (-1, 1), (1, -1)]
            else:
                V = [(-1, 1), (-1, -1), (1, 1)] if side == 0 else [(1, -1), (1, 1), (-1, -1)]
            t1 = V[0][0] + (V[1][0] - V[0][0]) * uv[:, 0] + (V[2][0] - V[0][0]) * uv[:, 1]
            t2 = V[0][1] + (V[1][1] - V[0][1]) * uv[:, 0] + (V[2][1] - V[0][1]) * uv[:, 1]
            out.append(ev(t1, t2).ravel())
    return np.stack(out)


def near_lists(sx, sw, hdim, targets=None, factor=1.75):
    """Ball-test near lists of the reference's GRF driver
    (stellarator_grf_core_mod.f90:652-688): for each panel, the targets within
    factor*sqrt(panel area) of the panel's node mean, in target order.
    Returns (tcxi 1-based, tcxrow 1-based, tcx)."""
    from scipy.spatial import cKDTree
    sx = np.asarray(sx).reshape(-1, 3)
    sw = np.asarray(sw).ravel()
    npan = sw.size // hdim
    T = sx if targets is None else np.asarray(targets).reshape(-1, 3)
    qp = sx.reshape(npan, hdim, 3).sum(1) / hdim
    qr = factor * np.sqrt(sw.reshape(npan, hdim).sum(1))
    tree = cKDTree(T)
    rows = []
    counts = np.zeros(npan, np.int64)
    for k in range(npan):
        cand = np.array(sorted(tree.query_ball_point(qp[k], qr[k] * (1 + 1e-12) + 1e-300)), dtype=np.int64)
        if cand.size:
            d2 = ((T[cand, 0] - qp[k, 0]) ** 2 + (T[cand, 1] - qp[k, 1]) ** 2 + (T[cand, 2] - qp[k, 2]) ** 2)
            cand = cand[d2 < qr[k] ** 2]
        rows.append(cand)
        counts[k] = cand.size
    tcxi = np.ones(npan + 1, np.int64)
    tcxi[1:] = 1 + np.cumsum(counts)
    tcxrow = np.concatenate(rows) + 1 if rows else np.zeros(0, np.int64)
    tcx = T[tcxrow - 1]
    return tcxi, tcxrow, tcx


def off_surface_targets(geo, nt, seed, hdim):
    """nt points at seeded surface nodes offset along +/- the normal by a
    distance log-uniform in [1e-6, 1e-1] times the local panel diameter."""
    rng = np.random.default_rng(seed)
    sx = geo["sx"].reshape(-1, 3); snx = geo["snx"].reshape(-1, 3); sw = geo["sw"].ravel()
    idx = rng.integers(0, sx.shape[0], nt)
    diam = np.sqrt(sw.reshape(-1, hdim).sum(1))[idx // hdim]
    d = 10.0 ** rng.uniform(-6.0, -1.0, nt) * diam
    sgn = np.where(rng.random(nt) < 0.5, -1.0, 1.0)
    return sx[idx] + (sgn * d)[:, None] * snx[idx]


def point_charges(surf, nq, seed, radius=6.0, clearance=0.1):
    """nq charges q ~ U(-1,1) at seeded points on |y| = radius, rejecting any
    point inside or within `clearance` of the solid torus (checked on (R, Z)
    against the poloidal cross-section at the point's toroidal angle)."""
    rng = np.random.default_rng(seed)
    ys, qs = [], []
    pp = np.linspace(0, 2 * math.pi, 721)
    while len(ys) < nq:
        v = rng.normal(size=3); v *= radius / np.linalg.norm(v)
        t = math.atan2(v[1], v[0]); Rv = math.hypot(v[0], v[1]); Zv = v[2]
        Rs, Zs = surf.rz(np.full_like(pp, t), pp)
        Rc = Rs.mean(); Zc = Zs.mean()
        ang = math.atan2(Zv - Zc, Rv - Rc)
        # boundary radius along that ray from the section centre
        ray = np.arctan2(Zs - Zc, Rs - Rc)
        k = np.argmin(np.abs(np.angle(np.exp(1j * (ray - ang)))))
        rb = math.hypot(Rs[k] - Rc, Zs[k] - Zc)
        if math.hypot(Rv - Rc, Zv - Zc) < rb + clearance:
            continue
        ys.append(v); qs.append(rng.uniform(-1, 1))
    return np.array(ys), np.array(qs)


def harmonic_density(x, n, charges, q):
    """u(x) = sum q_j/|x - y_j| and du/dn at points x with normals n."""
    x = np.asarray(x).reshape(-1, 3); n = np.asarray(n).reshape(-1, 3)
    u = np.zeros(len(x)); g = np.zeros_like(x)
    for y, qq in zip(charges, q):
        d = x - y
        r = np.linalg.norm(d, axis=1)
        u += qq / r
        g += -qq * d / r[:, None] ** 3
    return u, (g * n).sum(1)


def family_surface(rng):
    """A seeded surface of the batched family: R = R0 + a cos p + d cos(p - Nfp t),
    Z = a sin p - d sin(p - Nfp t), R0 ~ U(3, 6), a ~ U(0.5, 1.5), d ~ U(0, 0.3),
    Nfp in 1..5."""
    R0, a, d = rng.uniform(3.0, 6.0), rng.uniform(0.5, 1.5), rng.uniform(0.0, 0.3)
    nfp = int(rng.integers(1, 6))
    return Surface([(0, 0, R0, 0.0), (1, 0, a, a), (1, 1, d, -d)], nfp=nfp)
