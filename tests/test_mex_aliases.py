"""The reference's F77 link names (qol_*_mex_, every argument by reference,
no return value: matlab/qotential_mex.c:1096-1105 binds them so) against the
int-returning qol_* entry points: the same outputs byte for byte and the same
status in ier.  Host-only and argument-error cases run on CPU; the compute
cases on the GPU."""
import ctypes as C

import numpy as np
import pytest

I = C.c_longlong


def _r(v):
    return C.byref(I(v)) if isinstance(v, (int, np.integer)) else C.byref(C.c_double(v))


def _p(a):
    return C.c_void_p(a.ctypes.data)


def test_simplex_precomp_alias_matches(qol):
    L = qol.lib()
    nq, ko = 9, 6
    kp = (ko + 1) * (ko + 2) // 2
    outs = [np.zeros(n) for n in (nq, nq, nq * nq, nq, nq * nq, kp * kp, kp * kp)]
    ref = [np.zeros(n) for n in (nq, nq, nq * nq, nq, nq * nq, kp * kp, kp * kp)]
    L.qol_simplex_precomp_mex_(_r(nq), _r(ko), _r(kp), *[_p(a) for a in outs])
    assert L.qol_simplex_precomp(I(nq), I(ko), I(kp), *[_p(a) for a in ref]) == 0
    for a, b in zip(outs, ref):
        assert a.tobytes() == b.tobytes()


def test_error_status_through_ier(qol):
    """an unknown handle: status 2 in ier, as qol_lap3dsdlpmat_levels returns
    (patch_refine_mex.f90:79-93); clearing every handle: 0"""
    L = qol.lib()
    ier = np.full(1, -1, np.int64)
    L.qol_clear_patch_levels_all_mex_(_p(ier))
    assert ier[0] == 0
    m, npols = 3, 10
    tx = np.zeros(3 * m); As = np.zeros(m * npols); Ad = np.zeros(m * npols)
    idxs = np.zeros(m, np.int64); ms = np.zeros(1, np.int64)
    ier[0] = -1
    L.qol_lap3dsdlpmat_levels_mex_(_r(m), _p(tx), _r(npols), _r(12345), _r(0), _p(As), _p(Ad), _p(idxs), _p(ms),
                                   _p(ier))
    ier2 = np.full(1, -1, np.int64)
    rc = L.qol_lap3dsdlpmat_levels(I(m), _p(tx), I(npols), I(12345), I(0), _p(As), _p(Ad), _p(idxs), _p(ms),
                                   _p(ier2))
    assert ier[0] == ier2[0] == rc and rc != 0


@pytest.mark.gpu
def test_compute_aliases_match_on_gpu(qol):
    from qotential_b200 import geometry as G
    L = qol.lib()
    nterms = 6
    hd = nterms * (nterms + 1) // 2
    P = G.panels(G.torus(), 6, 12, nterms, split=False)
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 80, 9, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    npan = P["sw"].size // hd
    nq = nterms + 2
    nnz = int(tcxrow.size) * hd
    f = lambda a: np.ascontiguousarray(np.asarray(a, np.float64).ravel())
    sx, snx, sw, rts, rps = [f(P[k]) for k in ("sx", "snx", "sw", "rts", "rps")]
    tcxf = f(tcx); row = np.ascontiguousarray(tcxrow, np.int64); xi = np.ascontiguousarray(tcxi, np.int64)
    outs = [np.zeros(nnz, np.int64), np.zeros(nnz, np.int64), np.zeros(nnz), np.zeros(nnz), np.zeros(20)]
    ref = [np.zeros(nnz, np.int64), np.zeros(nnz, np.int64), np.zeros(nnz), np.zeros(nnz), np.zeros(20)]
    L.qol_getnearquad_lap_rrq_mex_(_r(npan), _r(nterms), _r(hd), _r(nq), _r(npan * hd), _p(sx), _p(snx), _p(sw),
                                   _p(rts), _p(rps), _r(int(row.size)), _p(tcxf), _p(row), _p(xi), _r(nq), _r(1.4),
                                   _r(30), _r(0), _r(nnz), *[_p(a) for a in outs])
    rc = L.qol_getnearquad_lap_rrq(I(npan), I(nterms), I(hd), I(nq), I(npan * hd), _p(sx), _p(snx), _p(sw), _p(rts),
                                   _p(rps), I(int(row.size)), _p(tcxf), _p(row), _p(xi), I(nq), C.c_double(1.4), I(30),
                                   I(0), I(nnz), *[_p(a) for a in ref])
    assert rc == 0
    for a, b in zip(outs[:4], ref[:4]):
        assert a.tobytes() == b.tobytes()
    # qol_rrq on one panel, targets its own nodes and neighbours
    k = 5
    sl = slice(3 * k * hd, 3 * (k + 1) * hd)
    geo = [np.ascontiguousarray(a[sl]) for a in (sx, snx, rts, rps)]
    swk = np.ascontiguousarray(sw[k * hd:(k + 1) * hd])
    txk = np.ascontiguousarray(sx[3 * (k - 1) * hd:3 * (k + 2) * hd])
    m = txk.size // 3
    tabs = [np.ascontiguousarray(np.asarray(t, np.float64).ravel(order="F"))
            for t in qol.qol_simplex_precomp(nq, nterms - 1, hd)]
    chart = np.zeros(3 * 3 * nq); rv = np.zeros(9)

    def call(fn, byref):
        out = [np.zeros(m * hd), np.zeros(m * hd), np.zeros(4 * hd * m), np.zeros(m), np.zeros(20)]
        g = _r if byref else (lambda v: I(v) if isinstance(v, int) else C.c_double(v))
        res = fn(g(m), _p(txk), g(hd), _p(geo[0]), _p(geo[1]), _p(swk), _p(geo[2]), _p(geo[3]), g(nterms), g(nq),
                 g(nq), g(1.4), g(1), g(0), g(0), _p(chart), _p(rv), *[_p(t) for t in tabs], *[_p(a) for a in out])
        return res, out

    _, a = call(L.qol_rrq_mex_, True)
    rc, b = call(L.qol_rrq, False)
    assert rc == 0
    for x, y in zip(a[:4], b[:4]):
        assert x.tobytes() == y.tobytes()
