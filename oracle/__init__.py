"""Oracle: CPU restatement of the RRQ near-field hot path (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
may import this package, and only as the checker or the timed CPU baseline.
The library (``qotential_b200``) never imports it.

Parity pin: the restatement is checked against the reference's frozen native
fixtures (``web/stellarator/fixtures/native/order{4,6}-direct.bin``), whose
relevant fields are committed under tests/golden/, and against the reference's
own C geometry generator (``utils/stellarator_geo_mex.c``) compiled from its
source into ``oracle/_ref/`` by ``oracle/Makefile``.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_geo = None

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
i64 = C.c_longlong


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liborc.so missing: run `make -C oracle`")
        _lib = C.CDLL(path)
    return _lib


def build():
    """Compile the oracle (and oracle/_ref when the reference checkout exists)."""
    import subprocess
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def set_refine(iadap):
    """the reference test's iadap (test/stellarator_grf.f90:46-47): 0 square
    levels (default), 1 the adaptive tree walk, 3 plain 4-split levels"""
    assert lib().orc_set_refine(C.c_int(int(iadap))) == 0


def set_simd(isimd):
    """Kernel-matrix sums with AVX2 over 4 targets (isimd = 256, the
    reference's SIMD path) or scalar (0); both give the same results."""
    lib().orc_set_simd(C.c_int(int(isimd)))


def gauss(n):
    x = np.zeros(n); w = np.zeros(n); D = np.zeros((n, n))
    lib().orc_gauss(C.c_int(n), _vp(x), _vp(w), _vp(D))
    return x, w, D.reshape(n, n).T.copy()   # return D in row-major math layout


def simplex_precomp(nquad, korder):
    kp = (korder + 1) * (korder + 2) // 2
    out = [np.zeros(nquad), np.zeros(nquad), np.zeros(nquad * nquad), np.zeros(nquad),
           np.zeros(nquad * nquad), np.zeros(kp * kp), np.zeros(kp * kp)]
    rc = lib().orc_simplex_precomp(C.c_int(nquad), C.c_int(korder), C.c_int(kp), *[_vp(a) for a in out])
    assert rc == 0
    return out


def ref_levels(korder, orderff, nlevel=4, sq=True):
    n = np.zeros(nlevel, np.int64); ns = np.zeros(nlevel, np.int64)
    lib().orc_ref_level_sizes(C.c_int(korder), C.c_int(orderff), C.c_int(nlevel), C.c_int(int(sq)), _vp(n), _vp(ns))
    npols = (korder + 1) * (korder + 2) // 2
    levs = []
    for l in range(nlevel):
        uv = np.zeros(2 * n[l]); wt = np.zeros(n[l]); it = np.zeros(n[l] * npols)
        so = np.zeros(ns[l] + 1, np.int64); st = np.zeros(ns[l], np.int64)
        lib().orc_ref_level_get(C.c_int(korder), C.c_int(orderff), C.c_int(nlevel), C.c_int(int(sq)), C.c_int(l),
                                _vp(uv), _vp(wt), _vp(it), _vp(so), _vp(st))
        levs.append(dict(n=int(n[l]), nsub=int(ns[l]), uv=uv.reshape(-1, 2), wt=wt,
                         interp=it.reshape(npols, n[l]).T.copy(), suboff=so, subtyp=st))
    return levs


def sdlpmat(tx, sx, snx, sw):
    tx = _f64(tx); sx = _f64(sx); snx = _f64(snx); sw = _f64(sw)
    m = tx.size // 3; n = sw.size
    A = np.zeros(m * n); B = np.zeros(m * n)
    lib().orc_sdlpmat(i64(m), _vp(tx), i64(n), _vp(sx), _vp(snx), _vp(sw), _vp(A), _vp(B))
    return A.reshape(n, m).T.copy(), B.reshape(n, m).T.copy()


def sdlpmat_levels(korder, sx, rts, rps, orderff, dist, tx, nlevel=4):
    sx = _f64(sx); rts = _f64(rts); rps = _f64(rps); tx = _f64(tx)
    npols = (korder + 1) * (korder + 2) // 2
    m = tx.size // 3
    As = np.zeros(m * npols); Ad = np.zeros(m * npols)
    idxs = np.zeros(m, np.int64); ms = np.zeros(1, np.int64); lvl = np.zeros(m, np.int64)
    rc = lib().orc_sdlpmat_levels(C.c_int(korder), C.c_int(npols), _vp(sx), _vp(rts), _vp(rps),
                                  C.c_int(orderff), C.c_double(dist), C.c_int(nlevel), i64(m), _vp(tx),
                                  _vp(As), _vp(Ad), _vp(idxs), _vp(ms), _vp(lvl))
    assert rc == 0
    return (As.reshape(npols, m).T.copy(), Ad.reshape(npols, m).T.copy(), idxs[:ms[0]].copy(), lvl)


def rrq(tx, sx, snx, sw, rts, rps, nterms, nquad, orderff, distff=1.4, exterior=True,
        ichart=0, sxbd_chart=None, rv_chart=None, force=False):
    tx = _f64(tx); sx = _f64(sx); snx = _f64(snx); sw = _f64(sw); rts = _f64(rts); rps = _f64(rps)
    m = tx.size // 3; n = sw.size; hd = nterms * (nterms + 1) // 2
    As = np.zeros(m * n); Ad = np.zeros(m * n); Om = np.zeros(4 * hd * m); Ia = np.zeros(m)
    lvl = np.zeros(m, np.int64)
    flag = (1 if exterior else 0) | (2 if force else 0)
    sb = _f64(sxbd_chart) if sxbd_chart is not None else None
    rv = _f64(rv_chart) if rv_chart is not None else None
    rc = lib().orc_rrq(i64(m), _vp(tx), i64(n), _vp(sx), _vp(snx), _vp(sw), _vp(rts), _vp(rps),
                       C.c_int(nterms), C.c_int(nquad), C.c_int(orderff), C.c_double(distff), C.c_int(flag),
                       C.c_int(ichart), _vp(sb), _vp(rv), _vp(As), _vp(Ad), _vp(Om), _vp(Ia), _vp(lvl))
    if rc != 0:
        raise RuntimeError(f"orc_rrq failed ({rc})")
    return (As.reshape(n, m).T.copy(), Ad.reshape(n, m).T.copy(), Om.reshape(m, 4 * hd).T.copy(), Ia, lvl)


def rrq_panel_systems(sx, snx, sw, nterms):
    """The D system A (4hd x 4hd, real form of the quaternion system) and the
    S system Msl^T (hd x hd) that the panel precompute factors
    (src/lap3d_close_mod.f90:851-863), as row-major math matrices."""
    hd = nterms * (nterms + 1) // 2
    DT = np.zeros(16 * hd * hd); MT = np.zeros(hd * hd)
    rc = lib().orc_rrq_panel_systems(C.c_int(nterms), _vp(_f64(sx)), _vp(_f64(snx)), _vp(_f64(sw)), _vp(DT), _vp(MT))
    if rc != 0:
        raise RuntimeError(f"orc_rrq_panel_systems failed ({rc})")
    # DT holds A^T column-major, i.e. A row-major; MT holds Msl^T column-major
    return DT.reshape(4 * hd, 4 * hd).copy(), MT.reshape(hd, hd).T.copy()


def getnearquad(npan, nterms, nquad, sx, snx, sw, rts, rps, tcx, tcxrow, tcxi, orderff,
                distff=1.4, iside=30, nthreads=0, pair_levels=False):
    """qol_getnearquad_lap_rrq restated; tcxrow/tcxi 1-based like the reference.
    With pair_levels, also returns each pair's resolving level (1-4 direct
    levels, 5 RRQ) in CSR order."""
    hdim = nterms * (nterms + 1) // 2
    sx = _f64(sx); snx = _f64(snx); sw = _f64(sw); rts = _f64(rts); rps = _f64(rps)
    tcx = _f64(tcx); tcxrow = _i64(tcxrow); tcxi = _i64(tcxi)
    ntcx = tcxrow.size; nsrc = sw.size; nnz = ntcx * hdim
    si = np.zeros(nnz, np.int64); sj = np.zeros(nnz, np.int64)
    vs = np.zeros(nnz); vd = np.zeros(nnz); hist = np.zeros(6, np.int64)
    lv = np.zeros(ntcx, np.int64) if pair_levels else None
    rc = lib().orc_getnearquad(i64(npan), C.c_int(nterms), i64(hdim), C.c_int(nquad), i64(nsrc),
                               _vp(sx), _vp(snx), _vp(sw), _vp(rts), _vp(rps), i64(ntcx), _vp(tcx),
                               _vp(tcxrow), _vp(tcxi), C.c_int(orderff), C.c_double(distff), i64(iside),
                               i64(nnz), _vp(si), _vp(sj), _vp(vs), _vp(vd), C.c_int(nthreads), _vp(hist),
                               _vp(lv))
    if rc != 0:
        raise RuntimeError(f"orc_getnearquad failed ({rc})")
    return (si, sj, vs, vd, hist, lv) if pair_levels else (si, sj, vs, vd, hist)


def ballcsr(npan, hdim, sx, sw, nthreads=0):
    """ball count + CSR fill of the GRF driver; csr_idx 1-based."""
    sx = _f64(sx); sw = _f64(sw); nsrc = sw.size
    cnt = np.zeros(npan, np.int64)
    lib().orc_ballcount(i64(npan), i64(hdim), i64(nsrc), _vp(sx), _vp(sw), _vp(cnt), C.c_int(nthreads))
    offs = np.zeros(npan + 1, np.int64); offs[1:] = np.cumsum(cnt)
    idx = np.zeros(int(offs[-1]), np.int64)
    lib().orc_ballfill(i64(npan), i64(hdim), i64(nsrc), _vp(sx), _vp(sw), _vp(offs), _vp(idx), C.c_int(nthreads))
    return offs, idx


def direct_farfield(sx, snx, sw, ub, ubn, nthreads=0):
    sx = _f64(sx); snx = _f64(snx); sw = _f64(sw); ub = _f64(ub); ubn = _f64(ubn)
    u = np.zeros(sw.size)
    lib().orc_direct_farfield(i64(sw.size), _vp(sx), _vp(snx), _vp(sw), _vp(ub), _vp(ubn), _vp(u), C.c_int(nthreads))
    return u


def grf_near(npan, nterms, nquad, orderff, sx, snx, sw, rts, rps, ub, ubn, offs, csr_idx, u,
             distff=1.4, exterior=True, xbuf=None, nthreads=0):
    """the GRF driver's near phase; returns (u + near corrections, csr_val, level histogram)"""
    u = _f64(u).copy()
    cv = np.zeros(int(offs[-1])); hist = np.zeros(6, np.int64)
    xb = _f64(xbuf) if xbuf is not None else None
    rc = lib().orc_grf_near(i64(npan), C.c_int(nterms), C.c_int(nquad), C.c_int(orderff), C.c_double(distff),
                            C.c_int(int(exterior)), C.c_int(1 if xbuf is not None else 0), _vp(xb),
                            _vp(_f64(sx)), _vp(_f64(snx)), _vp(_f64(sw)), _vp(_f64(rts)), _vp(_f64(rps)),
                            _vp(_f64(ub)), _vp(_f64(ubn)), _vp(_i64(offs)), _vp(_i64(csr_idx)), _vp(u), _vp(cv),
                            C.c_int(nthreads), _vp(hist))
    if rc != 0:
        raise RuntimeError(f"orc_grf_near failed ({rc})")
    return u, cv, hist


# ---------------- the reference's geometry generator (oracle/_ref) ----------------
def refgeo():
    global _geo
    if _geo is None:
        path = os.path.join(_HERE, "_ref", "libstellgeo.so")
        if not os.path.exists(path):
            return None
        _geo = C.CDLL(path)
    return _geo


def ref_geometry(mp, np_, nterms):
    """utils/stellarator_geo_mex.c:stellarator_geo on the built-in surface."""
    g = refgeo()
    if g is None:
        raise RuntimeError("oracle/_ref/libstellgeo.so missing")
    x0, w0, D = gauss(nterms)
    Dcm = np.asfortranarray(D).ravel(order="F").copy()
    uvs = np.zeros(2 * nterms * (nterms + 1) // 2)
    wts = np.zeros(nterms * (nterms + 1) // 2)
    lib().orc_vr_nodes_export(C.c_int(nterms - 1), _vp(uvs), _vp(wts))
    mpv, npv, pv = i64(mp), i64(np_), i64(nterms)
    g.stellarator_geo_ntri.restype = i64
    ntri = g.stellarator_geo_ntri(C.byref(mpv), C.byref(npv), C.byref(pv), _vp(x0))
    hd = nterms * (nterms + 1) // 2
    nsrc = ntri * hd
    sx = np.zeros(3 * nsrc); snx = np.zeros(3 * nsrc); sw = np.zeros(nsrc)
    rts = np.zeros(3 * nsrc); rps = np.zeros(3 * nsrc)
    g.stellarator_geo(C.byref(mpv), C.byref(npv), C.byref(pv), _vp(x0), _vp(Dcm), _vp(uvs), _vp(wts),
                      _vp(sx), _vp(snx), _vp(sw), _vp(rts), _vp(rps))
    return dict(ntri=int(ntri), sx=sx, snx=snx, sw=sw, rts=rts, rps=rps, x0=x0, D=Dcm)


def _modes_args(modes, nfp):
    m = np.asarray(modes, float).reshape(-1, 4)
    mn = np.ascontiguousarray(m[:, :2].ravel())
    rc, zs = np.ascontiguousarray(m[:, 2]), np.ascontiguousarray(m[:, 3])
    return [C.byref(i64(nfp)), C.byref(i64(m.shape[0])), _vp(mn), _vp(rc), _vp(zs)], (mn, rc, zs)


def ref_charts(mp, np_, p, modes, nfp, restol, cap=200000):
    """utils/stellarator_geo_mex.c:stellarator_charts (build_charts_adaptive)
    on the surface with VMEC modes (m, n, rc, zs): (nchart, 6) charts"""
    g = refgeo()
    if g is None:
        raise RuntimeError("oracle/_ref/libstellgeo.so missing")
    x0, _, D = gauss(p)
    Dcm = np.asfortranarray(D).ravel(order="F").copy()
    sargs, keep = _modes_args(modes, nfp)
    g.stellarator_charts.restype = i64
    args = [C.byref(i64(mp)), C.byref(i64(np_)), C.byref(i64(p)), _vp(x0), _vp(Dcm)] + sargs + \
           [C.byref(C.c_double(restol)), C.byref(i64(cap))]
    n = g.stellarator_charts(*args, None)
    if n < 0:
        raise RuntimeError("stellarator_charts: over cap")
    cl = np.zeros(6 * n)
    g.stellarator_charts(*args, _vp(cl))
    return cl.reshape(-1, 6)


def ref_geometry_charts(charts, mp, np_, nterms, modes, nfp):
    """utils/stellarator_geo_mex.c:stellarator_geo_charts: the panels of a chart list"""
    g = refgeo()
    x0, _, D = gauss(nterms)
    Dcm = np.asfortranarray(D).ravel(order="F").copy()
    hd = nterms * (nterms + 1) // 2
    uvs = np.zeros(2 * hd); wts = np.zeros(hd)
    lib().orc_vr_nodes_export(C.c_int(nterms - 1), _vp(uvs), _vp(wts))
    cl = np.ascontiguousarray(np.asarray(charts, float).ravel())
    n = cl.size // 6
    nsrc = 2 * n * hd
    out = {k: np.zeros(3 * nsrc) for k in ("sx", "snx", "rts", "rps")}
    out["sw"] = np.zeros(nsrc)
    sargs, keep = _modes_args(modes, nfp)
    g.stellarator_geo_charts(_vp(cl), C.byref(i64(n)), C.byref(i64(mp)), C.byref(i64(np_)), C.byref(i64(nterms)),
                             _vp(x0), _vp(Dcm), _vp(uvs), _vp(wts), *sargs, _vp(out["sx"]), _vp(out["snx"]),
                             _vp(out["sw"]), _vp(out["rts"]), _vp(out["rps"]))
    return out


def ref_uv2x(mp, np_, nterms, itri, uv):
    g = refgeo()
    x0, _, _ = gauss(nterms)
    uv = _f64(uv)
    nuv = uv.size // 2
    x = np.zeros(3 * nuv)
    g.stellarator_geo_uv2x(C.byref(i64(mp)), C.byref(i64(np_)), C.byref(i64(nterms)), _vp(x0),
                           C.byref(i64(itri)), C.byref(i64(nuv)), _vp(uv), _vp(x))
    return x
