"""qotential_b200: B200-native RRQ near-field hot path behind the reference's
qol_* operator API.

This module is the host-side mirror of the reference's MATLAB gateway
(``matlab/qotential.mw``): the same function names, argument meanings and
error behaviour, over the C ABI of ``libqol_b200.so`` (``include/qol_b200.h``).
There is no CPU fallback: if the CUDA library is missing, or no GPU is usable,
every compute function raises.
"""
import ctypes as C
import os

import numpy as np

__all__ = [
    "lib", "QolError", "qol_simplex_precomp", "qol_build_patch_levels", "qol_lap3dsdlpmat_levels",
    "qol_clear_patch_levels", "qol_clear_patch_levels_all", "qol_rrq", "qol_getnearquad_lap_rrq",
    "qol_getnearquad_lap_rrq_dev", "qol_getnearquad_lap_rrq_batch_dev", "qol_release_workspace", "qol_graph_stats", "qol_set_graphs",
    "qol_grf_near", "qol_grf_near_multi", "qol_grf_near_range", "qol_direct_farfield",
    "qol_direct_farfield_range", "qol_surface_panels", "qol_surface_charts", "qol_surface_panels_charts",
    "qol_interp_matrix", "qol_set_sum_precision",
    "SELECTOR_NW", "qol_selector_features", "qol_selector_grad", "qol_selector_train", "qol_selector_set",
    "qol_selector_stats", "qol_selector_force_level", "qol_set_patch_refine", "qol_ref_level_table",
    "qol_set_autotune",
    "qol_panel_shape",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libqol_b200.so")
_lib = None
i64 = C.c_longlong


class QolError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"qol status {code}: {msg}")
        self.code = code


def lib():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise QolError(5, f"{_LIB} is missing: build it with qotential_b200._build.build()")
        L = C.CDLL(_LIB)
        L.qol_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise QolError(rc, lib().qol_last_error().decode(errors="replace"))


def _vp(a):
    """a pointer to a's data that keeps a alive for the call (a temporary copy,
    e.g. of a strided column, would otherwise be freed before the call and its
    memory reused by the next argument's copy)"""
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f(a, n=None):
    """Flatten to the reference's memory layout.  Point arrays are accepted as
    (npts, 3) numpy arrays (row = point, the same bytes as the reference's
    column-major sx(3, npts)) or as (3, npts) Fortran-shaped arrays."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 2 and a.shape[0] == 3 and a.shape[1] != 3:
        a = a.T
    a = np.ascontiguousarray(a).ravel()
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _fm(a, n=None):
    """Flatten a matrix argument column-major (Fortran order), e.g. Dgl(n,n)."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _i(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).ravel(order="F"))


def qol_simplex_precomp(nquad, korder, kpols=None):
    """[tgl, wgl, Dgl, w_bclag, Legmat, umatr, vmatr] (matlab/qol_simplex_precomp_mex.m)."""
    kpols = (korder + 1) * (korder + 2) // 2 if kpols is None else kpols
    tgl = np.zeros(nquad); wgl = np.zeros(nquad); Dgl = np.zeros(nquad * nquad)
    wb = np.zeros(nquad); Leg = np.zeros(nquad * nquad)
    um = np.zeros(kpols * kpols); vm = np.zeros(kpols * kpols)
    _check(lib().qol_simplex_precomp(i64(nquad), i64(korder), i64(kpols), _vp(tgl), _vp(wgl), _vp(Dgl),
                                     _vp(wb), _vp(Leg), _vp(um), _vp(vm)))
    f = lambda a, n: a.reshape(n, n, order="F")
    return tgl, wgl, f(Dgl, nquad), wb, f(Leg, nquad), f(um, kpols), f(vm, kpols)


def qol_build_patch_levels(korder, sx, rts, rps, order, dist, nlevel=4):
    """lv handle (matlab/qol_build_patch_levels_mex.m); raises QolError with the ier code."""
    npols = (korder + 1) * (korder + 2) // 2
    lv = np.zeros(1, np.int64); ier = np.zeros(1, np.int64)
    rc = lib().qol_build_patch_levels(i64(korder), i64(npols), _vp(_f(sx, 3 * npols)), _vp(_f(rts, 3 * npols)),
                                      _vp(_f(rps, 3 * npols)), i64(order), C.c_double(dist), i64(nlevel),
                                      _vp(lv), _vp(ier))
    _check(rc)
    return int(lv[0])


def qol_lap3dsdlpmat_levels(tx, npols, lv, isimd=0, As=None, Ad=None):
    """[As, Ad, idxs, ms] (matlab/qol_lap3dsdlpmat_levels_mex.m); idxs 1-based."""
    tx = _f(tx)
    m = tx.size // 3
    As = np.zeros((m, npols)) if As is None else np.array(As, dtype=np.float64)
    Ad = np.zeros((m, npols)) if Ad is None else np.array(Ad, dtype=np.float64)
    Asf = _fm(As); Adf = _fm(Ad)
    idxs = np.zeros(max(m, 1), np.int64); ms = np.zeros(1, np.int64); ier = np.zeros(1, np.int64)
    rc = lib().qol_lap3dsdlpmat_levels(i64(m), _vp(tx), i64(npols), i64(lv), i64(isimd), _vp(Asf), _vp(Adf),
                                       _vp(idxs), _vp(ms), _vp(ier))
    _check(rc)
    return (Asf.reshape(m, npols, order="F"), Adf.reshape(m, npols, order="F"), idxs[:ms[0]].copy(), int(ms[0]))


def qol_clear_patch_levels(lv):
    ier = np.zeros(1, np.int64)
    _check(lib().qol_clear_patch_levels(i64(lv), _vp(ier)))


def qol_clear_patch_levels_all():
    ier = np.zeros(1, np.int64)
    _check(lib().qol_clear_patch_levels_all(_vp(ier)))


def qol_rrq(tx, sx, snx, sw, rts, rps, order, nquad, orderff, distff=1.4, exterior=True, isimd=0, ichart=0,
            sxbd_chart=None, rv_chart=None, tables=None, timeinfo=None):
    """[As, Ad, Omega, IalphaAsvestas, timeinfo] (matlab/qol_rrq_mex.m)."""
    hd = order * (order + 1) // 2
    tx = _f(tx); m = tx.size // 3
    if tables is None:
        tables = qol_simplex_precomp(nquad, order - 1, hd)
    tgl, wgl, Dgl, wb, Leg, um, vm = [_fm(t) for t in tables]
    As = np.zeros(m * hd); Ad = np.zeros(m * hd); Om = np.zeros(4 * hd * m); Ia = np.zeros(m)
    ti = np.zeros(20) if timeinfo is None else _f(timeinfo, 20).copy()
    nbd = 3 * nquad
    sb = _f(sxbd_chart, 3 * nbd) if sxbd_chart is not None else np.zeros(3 * nbd)
    rv = _f(rv_chart, 9) if rv_chart is not None else np.zeros(9)
    rc = lib().qol_rrq(i64(m), _vp(tx), i64(hd), _vp(_f(sx, 3 * hd)), _vp(_f(snx, 3 * hd)), _vp(_f(sw, hd)),
                       _vp(_f(rts, 3 * hd)), _vp(_f(rps, 3 * hd)), i64(order), i64(nquad), i64(orderff),
                       C.c_double(distff), i64(int(bool(exterior))), i64(isimd), i64(ichart), _vp(sb), _vp(rv),
                       _vp(tgl), _vp(wgl), _vp(Dgl), _vp(wb), _vp(Leg), _vp(um), _vp(vm), _vp(As), _vp(Ad),
                       _vp(Om), _vp(Ia), _vp(ti))
    _check(rc)
    return (As.reshape(m, hd, order="F"), Ad.reshape(m, hd, order="F"), Om.reshape(4 * hd, m, order="F"), Ia, ti)


def qol_getnearquad_lap_rrq(npan, nterms, hdim, nquad, nsrc, sx, snx, sw, rts, rps, ntcx, tcx, tcxrow, tcxi,
                            orderff, distff, iside, isimd=0, nnz=None, timeinfo=None, out=None):
    """[sparsei, sparsej, sparsevs, sparsevd, timeinfo] (matlab/qol_getnearquad_lap_rrq_mex.m).

    tcxrow/tcxi are 1-based; the COO output follows the reference's order
    (tcxi(k)-1)*hdim + (j-1)*m_k + i.  out=(sparsei, sparsej, sparsevs,
    sparsevd), contiguous int64/int64/float64/float64 arrays of nnz entries,
    are filled in place and returned (the C ABI's caller-allocated outputs, as
    a Fortran caller passes them; entries past the used ones are zeroed);
    without it fresh zeroed arrays are allocated."""
    tcxi = _i(tcxi)
    if hdim != nterms * (nterms + 1) // 2 or npan * hdim != nsrc:
        raise QolError(1, "The panel order, hdim, npan, and nsrc are inconsistent.")
    if tcxi[0] != 1 or np.any(np.diff(tcxi) < 0) or tcxi[-1] != ntcx + 1:
        raise QolError(1, "tcxi must be monotone, one-based, and cover tcx exactly.")
    need = int((tcxi[-1] - 1) * hdim)
    nnz = need if nnz is None else int(nnz)
    if need > nnz:
        raise QolError(2, "nnz is too small for the requested panel-target interactions.")
    if out is None:
        si = np.zeros(nnz, np.int64); sj = np.zeros(nnz, np.int64)
        vs = np.zeros(nnz); vd = np.zeros(nnz)
    else:
        si, sj, vs, vd = out
        for a, dt in ((si, np.int64), (sj, np.int64), (vs, np.float64), (vd, np.float64)):
            if not isinstance(a, np.ndarray) or a.dtype != dt or not a.flags.c_contiguous or a.size != nnz:
                raise QolError(1, "out must be four contiguous arrays (int64, int64, float64, float64) of nnz entries.")
        for a in (si, sj, vs, vd):
            a[need:] = 0
    ti = np.zeros(20) if timeinfo is None else _f(timeinfo, 20).copy()
    rc = lib().qol_getnearquad_lap_rrq(
        i64(npan), i64(nterms), i64(hdim), i64(nquad), i64(nsrc), _vp(_f(sx, 3 * nsrc)), _vp(_f(snx, 3 * nsrc)),
        _vp(_f(sw, nsrc)), _vp(_f(rts, 3 * nsrc)), _vp(_f(rps, 3 * nsrc)), i64(ntcx), _vp(_f(tcx, 3 * ntcx)),
        _vp(_i(tcxrow)), _vp(tcxi), i64(orderff), C.c_double(distff), i64(iside), i64(isimd), i64(nnz),
        _vp(si), _vp(sj), _vp(vs), _vp(vd), _vp(ti))
    _check(rc)
    return si, sj, vs, vd, ti


def qol_getnearquad_lap_rrq_dev(npan, nterms, nquad, sx, snx, sw, rts, rps, tcx, tcxrow, tcxi, orderff,
                                distff, iside, out, stream=0, sync=True, want_hist=False):
    """Device-resident form: every array argument is an object exposing
    ``data_ptr()`` (e.g. a CUDA torch tensor) or an integer device address.
    ``out`` = (sparsei, sparsej, sparsevs, sparsevd) device buffers of size nnz."""
    def ptr(a):
        return C.c_void_p(a if isinstance(a, int) else a.data_ptr())
    hdim = nterms * (nterms + 1) // 2
    si, sj, vs, vd = out
    nnz = vs.numel() if hasattr(vs, "numel") else int(out[4])
    ntcx = tcxrow.numel() if hasattr(tcxrow, "numel") else 0
    hist = np.zeros(6, np.int64)
    rc = lib().qol_getnearquad_lap_rrq_dev(
        i64(npan), i64(nterms), i64(hdim), i64(nquad), i64(npan * hdim), ptr(sx), ptr(snx), ptr(sw), ptr(rts),
        ptr(rps), i64(ntcx), ptr(tcx), ptr(tcxrow), ptr(tcxi), i64(orderff), C.c_double(distff), i64(iside),
        i64(nnz), ptr(si), ptr(sj), ptr(vs), ptr(vd), C.c_void_p(stream), C.c_int(int(sync)),
        _vp(hist) if want_hist else None)
    _check(rc)
    return hist if want_hist else None


class _NearJob(C.Structure):
    _fields_ = [("npan", C.c_longlong), ("nterms", C.c_longlong), ("hdim", C.c_longlong), ("nquad", C.c_longlong),
                ("nsrc", C.c_longlong), ("sx", C.c_void_p), ("snx", C.c_void_p), ("sw", C.c_void_p),
                ("rts", C.c_void_p), ("rps", C.c_void_p), ("ntcx", C.c_longlong), ("tcx", C.c_void_p),
                ("tcxrow", C.c_void_p), ("tcxi", C.c_void_p), ("orderff", C.c_longlong), ("distff", C.c_double),
                ("iside", C.c_longlong), ("nnz", C.c_longlong), ("sparsei", C.c_void_p), ("sparsej", C.c_void_p),
                ("sparsevs", C.c_void_p), ("sparsevd", C.c_void_p)]


def qol_getnearquad_lap_rrq_batch_dev(jobs, stream=0):
    """Batched device form: ``jobs`` is a list of dicts with npan, nterms,
    nquad, orderff (default nquad), distff (1.4), iside (30) and device arrays
    (objects with data_ptr(), e.g. CUDA tensors) sx, snx, sw, rts, rps, tcx,
    tcxrow, tcxi and out = (sparsei, sparsej, sparsevs, sparsevd).  One call;
    the level sums of all jobs in one persistent launch.  Returns the level
    histograms (njob x 6)."""
    ptr = lambda a: a if isinstance(a, int) else a.data_ptr()
    arr = (_NearJob * max(1, len(jobs)))()
    for k, j in enumerate(jobs):
        nterms = int(j["nterms"])
        hd = nterms * (nterms + 1) // 2
        si, sj, vs, vd = j["out"]
        nq = int(j["nquad"])
        arr[k] = _NearJob(int(j["npan"]), nterms, hd, nq, int(j["npan"]) * hd, ptr(j["sx"]), ptr(j["snx"]),
                          ptr(j["sw"]), ptr(j["rts"]), ptr(j["rps"]), int(j["tcxrow"].numel()), ptr(j["tcx"]),
                          ptr(j["tcxrow"]), ptr(j["tcxi"]), int(j.get("orderff", nq)), float(j.get("distff", 1.4)),
                          int(j.get("iside", 30)), int(vs.numel()), ptr(si), ptr(sj), ptr(vs), ptr(vd))
    hist = np.zeros((max(1, len(jobs)), 6), np.int64)
    _check(lib().qol_getnearquad_lap_rrq_batch_dev(i64(len(jobs)), arr, C.c_void_p(stream), _vp(hist)))
    return hist[:len(jobs)]


def qol_release_workspace():
    """free the device workspace the library keeps between calls"""
    _check(lib().qol_release_workspace())


def qol_set_graphs(enable):
    """1 (default): the device entry replays CUDA graphs of its back stage; 0: direct launches"""
    _check(lib().qol_set_graphs(C.c_int(int(enable))))


def qol_graph_stats():
    """(captured, replayed): CUDA graphs of the device entry's back stage since load"""
    c, r = C.c_longlong(0), C.c_longlong(0)
    _check(lib().qol_graph_stats(C.byref(c), C.byref(r)))
    return int(c.value), int(r.value)


def qol_grf_near(npan, nterms, nquad, sx, snx, sw, rts, rps, ub, ubn, u=None, orderff=None, distff=1.4,
                 iside=30, xbuf=None, timeinfo=None):
    """GRF near phase of the reference's stellarator driver
    (stellarator_grf_core_mod.f90:652-899): returns (u + near corrections,
    number of near pairs, pairs per resolving level [6]).  Targets are the
    surface's own nodes; ``u`` (default zeros) is added to, as the driver
    adds the near phase to its far field."""
    hd = nterms * (nterms + 1) // 2
    nsrc = npan * hd
    orderff = nquad if orderff is None else orderff
    uu = np.zeros(nsrc) if u is None else _f(u, nsrc).copy()
    nn = np.zeros(1, np.int64)
    hist = np.zeros(6, np.int64)
    ti = np.zeros(20) if timeinfo is None else _f(timeinfo, 20).copy()
    xb = None if xbuf is None else np.ascontiguousarray(np.asarray(xbuf, np.float64).ravel())
    rc = lib().qol_grf_near(i64(npan), i64(nterms), i64(nquad), i64(orderff), C.c_double(distff), i64(iside),
                            i64(nsrc), _vp(_f(sx, 3 * nsrc)), _vp(_f(snx, 3 * nsrc)), _vp(_f(sw, nsrc)),
                            _vp(_f(rts, 3 * nsrc)), _vp(_f(rps, 3 * nsrc)), _vp(xb), _vp(_f(ub, nsrc)),
                            _vp(_f(ubn, nsrc)), _vp(uu), _vp(nn), _vp(hist), _vp(ti))
    _check(rc)
    return uu, int(nn[0]), hist


def qol_grf_near_multi(npan, nterms, nquad, sx, snx, sw, rts, rps, ub, ubn, u=None, orderff=None, distff=1.4,
                       iside=30, xbuf=None, timeinfo=None):
    """qol_grf_near for several densities: ub, ubn (and u) of shape (nsrc,
    nrhs); the corrections are computed once and applied to each.  Returns
    (u (nsrc, nrhs), near pairs, level histogram)."""
    hd = nterms * (nterms + 1) // 2
    nsrc = npan * hd
    orderff = nquad if orderff is None else orderff
    ubm = np.asfortranarray(np.asarray(ub, np.float64).reshape(nsrc, -1))
    ubnm = np.asfortranarray(np.asarray(ubn, np.float64).reshape(nsrc, -1))
    nrhs = ubm.shape[1]
    if ubnm.shape != ubm.shape:
        raise QolError(8, "ub and ubn must have the same shape")
    uu = np.zeros((nsrc, nrhs), order="F") if u is None else np.array(np.asarray(u, np.float64).reshape(nsrc, nrhs),
                                                                      order="F")
    nn = np.zeros(1, np.int64)
    hist = np.zeros(6, np.int64)
    ti = np.zeros(20) if timeinfo is None else _f(timeinfo, 20).copy()
    xb = None if xbuf is None else np.ascontiguousarray(np.asarray(xbuf, np.float64).ravel())
    rc = lib().qol_grf_near_multi(i64(npan), i64(nterms), i64(nquad), i64(orderff), C.c_double(distff), i64(iside),
                                  i64(nsrc), _vp(_f(sx, 3 * nsrc)), _vp(_f(snx, 3 * nsrc)), _vp(_f(sw, nsrc)),
                                  _vp(_f(rts, 3 * nsrc)), _vp(_f(rps, 3 * nsrc)), _vp(xb), i64(nrhs), _vp(ubm),
                                  _vp(ubnm), _vp(uu), _vp(nn), _vp(hist), _vp(ti))
    _check(rc)
    return uu, int(nn[0]), hist


def qol_grf_near_range(npan, nterms, nquad, sx, snx, sw, rts, rps, ub, ubn, plo, phi, u=None, orderff=None,
                       distff=1.4, iside=30, xbuf=None, timeinfo=None):
    """qol_grf_near restricted to the panels [plo, phi): returns u plus their
    near corrections (all nodes stay targets).  The ranges of a partition of
    [0, npan) add up to qol_grf_near's corrections (multi-GPU split)."""
    hd = nterms * (nterms + 1) // 2
    nsrc = npan * hd
    orderff = nquad if orderff is None else orderff
    uu = np.zeros(nsrc) if u is None else _f(u, nsrc).copy()
    nn = np.zeros(1, np.int64)
    hist = np.zeros(6, np.int64)
    ti = np.zeros(20) if timeinfo is None else _f(timeinfo, 20).copy()
    xb = None if xbuf is None else np.ascontiguousarray(np.asarray(xbuf, np.float64).ravel())
    rc = lib().qol_grf_near_range(i64(npan), i64(nterms), i64(nquad), i64(orderff), C.c_double(distff), i64(iside),
                                  i64(nsrc), _vp(_f(sx, 3 * nsrc)), _vp(_f(snx, 3 * nsrc)), _vp(_f(sw, nsrc)),
                                  _vp(_f(rts, 3 * nsrc)), _vp(_f(rps, 3 * nsrc)), _vp(xb), _vp(_f(ub, nsrc)),
                                  _vp(_f(ubn, nsrc)), i64(plo), i64(phi), _vp(uu), _vp(nn), _vp(hist), _vp(ti))
    _check(rc)
    return uu


def qol_direct_farfield_range(sx, snx, sw, ub, ubn, tlo, thi, u):
    """Direct far field for the targets [tlo, thi) only, written into u
    (float64, nsrc, contiguous) in place."""
    sw = _f(sw)
    nsrc = sw.size
    if not (isinstance(u, np.ndarray) and u.dtype == np.float64 and u.flags.c_contiguous and u.size == nsrc):
        raise QolError(8, "u must be a contiguous float64 array of nsrc entries")
    rc = lib().qol_direct_farfield_range(i64(nsrc), _vp(_f(sx, 3 * nsrc)), _vp(_f(snx, 3 * nsrc)), _vp(sw),
                                         _vp(_f(ub, nsrc)), _vp(_f(ubn, nsrc)), i64(tlo), i64(thi), _vp(u))
    _check(rc)
    return u


def qol_surface_panels(surface, mp, np_, nterms, split=True):
    """The surface's panels from the GPU geometry generator (the reference's
    utils/stellarator_geo_mex.c geo_core): dict(sx, snx, sw, rts, rps) as
    (nsrc, 3)/(nsrc,) arrays, ntri, hdim, the layout geometry.panels gives.
    ``surface`` has vmec_modes() (geometry.Surface, geometry.BuiltinSurface)."""
    modes, nfp = surface.vmec_modes()
    modes = np.ascontiguousarray(np.asarray(modes, np.float64).reshape(-1, 4))
    nt = np.zeros(1, np.int64)
    args = (i64(modes.shape[0]), _vp(modes), i64(nfp), i64(mp), i64(np_), i64(nterms), i64(int(bool(split))))
    _check(lib().qol_surface_panels(*args, _vp(nt), None, None, None, None, None))
    hd = nterms * (nterms + 1) // 2
    nsrc = int(nt[0]) * hd
    out = {k: np.zeros((nsrc, 3)) for k in ("sx", "snx", "rts", "rps")}
    out["sw"] = np.zeros(nsrc)
    _check(lib().qol_surface_panels(*args, _vp(nt), _vp(out["sx"]), _vp(out["snx"]), _vp(out["sw"]),
                                    _vp(out["rts"]), _vp(out["rps"])))
    out["ntri"] = int(nt[0])
    out["hdim"] = hd
    return out


def qol_surface_charts(surface, mp, np_, p, restol, cap=200000):
    """(nchart, 6) adaptive charts (a1, b1, a2, b2, jj, ii) of the surface
    (utils/stellarator_geo_mex.c build_charts_adaptive): aspect splits, then
    for restol > 0 curvature refinement and 2:1 balance"""
    modes, nfp = surface.vmec_modes()
    modes = np.ascontiguousarray(np.asarray(modes, np.float64).reshape(-1, 4))
    n = np.zeros(1, np.int64)
    args = (i64(modes.shape[0]), _vp(modes), i64(nfp), i64(mp), i64(np_), i64(p), C.c_double(restol), i64(cap))
    _check(lib().qol_surface_charts(*args, _vp(n), None))
    cl = np.zeros(6 * int(n[0]))
    _check(lib().qol_surface_charts(*args, _vp(n), _vp(cl)))
    return cl.reshape(-1, 6)


def qol_surface_panels_charts(surface, mp, np_, nterms, charts):
    """the GPU geometry generator over a chart list: dict as qol_surface_panels"""
    modes, nfp = surface.vmec_modes()
    modes = np.ascontiguousarray(np.asarray(modes, np.float64).reshape(-1, 4))
    cl = np.ascontiguousarray(np.asarray(charts, np.float64).ravel())
    nt = np.zeros(1, np.int64)
    args = (i64(modes.shape[0]), _vp(modes), i64(nfp), i64(mp), i64(np_), i64(nterms), i64(cl.size // 6), _vp(cl))
    _check(lib().qol_surface_panels_charts(*args, _vp(nt), None, None, None, None, None))
    hd = nterms * (nterms + 1) // 2
    nsrc = int(nt[0]) * hd
    out = {k: np.zeros((nsrc, 3)) for k in ("sx", "snx", "rts", "rps")}
    out["sw"] = np.zeros(nsrc)
    _check(lib().qol_surface_panels_charts(*args, _vp(nt), _vp(out["sx"]), _vp(out["snx"]), _vp(out["sw"]),
                                           _vp(out["rts"]), _vp(out["rps"])))
    out["ntri"] = int(nt[0])
    out["hdim"] = hd
    return out


def qol_interp_matrix(korder, uv):
    """Matrix (n x npols) interpolating values at the degree-korder VR nodes to
    the reference-triangle points uv (n x 2)."""
    uv = np.ascontiguousarray(np.asarray(uv, np.float64).reshape(-1, 2))
    npols = (korder + 1) * (korder + 2) // 2
    M = np.zeros(uv.shape[0] * npols)
    _check(lib().qol_interp_matrix(i64(korder), i64(uv.shape[0]), _vp(uv), _vp(M)))
    return M.reshape(npols, uv.shape[0]).T.copy()


def qol_direct_farfield(sx, snx, sw, ub, ubn):
    """Direct far field u_i = sum_j S_ij ubn_j - D_ij ub_j, zero self term
    (stellarator_grf_core_mod.f90:566-606)."""
    sw = _f(sw)
    nsrc = sw.size
    u = np.zeros(nsrc)
    rc = lib().qol_direct_farfield(i64(nsrc), _vp(_f(sx, 3 * nsrc)), _vp(_f(snx, 3 * nsrc)), _vp(sw),
                                   _vp(_f(ub, nsrc)), _vp(_f(ubn, nsrc)), _vp(u))
    _check(rc)
    return u


def qol_set_sum_precision(mode):
    """0: FP64 level sums (default, the drop-in); 1: FP32 level sums, a 3xTF32
    contraction on the tcgen05 tensor cores, FP32 over 32-node tiles and
    compensated sums across them (precision variant)."""
    _check(lib().qol_set_sum_precision(C.c_int(int(mode))))


# ---------------- learned level selector (no reference counterpart) ----------------
SELECTOR_NW = 5061  # W1 8x64, b1 64, W2 64x64, b2 64, W3 64x5, b3 5


def qol_selector_features(npan, nterms, nquad, sx, snx, sw, rts, rps, tcx, tcxrow, tcxi, orderff, distff=1.4):
    """(features float32 (ntcx, 8), plain-walk level int8 (ntcx,), 1..5) of every
    near pair of a getnearquad input; the selector's classes are level - 1."""
    tcxi = _i(tcxi)
    tcxrow = _i(tcxrow)
    ntcx = tcxrow.size
    nsrc = int(npan) * (int(nterms) * (int(nterms) + 1) // 2)
    feat = np.zeros((ntcx, 8), np.float32)
    lev = np.zeros(ntcx, np.int8)
    rc = lib().qol_selector_features(i64(npan), i64(nterms), i64(nquad), _vp(_f(sx, 3 * nsrc)),
                                     _vp(_f(snx, 3 * nsrc)), _vp(_f(sw, nsrc)), _vp(_f(rts, 3 * nsrc)),
                                     _vp(_f(rps, 3 * nsrc)), i64(ntcx), _vp(_f(tcx, 3 * ntcx)), _vp(tcxrow),
                                     _vp(tcxi), i64(orderff), C.c_double(distff), _vp(feat), _vp(lev))
    _check(rc)
    return feat, lev


def _sel_args(feat, label):
    feat = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 8)
    label = np.ascontiguousarray(label, dtype=np.int8).reshape(-1)
    if label.size != feat.shape[0]:
        raise QolError(8, "one label per feature row")
    return feat, label


def qol_selector_grad(feat, label, w):
    """(mean cross-entropy, its gradient) of the MLP with weights w over the samples."""
    feat, label = _sel_args(feat, label)
    w = np.ascontiguousarray(w, dtype=np.float32)
    g = np.zeros(SELECTOR_NW, np.float32)
    loss = np.zeros(1)
    _check(lib().qol_selector_grad(i64(label.size), _vp(feat), _vp(label), _vp(w), _vp(g), _vp(loss)))
    return float(loss[0]), g


def qol_selector_init(seed=0):
    """He-initialised weights (zero biases), seeded."""
    rng = np.random.default_rng(seed)
    w = np.zeros(SELECTOR_NW, np.float32)
    w[0:512] = rng.normal(0.0, np.sqrt(2.0 / 8), 512)
    w[576:576 + 4096] = rng.normal(0.0, np.sqrt(2.0 / 64), 4096)
    w[4736:4736 + 320] = rng.normal(0.0, np.sqrt(1.0 / 64), 320)
    return w


def qol_selector_train(feat, label, w=None, epochs=20, batch=16384, lr=3e-3, seed=0):
    """(trained weights, mean loss per epoch): Adam on the GPU."""
    feat, label = _sel_args(feat, label)
    w = qol_selector_init(seed) if w is None else np.array(w, dtype=np.float32)
    loss = np.zeros(int(epochs))
    _check(lib().qol_selector_train(i64(label.size), _vp(feat), _vp(label), i64(epochs), i64(batch), C.c_double(lr),
                                    C.c_ulonglong(seed), _vp(w), _vp(loss)))
    return w, loss


def qol_selector_set(mode, w=None, conf=0.9, tol=None):
    """mode 1: the calls that follow take their pair levels from the selector
    (weights w rounded to BF16, softmax confidence >= conf, ball check at the
    predicted level); mode 2: the same with the two-level check at tolerance
    tol (error-judged labels); mode 0: the plain ball-test walk."""
    if tol is not None:
        _check(lib().qol_selector_set_tol(C.c_double(tol)))
    wp = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
    _check(lib().qol_selector_set(C.c_int(int(mode)), _vp(wp), C.c_double(conf)))


def qol_set_patch_refine(iadap):
    """patch refinement of the calls that follow, the reference GRF test's
    iadap: 0 square levels (default), 1 the adaptive tree walk (PR_ADAPTIVE),
    3 plain 4-split levels"""
    _check(lib().qol_set_patch_refine(C.c_int(int(iadap))))


def qol_ref_level_table(nterms, orderff, level):
    """dict(uv (n, 2), wt, suboff, subtyp) of the reference element's level
    0..3 under the current refinement mode"""
    n, ns = np.zeros(1, np.int64), np.zeros(1, np.int64)
    _check(lib().qol_ref_level_table(i64(nterms), i64(orderff), i64(level), _vp(n), _vp(ns), None, None, None, None))
    uv, wt = np.zeros(2 * n[0]), np.zeros(n[0])
    so, st = np.zeros(ns[0] + 1, np.int64), np.zeros(ns[0], np.int64)
    _check(lib().qol_ref_level_table(i64(nterms), i64(orderff), i64(level), _vp(n), _vp(ns), _vp(uv), _vp(wt),
                                     _vp(so), _vp(st)))
    return dict(uv=uv.reshape(-1, 2), wt=wt, suboff=so, subtyp=st)


def qol_selector_force_level(level):
    """1..4: the calls that follow compute every pair that the plain walk
    resolves by a direct sum on that level (RRQ pairs unchanged); 0: the walk."""
    _check(lib().qol_selector_force_level(C.c_int(int(level))))


def qol_selector_stats():
    """{accepted, low_confidence, check_failed} pair counts since the last call."""
    c = np.zeros(3, np.int64)
    _check(lib().qol_selector_stats(_vp(c)))
    return {"accepted": int(c[0]), "low_confidence": int(c[1]), "check_failed": int(c[2])}


def qol_set_autotune(on):
    """1 (default): the first call of an order with >= 256 panels measures the
    per-panel precompute kernel's shapes and keeps the fastest; 0: built-in shape."""
    _check(lib().qol_set_autotune(C.c_int(int(on))))


def qol_panel_shape(nterms, orderff, nquad):
    """(cluster size, CTA threads) kept for an order, (0, 0) before any"""
    cs, nt = C.c_int(0), C.c_int(0)
    _check(lib().qol_panel_shape(i64(nterms), i64(orderff), i64(nquad), C.byref(cs), C.byref(nt)))
    return cs.value, nt.value
