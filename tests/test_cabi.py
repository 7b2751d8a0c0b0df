"""C-ABI boundary (CPU): the library loads, exports every declared symbol,
and validates arguments as the reference's gateway does; compute calls
without a GPU fail loudly (no CPU path)."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    h = open(os.path.join(ROOT, "include", "qol_b200.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)   # declarations only, not comments
    return sorted(set(re.findall(r"\b(qol_\w+)\s*\(", h)))


def test_exports_every_declared_symbol(qol):
    L = qol.lib()
    syms = declared_symbols()
    assert len(syms) >= 17
    for s in syms:
        assert hasattr(L, s), s


def test_header_cites_reference(qol):
    h = open(os.path.join(ROOT, "include", "qol_b200.h")).read()
    for name in ("qol_getnearquad_lap_rrq", "qol_rrq", "qol_build_patch_levels", "qol_lap3dsdlpmat_levels"):
        block = h[:h.index(f"int {name}(")]
        assert "src/" in block[-900:], name


def test_simplex_precomp_host_only(qol):
    tgl, wgl, Dgl, wb, Leg, um, vm = qol.qol_simplex_precomp(8, 5)
    assert np.allclose(um @ vm, np.eye(21), atol=1e-10)
    with pytest.raises(qol.QolError) as e:
        import ctypes as C
        z = np.zeros(100)
        rc = qol.lib().qol_simplex_precomp(C.c_longlong(8), C.c_longlong(5), C.c_longlong(20), *([C.c_void_p(z.ctypes.data)] * 7))
        qol._check(rc)
    assert e.value.code == 3


def test_getnearquad_layout_errors(qol):
    npan, nterms = 2, 3
    hd = 6
    sx = np.zeros((npan * hd, 3))
    tcx = np.zeros((3, 3))
    args = dict(npan=npan, nterms=nterms, hdim=hd, nquad=5, nsrc=npan * hd, sx=sx, snx=sx, sw=np.ones(npan * hd),
                rts=sx, rps=sx, ntcx=3, tcx=tcx, tcxrow=np.array([1, 2, 3]), orderff=5, distff=1.4, iside=30)
    with pytest.raises(qol.QolError) as e:
        qol.qol_getnearquad_lap_rrq(tcxi=np.array([1, 3, 3]), **args)   # does not cover tcx
    assert e.value.code == 1
    with pytest.raises(qol.QolError) as e:
        qol.qol_getnearquad_lap_rrq(tcxi=np.array([1, 3, 4]), nnz=5, **args)   # nnz too small
    assert e.value.code == 2
    with pytest.raises(qol.QolError) as e:
        qol.qol_getnearquad_lap_rrq(tcxi=np.array([2, 3, 4]), **args)   # not one-based
    assert e.value.code == 1
    # the C entry point itself (not only the Python mirror) rejects bad layouts
    import ctypes as C
    xi = np.array([1, 4, 3], np.int64)
    z = np.zeros(64); zi = np.zeros(64, np.int64); ti = np.zeros(20)
    p = lambda a: C.c_void_p(a.ctypes.data)
    L = C.c_longlong
    rc = qol.lib().qol_getnearquad_lap_rrq(L(2), L(3), L(6), L(5), L(12), p(z), p(z), p(z), p(z), p(z), L(3), p(z),
                                           p(zi), p(xi), L(5), C.c_double(1.4), L(30), L(0), L(18), p(zi), p(zi),
                                           p(z), p(z), p(ti))
    assert rc == 1


def test_handle_errors_without_gpu(qol):
    # bad handles are rejected before any device work
    with pytest.raises(qol.QolError) as e:
        qol.qol_clear_patch_levels(12345)
    assert e.value.code == 2


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback(qol):
    from qotential_b200 import geometry as G
    P = G.panels(G.torus(), 2, 3, 3, split=False)
    with pytest.raises(qol.QolError) as e:
        qol.qol_rrq(P["sx"][:3], P["sx"][:6], P["snx"][:6], P["sw"][:6], P["rts"][:6], P["rps"][:6], 3, 5, 5)
    assert e.value.code == 5


def test_getnearquad_out_checked(qol):
    """caller-allocated outputs: four contiguous int64/int64/float64/float64
    arrays of nnz entries, else QolError(1) before any device work"""
    npan, nterms, hd = 2, 3, 6
    sx = np.zeros((npan * hd, 3))
    args = dict(npan=npan, nterms=nterms, hdim=hd, nquad=5, nsrc=npan * hd, sx=sx, snx=sx, sw=np.ones(npan * hd),
                rts=sx, rps=sx, ntcx=3, tcx=np.zeros((3, 3)), tcxrow=np.array([1, 2, 3]), tcxi=np.array([1, 3, 4]),
                orderff=5, distff=1.4, iside=30)
    good = (np.zeros(18, np.int64), np.zeros(18, np.int64), np.zeros(18), np.zeros(18))
    for bad in ((good[0].astype(np.int32),) + good[1:], good[:2] + (np.zeros(17),) + good[3:],
                good[:3] + (np.zeros((18, 2))[:, 0],)):
        with pytest.raises(qol.QolError) as e:
            qol.qol_getnearquad_lap_rrq(out=bad, **args)
        assert e.value.code == 1


def test_selector_arguments_checked(qol):
    """selector entry points reject bad arguments before any device work"""
    w = np.zeros(qol.SELECTOR_NW, np.float32)
    for mode, conf in ((3, 0.9), (1, 1.5), (2, 0.0)):
        with pytest.raises(qol.QolError) as e:
            qol.qol_selector_set(mode, w, conf)
        assert e.value.code == 8
    qol.qol_selector_set(0)  # back to the plain walk: no device needed
    for tol in (0.0, -1e-8, 1.0):
        with pytest.raises(qol.QolError) as e:
            qol.qol_selector_set(0, tol=tol)
        assert e.value.code == 8
    for level in (-1, 5):
        with pytest.raises(qol.QolError) as e:
            qol.qol_selector_force_level(level)
        assert e.value.code == 8
    qol.qol_selector_force_level(0)
    f = np.zeros((4, 8), np.float32)
    with pytest.raises(qol.QolError) as e:
        qol.qol_selector_grad(f, np.array([0, 1, 7, 2]), w)  # class out of range
    assert e.value.code == 8
    with pytest.raises(qol.QolError) as e:
        qol.qol_selector_train(f, np.zeros(4), w, epochs=1, batch=100)  # batch not a multiple of 256
    assert e.value.code == 8


def test_patch_refine_switch_host_only(qol):
    """iadap 0, 1 and 3 only (square + adaptive is refused, as the reference's
    build_patch_ref_r64 refuses it)"""
    for bad in (2, 4, -1):
        with pytest.raises(qol.QolError) as e:
            qol.qol_set_patch_refine(bad)
        assert e.value.code == 8
    for ok in (1, 3, 0):
        qol.qol_set_patch_refine(ok)


def test_autotune_switch_host_only(qol):
    """the autotune switch accepts 0 and 1 only; an order never run has no kept shape"""
    with pytest.raises(qol.QolError) as e:
        qol.qol_set_autotune(2)
    assert e.value.code == 8
    qol.qol_set_autotune(0)
    qol.qol_set_autotune(1)
    assert qol.qol_panel_shape(15, 17, 17) == (0, 0)


def test_wrappers_keep_argument_copies_alive(qol, monkeypatch):
    """strided (non-contiguous) array arguments are copied by the wrappers; the
    pointers handed to the C ABI must stay valid through the call (a stand-in
    library records what each pointer holds during the call)"""
    import ctypes as C
    nterms, npan = 6, 4
    nsrc = npan * 21
    seen = {}

    class Rec:
        def __getattr__(self, name):
            def f(*a):
                get = lambda p: np.ctypeslib.as_array((C.c_double * nsrc).from_address(p.value)).copy()
                seen["ub"], seen["ubn"], seen["u"] = get(a[13]), get(a[14]), get(a[15])
                return 0
            return f

    monkeypatch.setattr(qol, "_lib", Rec())
    rng = np.random.default_rng(3)
    ub, ubn, u = rng.random((nsrc, 3)), rng.random((nsrc, 3)), rng.random((nsrc, 3))
    z = np.zeros((nsrc, 3))
    qol.qol_grf_near(npan, nterms, 8, z, z, np.zeros(nsrc), z, z, ub[:, 1], ubn[:, 1], u=u[:, 1])
    assert np.array_equal(seen["ub"], ub[:, 1]) and np.array_equal(seen["ubn"], ubn[:, 1])
    assert np.array_equal(seen["u"], u[:, 1])
