"""Edge cases of qol_getnearquad_lap_rrq on the GPU against the oracle: no near
targets at all, ragged near lists (panels with all, none or one of their
targets), a single panel with a single target."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_LOW = 1e-12  # as the parity tests at nterms <= 6: whole matrix relative to its largest entry


def _case(G, nterms=5):
    P = G.panels(G.torus(), 6, 12, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 60, 2, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    return P, hd, tcxi, tcxrow, tcx


def _run(qol, P, hd, nterms, npan, tcxi, tcxrow, tcx):
    nq = nterms + 2
    return qol.qol_getnearquad_lap_rrq(npan, nterms, hd, nq, npan * hd, P["sx"][:npan * hd], P["snx"][:npan * hd],
                                       P["sw"][:npan * hd], P["rts"][:npan * hd], P["rps"][:npan * hd], tcxrow.size,
                                       tcx, tcxrow, tcxi, nq, 1.4, 30)


def _compare(orc, P, hd, nterms, npan, tcxi, tcxrow, tcx, got):
    nq = nterms + 2
    oi, oj, ovs, ovd, hist = orc.getnearquad(npan, nterms, nq, P["sx"][:npan * hd], P["snx"][:npan * hd],
                                             P["sw"][:npan * hd], P["rts"][:npan * hd], P["rps"][:npan * hd], tcx,
                                             tcxrow, tcxi, nq)
    assert np.array_equal(got[0], oi) and np.array_equal(got[1], oj)
    for a, b in ((got[2], ovs), (got[3], ovd)):
        if b.size:
            assert np.abs(a - b).max() <= TOL_LOW * np.abs(b).max()
    return hist


def test_no_near_targets(qol):
    from qotential_b200 import geometry as G
    nterms = 5
    P, hd, _, _, _ = _case(G, nterms)
    npan = P["sw"].size // hd
    tcxi = np.ones(npan + 1, np.int64)
    r = _run(qol, P, hd, nterms, npan, tcxi, np.zeros(0, np.int64), np.zeros((0, 3)))
    assert all(np.asarray(x).size == 0 for x in r[:4])


def test_ragged_near_lists(qol, orc):
    from qotential_b200 import geometry as G
    nterms = 5
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    npan = P["sw"].size // hd
    keep, xi = [], [1]
    for k in range(npan):
        a, b = tcxi[k] - 1, tcxi[k + 1] - 1
        sel = range(a, b) if k % 3 == 0 else (range(0) if k % 3 == 1 else range(a, min(a + 1, b)))
        keep.extend(sel)
        xi.append(xi[-1] + len(sel))
    keep = np.asarray(keep, np.int64)
    ntcxi, nrow, ntcx = np.asarray(xi, np.int64), tcxrow[keep], tcx[keep]
    got = _run(qol, P, hd, nterms, npan, ntcxi, nrow, ntcx)
    hist = _compare(orc, P, hd, nterms, npan, ntcxi, nrow, ntcx, got)
    assert hist[5] > 0 and hist[1:5].sum() > 0  # both methods occur


def test_single_panel_single_target(qol, orc):
    from qotential_b200 import geometry as G
    nterms = 6
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    k = 7
    a = tcxi[k] - 1
    # the panel's own first node as the target (self pair: RRQ and the masked naive entry)
    sel = [i for i in range(a, tcxi[k + 1] - 1) if tcxrow[i] == k * hd + 1][:1]
    assert sel
    Pk = {key: P[key][k * hd:(k + 1) * hd] for key in ("sx", "snx", "sw", "rts", "rps")}
    row = np.array([1], np.int64)  # the panel's first node, renumbered
    got = _run(qol, Pk, hd, nterms, 1, np.array([1, 2], np.int64), row, tcx[sel])
    _compare(orc, Pk, hd, nterms, 1, np.array([1, 2], np.int64), row, tcx[sel], got)
