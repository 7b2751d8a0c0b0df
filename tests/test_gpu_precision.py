"""The precision variant of the level sums (qol_set_sum_precision(1): FP32
kernel values, 3xTF32 contraction on the tcgen05 tensor cores, compensated
accumulation across 32-node tiles) against the FP64 drop-in and the oracle:
its error on the correction rows, stated here, and the GRF identity at matched
error (the metric compares the two forms there)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_ROWS = 1e-6   # FP32-form correction values vs FP64, per target row: max |diff| / max |value| of the row
GRF_MATCH = 1.10  # FP32-form GRF error at most 10 % above the FP64 form's


def _near(qol, P, hd, nterms, tcxi, tcxrow, tcx):
    npan = P["sw"].size // hd
    nq = nterms + 2
    return qol.qol_getnearquad_lap_rrq(npan, nterms, hd, nq, npan * hd, P["sx"], P["snx"], P["sw"], P["rts"],
                                       P["rps"], tcxrow.size, tcx, tcxrow, tcxi, nq, 1.4, 30)


@pytest.mark.parametrize("nterms", [5, 9])
def test_fp32_sums_rows_vs_fp64(qol, nterms):
    from qotential_b200 import geometry as G
    P = G.panels(G.stellarator(), 4, 10, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 300, 1, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    a = _near(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    qol.qol_set_sum_precision(1)
    try:
        b = _near(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    finally:
        qol.qol_set_sum_precision(0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    rows = a[0] - a[0].min()
    for x, y in ((a[2], b[2]), (a[3], b[3])):
        d = np.zeros(rows.max() + 1)
        v = np.zeros(rows.max() + 1)
        np.maximum.at(d, rows, np.abs(x - y))
        np.maximum.at(v, rows, np.abs(x))
        err = (d[v > 0] / v[v > 0]).max()
        assert 0 < err < TOL_ROWS, err  # > 0: the FP32 path did run


def _pair_of_entry(tcxi, hd):
    """COO entry -> pair (the entries of a panel: column-major over its m targets)"""
    xi = np.asarray(tcxi, np.int64)
    m = np.diff(xi)
    pan = np.repeat(np.arange(m.size), hd * m)
    local = np.arange(pan.size) - (xi[:-1] - 1)[pan] * hd
    return (xi[:-1] - 1)[pan] + local % m[pan]


@pytest.mark.parametrize("nterms", [5, 9])
def test_fp32_sums_vs_oracle(qol, orc, nterms):
    """the FP32 form against the oracle's FP64 values: level-resolved entries
    within TOL_ROWS per target row (relative to the row's largest entry, as in
    test_fp32_sums_rows_vs_fp64); RRQ entries, FP64 in both forms,
    bit-identical to the plain form's"""
    from qotential_b200 import geometry as G
    P = G.panels(G.stellarator(), 4, 10, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 300, 2, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    npan = P["sw"].size // hd
    nq = nterms + 2
    a = _near(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    qol.qol_set_sum_precision(1)
    try:
        b = _near(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    finally:
        qol.qol_set_sum_precision(0)
    oi, oj, ovs, ovd, hist, lv = orc.getnearquad(npan, nterms, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                                 tcx, tcxrow, tcxi, nq, pair_levels=True)
    assert np.array_equal(b[0], oi) and np.array_equal(b[1], oj)
    lev = np.asarray(lv)[_pair_of_entry(tcxi, hd)]
    rrq, direct = lev == 5, lev <= 4
    assert rrq.any() and direct.any()
    assert np.array_equal(b[2][rrq], a[2][rrq]) and np.array_equal(b[3][rrq], a[3][rrq])
    rows = b[0] - b[0].min()
    for x, y in ((b[2], ovs), (b[3], ovd)):
        d = np.zeros(rows.max() + 1)
        v = np.zeros(rows.max() + 1)
        np.maximum.at(d, rows[direct], np.abs(x - y)[direct])
        np.maximum.at(v, rows, np.abs(y))
        err = (d[v > 0] / v[v > 0]).max()
        assert 0 < err < TOL_ROWS, err


def test_fp32_sums_grf_matched(qol):
    from qotential_b200 import geometry as G
    for nterms in (4, 6, 8):
        surf = G.torus()
        P = G.panels(surf, 12, 24, nterms, split=False)
        ys, q = G.point_charges(surf, 4, seed=7)
        ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
        hd = nterms * (nterms + 1) // 2
        npan = P["sw"].size // hd
        u = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
        errs = []
        for mode in (0, 1):
            qol.qol_set_sum_precision(mode)
            try:
                un, _, _ = qol.qol_grf_near(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"],
                                            P["rps"], ub, ubn, u=u)
            finally:
                qol.qol_set_sum_precision(0)
            errs.append(np.abs(un).max() / np.abs(ubn).max())
        assert errs[1] <= GRF_MATCH * errs[0], (nterms, errs)


def test_sum_precision_rejects_unknown_mode(qol):
    with pytest.raises(qol.QolError) as e:
        qol.qol_set_sum_precision(2)
    assert e.value.code == 8
