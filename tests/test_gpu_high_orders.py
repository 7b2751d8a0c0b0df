"""GPU parity above the headline orders: nterms 14 and 15 (hdim 105 and
120: the wide panel kernel, four-CTA clusters, four 32-column blocks of the
level sums), through the C ABI against the oracle on the stellarator slice of
test_gpu_headline_orders (4 x 10 quads, 300 off-surface targets), with the
same kinds of bounds: indices bit-exact, level-resolved rows TOL_LEVEL relative
to the panel's largest level-row entry, RRQ rows condition-scaled
(conftest.row_errors; measured at 0.22 and 0.20 of the bound), and the rows
contracted with a smooth density TOL_SMOOTH.  The FP32 level
sums at these orders against the FP64 form, as in test_gpu_precision.
nterms 16 (hdim 136) has no launch shape of the panel kernel and is refused
with QOL_ERR_ORDER before any work."""
import numpy as np
import pytest

from conftest import row_errors

pytestmark = pytest.mark.gpu

# level-resolved rows: rounding of the direct sums and the contraction grows with the nodes and
# columns (measured 4.8e-13 at nterms 13, 9.0e-13 at 14, 1.8e-12 at 15)
TOL_LEVEL = {14: 2e-12, 15: 4e-12}
# contracted rows: they follow kappa, about tenfold an order (measured 5.7e-12 at nterms 13,
# 4.7e-11 at 14, 2.2e-9 at 15)
TOL_SMOOTH = {14: 1e-10, 15: 5e-9}
TOL_ROWS = 1e-6  # FP32 level sums vs FP64, per target row: max |diff| / max |value| of the row


def _case(G, nterms):
    P = G.panels(G.stellarator(), 4, 10, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 300, 1, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    return P, hd, tcxi, tcxrow, tcx


def _near(qol, P, hd, nterms, tcxi, tcxrow, tcx):
    npan = P["sw"].size // hd
    nq = nterms + 2
    return qol.qol_getnearquad_lap_rrq(npan, nterms, hd, nq, npan * hd, P["sx"], P["snx"], P["sw"], P["rts"],
                                       P["rps"], tcxrow.size, tcx, tcxrow, tcxi, nq, 1.4, 30)


@pytest.mark.parametrize("nterms", [14, 15])
def test_high_order_rows(qol, orc, nterms):
    from qotential_b200 import geometry as G
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    npan = P["sw"].size // hd
    nq = nterms + 2
    si, sj, vs, vd, _ = _near(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    oi, oj, ovs, ovd, hist, lv = orc.getnearquad(npan, nterms, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                                 tcx, tcxrow, tcxi, nq, pair_levels=True)
    assert np.array_equal(si, oi) and np.array_equal(sj, oj)
    assert hist[5] > 100 and hist[1] > 100
    ys, q = G.point_charges(G.stellarator(), 8, seed=5, radius=12.0)
    ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
    worst_level, worst_ratio = row_errors(orc, P, hd, nterms, tcxi, lv, ((vs, ovs), (vd, ovd)))
    g, o = [], []
    for k in range(npan):
        lo, hi = int(tcxi[k]) - 1, int(tcxi[k + 1]) - 1
        m = hi - lo
        if m == 0:
            continue
        blk, sl = slice(lo * hd, hi * hd), slice(k * hd, (k + 1) * hd)
        f = lambda a, b: a[blk].reshape(hd, m).T @ ubn[sl] - b[blk].reshape(hd, m).T @ ub[sl]
        g.append(f(vs, vd))
        o.append(f(ovs, ovd))
    g, o = np.concatenate(g), np.concatenate(o)
    es = np.abs(g - o).max() / np.abs(o).max()
    print(f"nterms {nterms}: level rows {worst_level:.2e}, RRQ worst / bound {worst_ratio:.3f}, smooth {es:.2e}")
    assert worst_level < TOL_LEVEL[nterms], worst_level
    assert worst_ratio < 1.0, worst_ratio
    assert es < TOL_SMOOTH[nterms], es


@pytest.mark.parametrize("nterms", [14, 15])
def test_high_order_fp32_sums(qol, nterms):
    from qotential_b200 import geometry as G
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
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
        assert 0 < err < TOL_ROWS, err


def test_nterms16_refused(qol):
    from qotential_b200 import geometry as G
    nterms = 16
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    with pytest.raises(qol.QolError) as e:
        _near(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    assert e.value.code == 6 and "no launch shape" in str(e.value)
