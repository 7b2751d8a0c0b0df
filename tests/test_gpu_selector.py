"""Learned level selector on the GPU (no reference counterpart): features and
the training gradient against the oracle's numpy restatement (FP32 vs FP64),
deterministic training that learns the plain walk's levels, and the learned
form of qol_getnearquad_lap_rrq against the plain one (a prediction is used
only after the ball check at its level, so no pair gets a level the plain walk
would reject, and RRQ only where the walk gives it)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FEAT = 2e-5   # FP32 features vs FP64 (logs and tanh of O(1) arguments)
TOL_GRAD = 2e-4   # FP32 sums vs FP64 with the same BF16 operands, relative to max |g|
TOL_LEARNED = 2e-4  # learned vs plain rows: another accurate level differs by its quadrature error (nterms 6, where the GRF error is ~1e-4)
GRF_MATCH = 1.05    # learned-form GRF error at most 5 % above the plain form's


def _case(G, nterms=6, off=300):
    P = G.panels(G.stellarator(), 4, 10, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, off, 3, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    return P, hd, tcxi, tcxrow, tcx


def test_selector_features_match_oracle(qol, orc):
    from oracle import selector as S
    from qotential_b200 import geometry as G
    nterms = 6
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    npan = P["sw"].size // hd
    f, lev = qol.qol_selector_features(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                       tcxrow, tcxi, nterms + 2)
    fo = S.pair_features(npan, hd, P["sx"], P["snx"], P["sw"], tcx, tcxi)
    keep = fo[:, 4] > -8.0  # f4 = log10 |normal offset|: compare away from the 1e-12 clamp
    for c in range(8):
        rows = keep if c == 4 else slice(None)
        err = np.abs(f[rows, c] - fo[rows, c]).max()
        assert err < TOL_FEAT * (1.0 + np.abs(fo[rows, c]).max()), (c, err)
    # the labels are the plain walk's levels: their histogram is the oracle's
    _, _, _, _, hist = orc.getnearquad(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                       tcxrow, tcxi, nterms + 2)
    assert np.array_equal(np.bincount(lev, minlength=6)[1:6], hist[1:6])


def test_selector_gradient_matches_oracle(qol):
    from oracle import selector as S
    rng = np.random.default_rng(2)
    x = rng.normal(0.0, 1.0, (3000, 8)).astype(np.float32)
    y = rng.integers(0, 5, 3000).astype(np.int8)
    w = qol.qol_selector_init(4)
    loss, g = qol.qol_selector_grad(x, y, w)
    lo, go = S.loss_grad(w, x, y, bf=True)  # BF16 operands as the kernels
    assert abs(loss - lo) < 1e-5 * (1.0 + abs(lo))
    assert np.abs(g - go).max() < TOL_GRAD * np.abs(go).max()


def test_selector_trains_deterministically(qol):
    from qotential_b200 import selector as Sel
    feat, lab, _ = Sel.training_set(60000, seed=3, orders=(4, 6), noff=2000, max_grid=(6, 16))
    w1, loss1 = qol.qol_selector_train(feat, lab, epochs=12, batch=4096, lr=3e-3, seed=9)
    w2, loss2 = qol.qol_selector_train(feat, lab, epochs=12, batch=4096, lr=3e-3, seed=9)
    assert np.array_equal(w1, w2) and np.array_equal(loss1, loss2)
    assert loss1[-1] < 0.5 * loss1[0]
    cls, _ = Sel.predict(w1, feat)
    acc, majority = (cls == lab).mean(), np.bincount(lab).max() / lab.size
    assert acc > max(0.8, majority + 0.1), (acc, majority)


def test_learned_form_matches_plain(qol):
    from qotential_b200 import geometry as G
    from qotential_b200 import selector as Sel
    feat, lab, _ = Sel.training_set(60000, seed=3, orders=(4, 6), noff=2000, max_grid=(6, 16))
    w, _ = qol.qol_selector_train(feat, lab, epochs=12, batch=4096, lr=3e-3, seed=9)
    nterms = 6
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    npan = P["sw"].size // hd
    args = (npan, nterms, hd, nterms + 2, npan * hd, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcxrow.size, tcx,
            tcxrow, tcxi, nterms + 2, 1.4, 30)
    a = qol.qol_getnearquad_lap_rrq(*args)
    qol.qol_selector_stats()
    qol.qol_selector_set(1, w, 0.9)
    try:
        b = qol.qol_getnearquad_lap_rrq(*args)
        st = qol.qol_selector_stats()
    finally:
        qol.qol_selector_set(0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert st["accepted"] + st["low_confidence"] + st["check_failed"] == tcxrow.size
    assert st["accepted"] > 0.5 * tcxrow.size
    rows = a[0] - a[0].min()
    for x, y in ((a[2], b[2]), (a[3], b[3])):
        d = np.zeros(rows.max() + 1)
        v = np.zeros(rows.max() + 1)
        np.maximum.at(d, rows, np.abs(x - y))
        np.maximum.at(v, rows, np.abs(x))
        assert (d[v > 0] / v[v > 0]).max() < TOL_LEARNED


def test_learned_form_grf_matched(qol):
    """the GRF identity S[du/dn] - D[u] = 0 on the torus with the near phase in
    the learned form: its error matches the plain form's"""
    from qotential_b200 import geometry as G
    from qotential_b200 import selector as Sel
    feat, lab, _ = Sel.training_set(60000, seed=3, orders=(4, 6), noff=2000, max_grid=(6, 16))
    w, _ = qol.qol_selector_train(feat, lab, epochs=12, batch=4096, lr=3e-3, seed=9)
    nterms = 6
    surf = G.torus()
    P = G.panels(surf, 12, 24, nterms, split=False)
    ys, q = G.point_charges(surf, 4, seed=7)
    ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
    hd = nterms * (nterms + 1) // 2
    npan = P["sw"].size // hd
    u = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    errs = []
    for mode in (0, 1):
        qol.qol_selector_set(mode, w, 0.9)
        try:
            un, _, _ = qol.qol_grf_near(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub,
                                        ubn, u=u)
        finally:
            qol.qol_selector_set(0)
        errs.append(np.abs(un).max() / np.abs(ubn).max())
    assert errs[1] <= GRF_MATCH * errs[0], errs
