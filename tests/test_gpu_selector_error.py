"""The error-judged selector (mode 2) on the GPU, no reference counterpart.

Labelling runs (qol_selector_force_level) put every direct pair on one level:
where that is the plain walk's own level they reproduce its values bit for
bit.  A selector trained on error-judged labels (the lowest level whose row
is within TOL of the finest level's) and guarded by the two-level check must
gain over the walk -- less direct-sum work, counted in level nodes -- while
keeping the COO indices, every direct row within the walk's own error scale
of the finest level's, and the GRF error of the plain form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-6          # label and check tolerance (row 1-norm; single layer over the panel diameter): at
                    # nterms 7-9 the walk's own direct rows reach 1e-5 of the finest level's, p99.9 2e-6
WORK_GAIN = 0.85    # direct-sum work (level nodes x pairs) of the selector over the walk's, at most
ERR_SCALE = 2.0     # selector's worst direct-row error over max(walk's worst, 3 TOL), at most
GRF_MATCH = 2.0     # GRF error of the selector form over the plain form's, at most


def _case(G, nterms, mp=6, np_=24, off=1500, seed=4):
    P = G.panels(G.stellarator(), mp, np_, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, off, seed, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    return P, hd, tcxi, tcxrow, tcx


def _pair_index(tcxi, hd):
    xi = np.asarray(tcxi, np.int64)
    m = np.diff(xi)
    pan = np.repeat(np.arange(m.size), hd * m)
    local = np.arange(pan.size) - (xi[:-1] - 1)[pan] * hd
    return pan, (xi[:-1] - 1)[pan] + local % m[pan]


def _pair_err(P, hd, tcxi, a, b):
    """per pair: max(1-norm single-layer difference / sqrt(panel area), 1-norm double-layer difference)"""
    pan, pair = _pair_index(tcxi, hd)
    n = int(tcxi[-1] - 1)
    diam = np.sqrt(np.asarray(P["sw"]).reshape(-1, hd).sum(1))[pan]
    es = np.bincount(pair, np.abs(a[2] - b[2]) / diam, minlength=n)
    ed = np.bincount(pair, np.abs(a[3] - b[3]), minlength=n)
    return np.maximum(es, ed)


class _Runner:
    def __init__(self, qol, P, hd, nterms, tcxi, tcxrow, tcx):
        import torch
        self.qol, self.torch, self.nterms = qol, torch, nterms
        dev = torch.device("cuda", torch.cuda.current_device())
        t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
        self.D = {k: t(P[k]) for k in ("sx", "snx", "sw", "rts", "rps")}
        self.q = (t(tcx), t(tcxrow, torch.int64), t(tcxi, torch.int64))
        self.npan = P["sw"].size // hd
        nnz = tcxrow.size * hd
        self.out = (torch.empty(nnz, dtype=torch.int64, device=dev), torch.empty(nnz, dtype=torch.int64, device=dev),
                    torch.empty(nnz, dtype=torch.float64, device=dev), torch.empty(nnz, dtype=torch.float64, device=dev))

    def __call__(self):
        nq = self.nterms + 2
        D = self.D
        h = self.qol.qol_getnearquad_lap_rrq_dev(self.npan, self.nterms, nq, D["sx"], D["snx"], D["sw"], D["rts"],
                                                 D["rps"], *self.q, nq, 1.4, 30, self.out, want_hist=True)
        return [o.cpu().numpy() for o in self.out], h


def test_forced_levels_reproduce_the_walk(qol):
    from qotential_b200 import geometry as G
    nterms = 7
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms, 4, 12, 400)
    npan = P["sw"].size // hd
    _, lev = qol.qol_selector_features(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                       tcxrow, tcxi, nterms + 2)
    run = _Runner(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    plain, hist = run()
    _, pair = _pair_index(tcxi, hd)
    lev_e = lev[pair]
    try:
        for L in (1, 2, 3, 4):
            qol.qol_selector_force_level(L)
            forced, fh = run()
            assert np.array_equal(forced[0], plain[0]) and np.array_equal(forced[1], plain[1])
            keep = (lev_e == L) | (lev_e == 5)
            assert np.array_equal(forced[2][keep], plain[2][keep]) and np.array_equal(forced[3][keep], plain[3][keep])
            assert fh[L] == hist[1:5].sum() and fh[5] == hist[5]
    finally:
        qol.qol_selector_force_level(0)


@pytest.fixture(scope="module")
def trained(qol):
    from qotential_b200 import selector as Sel
    feat, lab, _ = Sel.training_set(150000, seed=3, orders=(6, 8), noff=3000, max_grid=(8, 24), labels="error",
                                    tol=TOL)
    w, loss = qol.qol_selector_train(feat, lab, epochs=15, batch=4096, lr=3e-3, seed=9)
    assert loss[-1] < 0.5 * loss[0]
    return w


def test_error_judged_selector_gains_over_the_walk(qol, orc, trained):
    from qotential_b200 import geometry as G
    nterms = 9
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    npan = P["sw"].size // hd
    _, lev = qol.qol_selector_features(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                       tcxrow, tcxi, nterms + 2)
    nodes = np.array([L["n"] for L in orc.ref_levels(nterms - 1, nterms + 2, 4)])
    run = _Runner(qol, P, hd, nterms, tcxi, tcxrow, tcx)
    plain, hw = run()
    qol.qol_selector_force_level(4)
    try:
        fine, _ = run()
    finally:
        qol.qol_selector_force_level(0)
    qol.qol_selector_stats()
    qol.qol_selector_set(2, trained, 0.5, tol=TOL)
    try:
        sel, hs = run()
        st = qol.qol_selector_stats()
    finally:
        qol.qol_selector_set(0)
    assert np.array_equal(sel[0], plain[0]) and np.array_equal(sel[1], plain[1])  # the same CSR sparsity
    work_walk, work_sel = float(nodes @ hw[1:5]), float(nodes @ hs[1:5])
    direct = lev <= 4
    e_walk = _pair_err(P, hd, tcxi, plain, fine)[direct]
    e_sel = _pair_err(P, hd, tcxi, sel, fine)[direct]
    e_rrq = _pair_err(P, hd, tcxi, sel, plain)[~direct]
    print(f"work ratio {work_sel / work_walk:.3f}, decisions {st}, hist walk {hw[1:]}, selector {hs[1:]}, "
          f"worst direct-row error walk {e_walk.max():.2e} selector {e_sel.max():.2e}, RRQ rows {e_rrq.max():.2e}")
    assert st["accepted"] > 0.5 * tcxrow.size
    assert work_sel <= WORK_GAIN * work_walk
    assert e_sel.max() <= ERR_SCALE * max(e_walk.max(), 3 * TOL)
    assert e_rrq.max() == 0.0  # the walk's RRQ pairs stay RRQ


def test_error_judged_selector_grf_matched(qol, trained):
    """the GRF identity on the torus with the near phase in the selector form:
    its error within GRF_MATCH of the plain form's"""
    from qotential_b200 import geometry as G
    nterms = 7
    surf = G.torus()
    P = G.panels(surf, 12, 24, nterms, split=False)
    ys, q = G.point_charges(surf, 4, seed=7)
    ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
    hd = nterms * (nterms + 1) // 2
    npan = P["sw"].size // hd
    u = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    errs = []
    for mode in (0, 2):
        qol.qol_selector_set(mode, trained, 0.5, tol=TOL)
        try:
            un, _, _ = qol.qol_grf_near(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub,
                                        ubn, u=u)
        finally:
            qol.qol_selector_set(0)
        errs.append(np.abs(un).max() / np.abs(ubn).max())
    print("GRF error plain, selector:", errs)
    assert errs[1] <= GRF_MATCH * errs[0], errs
