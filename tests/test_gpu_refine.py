"""The reference's other patch refinements on the GPU against the oracle:
iadap 1, the adaptive tree walk (PR_ADAPTIVE: plain 4-split levels, a cut of
sub-patches per target, patch_refine_mod.f90:617-771) and iadap 3, plain
4-split levels with the level walk (PR_SQUARE off) -- the switches of the
reference's GRF test (test/stellarator_grf.f90:46-47).  Same bounds as the
default levels: indices and the pair classes bit-exact, level and cut rows
TOL_LEVEL relative to the panel's largest level-row entry, RRQ rows within
the condition-scaled bound."""
import numpy as np
import pytest

from conftest import row_errors

pytestmark = pytest.mark.gpu

TOL_LEVEL = 1e-12


def _case(G, nterms, off=300):
    P = G.panels(G.stellarator(), 4, 10, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, off, 1, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    return P, hd, tcxi, tcxrow, tcx


@pytest.mark.parametrize("iadap,nterms", [(1, 5), (1, 9), (1, 13), (3, 5), (3, 13)])
def test_refinement_modes_match_oracle(qol, orc, iadap, nterms):
    import torch
    from qotential_b200 import geometry as G
    P, hd, tcxi, tcxrow, tcx = _case(G, nterms)
    npan = P["sw"].size // hd
    nq = nterms + 2
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
    D = {k: t(P[k]) for k in ("sx", "snx", "sw", "rts", "rps")}
    nnz = tcxrow.size * hd
    out = (torch.empty(nnz, dtype=torch.int64, device=dev), torch.empty(nnz, dtype=torch.int64, device=dev),
           torch.empty(nnz, dtype=torch.float64, device=dev), torch.empty(nnz, dtype=torch.float64, device=dev))
    qol.qol_set_patch_refine(iadap)
    orc.set_refine(iadap)
    try:
        hist = qol.qol_getnearquad_lap_rrq_dev(npan, nterms, nq, D["sx"], D["snx"], D["sw"], D["rts"], D["rps"],
                                               t(tcx), t(tcxrow, torch.int64), t(tcxi, torch.int64), nq, 1.4, 30, out,
                                               want_hist=True)
        oi, oj, ovs, ovd, ohist, lv = orc.getnearquad(npan, nterms, nq, P["sx"], P["snx"], P["sw"], P["rts"],
                                                      P["rps"], tcx, tcxrow, tcxi, nq, pair_levels=True)
    finally:
        qol.qol_set_patch_refine(0)
        orc.set_refine(0)
    si, sj, vs, vd = [o.cpu().numpy() for o in out]
    assert np.array_equal(si, oi) and np.array_equal(sj, oj)
    assert np.array_equal(np.asarray(hist), np.asarray(ohist)), (hist, ohist)
    if iadap == 1:
        assert hist[0] > 100 and hist[1:4].sum() == 0  # every direct pair below the finest level is a cut
    else:
        assert hist[0] == 0 and hist[1] > 100
    worst_level, worst_ratio = row_errors(orc, P, hd, nterms, tcxi, lv, ((vs, ovs), (vd, ovd)))
    assert worst_level < TOL_LEVEL, worst_level
    assert worst_ratio < 1.0, worst_ratio


def test_adaptive_grf_matches_plain_levels(qol):
    """the GRF identity on the torus with each refinement: the adaptive walk and
    the plain levels resolve the same pairs by quadratures of the same
    accuracy, so their GRF errors agree"""
    from qotential_b200 import geometry as G
    nterms = 7
    surf = G.torus()
    P = G.panels(surf, 12, 24, nterms, split=False)
    ys, q = G.point_charges(surf, 4, seed=7)
    ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
    hd = nterms * (nterms + 1) // 2
    npan = P["sw"].size // hd
    u = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    errs = {}
    try:
        for iadap in (0, 1, 3):
            qol.qol_set_patch_refine(iadap)
            un, nn, hist = qol.qol_grf_near(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                            ub, ubn, u=u)
            errs[iadap] = np.abs(un).max() / np.abs(ubn).max()
    finally:
        qol.qol_set_patch_refine(0)
    print("GRF error by iadap:", errs)
    assert errs[1] <= 1.5 * errs[3] and errs[3] <= 1.5 * errs[1]
    assert errs[1] <= 2.0 * errs[0]
