"""GPU GRF near phase (qol_grf_near) and Direct far field (qol_direct_farfield)
against the oracle's restatement of the reference's stellarator driver
(web/stellarator/fortran/stellarator_grf_core_mod.f90:566-606, 652-899), and
the Green's-representation identity computed on the GPU alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_U = 1e-10   # near-phase sums of ~10 RRQ/level rows per node, relative to max |u|
TOL_FAR = 1e-12  # all-pairs sums (rsqrt vs sqrt and division), relative to max |u|


def _surface(G, surf, mp, np_, nterms, seed=7):
    P = G.panels(surf, mp, np_, nterms, split=False)
    ys, q = G.point_charges(surf, 4, seed=seed)
    ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
    return P, ub, ubn


@pytest.mark.parametrize("which,nterms", [("torus", 4), ("stellarator", 6)])
def test_grf_near_matches_oracle(qol, orc, which, nterms):
    from qotential_b200 import geometry as G
    surf = G.torus() if which == "torus" else G.stellarator()
    mp, np_ = (6, 12) if which == "torus" else (4, 10)
    P, ub, ubn = _surface(G, surf, mp, np_, nterms)
    hd = nterms * (nterms + 1) // 2
    npan = P["sw"].size // hd
    nq = nterms + 2
    u0 = np.linspace(-1.0, 1.0, P["sw"].size)  # the near phase adds into u
    ug, nn, hist = qol.qol_grf_near(npan, nterms, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub, ubn,
                                    u=u0)
    offs, idx = orc.ballcsr(npan, hd, P["sx"], P["sw"])
    uo, _, histo = orc.grf_near(npan, nterms, nq, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub, ubn,
                                offs, idx, u0)
    assert nn == int(offs[-1])
    assert np.array_equal(hist, histo) and hist[5] > 0
    err = np.abs(ug - uo).max() / np.abs(uo).max()
    assert err < TOL_U, err


def test_direct_farfield_matches_oracle(qol, orc):
    from qotential_b200 import geometry as G
    P, ub, ubn = _surface(G, G.stellarator(), 4, 10, 5)
    ug = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    uo = orc.direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    err = np.abs(ug - uo).max() / np.abs(uo).max()
    assert err < TOL_FAR, err


def test_grf_identity_gpu_only(qol):
    """S[du/dn] - D[u] = 0 (exterior limit) on the torus for a harmonic u from
    exterior point charges, far field and near phase both on the GPU; the error
    per order falls as for the oracle (4.1e-4, 9.0e-6, 8.8e-7 at nterms 4/6/8)"""
    from qotential_b200 import geometry as G
    errs = []
    for nterms in (4, 6, 8):
        P, ub, ubn = _surface(G, G.torus(), 12, 24, nterms)
        hd = nterms * (nterms + 1) // 2
        npan = P["sw"].size // hd
        u = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
        un, _, _ = qol.qol_grf_near(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub,
                                    ubn, u=u)
        errs.append(np.abs(un).max() / np.abs(ubn).max())
    assert errs[0] < 1e-3 and errs[1] < 2e-5 and errs[2] < 2e-6, errs


def test_ranges_add_up_to_the_whole(qol):
    """The multi-GPU split on one GPU: qol_grf_near_range over a partition of
    the panels and qol_direct_farfield_range over a partition of the targets
    add up to the single calls (to rounding: only the order in which a node's
    corrections are added differs), and getnearquad shards with renumbered
    rows concatenate to the single call's output byte for byte."""
    from qotential_b200 import geometry as G
    from qotential_b200 import sharding as S
    nterms = 6
    P, ub, ubn = _surface(G, G.stellarator(), 4, 10, nterms)
    hd = nterms * (nterms + 1) // 2
    npan = P["sw"].size // hd
    nsrc = npan * hd
    nq = nterms + 2
    full_far = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    full, nn, hist = qol.qol_grf_near(npan, nterms, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub, ubn,
                                      u=full_far)
    tcxi, _, tcx = G.near_lists(P["sx"], P["sw"], hd)
    ranges = S.balanced_ranges(S.panel_costs(tcxi, tcx, P["sx"], P["sw"], hd), 3)
    total = np.zeros(nsrc)
    for r, (a, b) in enumerate(ranges):
        part = np.zeros(nsrc)
        qol.qol_direct_farfield_range(P["sx"], P["snx"], P["sw"], ub, ubn, (r * nsrc) // 3, ((r + 1) * nsrc) // 3,
                                      part)
        part = qol.qol_grf_near_range(npan, nterms, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub, ubn, a, b,
                                      u=part)
        total += part
    assert np.abs(total - full).max() <= 1e-13 * np.abs(full).max()
    # getnearquad: per-rank shards
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 200, 4, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    one = qol.qol_getnearquad_lap_rrq(npan, nterms, hd, nq, nsrc, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                      tcxrow.size, tcx, tcxrow, tcxi, nq, 1.4, 30)
    parts = [S.getnearquad_shard(r, 2, npan, nterms, hd, nq, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                 tcxrow, tcxi, nq) for r in range(2)]
    for k in range(4):
        assert np.concatenate([p[k] for p in parts]).tobytes() == one[k].tobytes()


def test_multi_density_matches_single_calls(qol):
    """qol_grf_near_multi with 4 point-charge densities (BASELINE config 3's 4
    right-hand sides): each column equals its own qol_grf_near call byte for
    byte (the same corrections, applied once a density)"""
    from qotential_b200 import geometry as G
    nterms = 6
    surf = G.stellarator()
    P = G.panels(surf, 4, 12, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    npan = P["sw"].size // hd
    ubs, ubns = [], []
    for seed in range(4):
        ys, q = G.point_charges(surf, 8, seed=seed)
        ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
        ubs.append(ub); ubns.append(ubn)
    ub, ubn = np.stack(ubs, 1), np.stack(ubns, 1)
    u0 = np.random.default_rng(1).random(ub.shape)
    um, nn, hist = qol.qol_grf_near_multi(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub,
                                          ubn, u=u0)
    for r in range(4):
        us, ns, hs = qol.qol_grf_near(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                      ub[:, r], ubn[:, r], u=u0[:, r])
        assert ns == nn and np.array_equal(hs, hist)
        assert np.ascontiguousarray(um[:, r]).tobytes() == us.tobytes()


def test_grf_error_converges_with_order(qol):
    """the GRF identity on the stellarator (16 x 80 quads) with charges the
    panels resolve (8 on |y| = 12), nquad = nterms + 6 (the edge quadrature
    that resolves the moment integrands at high order): the error falls at
    every order through nterms 11, and at nterms 13 stays within the rounding
    floor that the systems' conditioning sets (kappa u ~ 6e-6 of a panel's near
    correction; measured 1.2e-6 against 4.0e-7 at nterms 11)"""
    from qotential_b200 import geometry as G
    surf = G.stellarator()
    ys, q = G.point_charges(surf, 8, seed=5, radius=12.0)
    errs = {}
    for nterms in (5, 7, 9, 11, 13):
        P = G.panels(surf, 16, 80, nterms, split=False)
        hd = nterms * (nterms + 1) // 2
        npan = P["sw"].size // hd
        ub, ubn = G.harmonic_density(P["sx"], P["snx"], ys, q)
        u = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
        un, _, _ = qol.qol_grf_near(npan, nterms, nterms + 6, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub, ubn,
                                    u=u)
        errs[nterms] = float(np.abs(un).max() / np.abs(ubn).max())
    print("GRF error by nterms:", errs)
    for a, b in ((5, 7), (7, 9), (9, 11)):
        assert errs[b] < errs[a], errs
    assert errs[11] < 1e-6 and errs[13] < 5e-6, errs
