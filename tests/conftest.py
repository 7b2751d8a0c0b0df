import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this container")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "liborc.so")):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def qol():
    import qotential_b200 as q
    from qotential_b200 import _build
    _build.build()
    return q


def grf_apply(u, si, sj, vs, vd, ub, ubn):
    """u[i] += sum over COO entries (S - S_naive) ubn_j - (D - D_naive) ub_j,
    accumulated in COO order."""
    u = u.copy()
    np.add.at(u, si - 1, vs * ubn[sj - 1] - vd * ub[sj - 1])
    return u


def fixture_case(orc, order):
    """Inputs of the reference's frozen native fixtures
    (web/stellarator/fixtures/native/order{4,6}-direct.bin): the built-in
    surface on mp 12 x np 36, nterms = order, density u = exp(x/2) cos(y/2)
    (stellarator_grf_core_mod.f90:1089-1103), and the chart boundary of every
    triangle (ichart = 1: the surface map at the edge Gauss nodes and the
    vertices)."""
    from qotential_b200 import geometry as G
    P = G.panels(G.BuiltinSurface(), 12, 36, order)
    hd = order * (order + 1) // 2
    nq = order + 2
    x = P["sx"]
    ub = np.exp(0.5 * x[:, 0]) * np.cos(0.5 * x[:, 1])
    gr = np.stack([0.5 * ub, -0.5 * np.exp(0.5 * x[:, 0]) * np.sin(0.5 * x[:, 1]), 0 * ub], 1)
    ubn = (P["snx"] * gr).sum(1)
    tgl, _, _ = orc.gauss(nq)
    uv = []
    th1, th2 = 2 * np.pi / 3, 4 * np.pi / 3
    for k in range(3):
        for i in range(nq):
            tt = k * th1 + 0.5 * (1 + tgl[i]) * th1
            if tt < th1:
                uv.append((0.0, 1 - tt / th1))
            elif tt < th2:
                uv.append(((tt - th1) / th1, 0.0))
            else:
                uv.append((1 - (tt - th2) / th1, (tt - th2) / th1))
    uv += [(0, 0), (1, 0), (0, 1)]
    xbuf = G.panel_uv2x(G.BuiltinSurface(), 12, 36, order, np.array(uv))
    return dict(P=P, hd=hd, nq=nq, npan=int(P["ntri"]), ub=ub, ubn=ubn, xbuf=xbuf)


U64 = 2.0 ** -53
C_KAPPA = 8.0       # RRQ rows: |gpu - oracle| <= (C_KAPPA kappa u + FLOOR_RRQ) max |panel's RRQ rows|
FLOOR_RRQ = 3e-11   # rounding outside the D system (moment sums), dominant where kappa < 1e4


def row_errors(orc, P, hd, nterms, tcxi, levels, pairs, kappa_cache=None):
    """Per (target, panel) row of COO values in the reference's block order
    (lap3d_close_mod.f90:948-956), GPU against oracle.  ``levels`` is each
    pair's resolving level from the oracle (5 = RRQ); ``pairs`` lists
    (gpu values, oracle values) arrays, S and D.  Returns (largest error of the
    level-resolved rows relative to the panel's largest level-row entry,
    largest ratio of an RRQ error to its bound).  Errors are taken relative to
    the panel's largest entry of the same kind because rounding sits on the
    scale of the panel's weights: a small row (a far target, or entries that
    cancel in the interpolation contraction) carries the same absolute error.
    The RRQ bound is C_KAPPA kappa u + FLOOR_RRQ with kappa the 2-norm
    condition number of the panel's D system, the amplification any FP64
    evaluation of these rows carries (tests/test_oracle.py::
    test_rrq_rows_move_by_kappa_u)."""
    npan = len(tcxi) - 1
    worst_level, worst_ratio = 0.0, 0.0
    for k in range(npan):
        lo, hi = int(tcxi[k]) - 1, int(tcxi[k + 1]) - 1
        m = hi - lo
        if m == 0:
            continue
        blk = slice(lo * hd, hi * hd)
        rows = [(g[blk].reshape(hd, m).T, o[blk].reshape(hd, m).T) for g, o in pairs]
        rrq = np.asarray(levels[lo:hi]) == 5
        if (~rrq).any():
            for g, o in rows:
                e = np.abs(g[~rrq] - o[~rrq]).max() / max(np.abs(o[~rrq]).max(), 1e-300)
                worst_level = max(worst_level, float(e))
        if rrq.any():
            if kappa_cache is not None and k in kappa_cache:
                kap = kappa_cache[k]
            else:
                sl = slice(k * hd, (k + 1) * hd)
                A, _ = orc.rrq_panel_systems(P["sx"][sl], P["snx"][sl], P["sw"][sl], nterms)
                kap = float(np.linalg.cond(A))
                if kappa_cache is not None:
                    kappa_cache[k] = kap
            for g, o in rows:
                e = np.abs(g[rrq] - o[rrq]).max() / np.abs(o[rrq]).max()
                worst_ratio = max(worst_ratio, float(e / (C_KAPPA * kap * U64 + FLOOR_RRQ)))
    return worst_level, worst_ratio
