"""The geometry generator on the GPU (qol_surface_panels: the reference's
utils/stellarator_geo_mex.c geo_core) against the host restatement
(geometry.panels) and the reference's frozen fixture geometry, and a full GRF
run on the fixture inputs written as STGRF001 and read back."""
import os

import numpy as np
import pytest

from conftest import fixture_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-12  # relative to the field's largest magnitude (cos/sin and FMA rounding)


def _cmp(a, b):
    for k in ("sx", "snx", "sw", "rts", "rps"):
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.shape == y.shape, k
        assert np.abs(x - y).max() <= TOL * np.abs(y).max(), (k, np.abs(x - y).max())


@pytest.mark.parametrize("case", ["stellarator", "stellarator_split", "torus", "family", "builtin"])
def test_surface_panels_match_host(qol, case):
    from qotential_b200 import geometry as G
    nterms = 7
    if case == "stellarator":
        surf, mp, np_, split = G.stellarator(), 16, 80, False
    elif case == "stellarator_split":
        surf, mp, np_, split = G.stellarator(), 6, 12, True
    elif case == "torus":
        surf, mp, np_, split = G.torus(), 6, 12, False
    elif case == "family":
        surf, mp, np_, split = G.family_surface(np.random.default_rng(4)), 8, 24, True
    else:
        surf, mp, np_, split = G.BuiltinSurface(), 12, 36, True
    a = qol.qol_surface_panels(surf, mp, np_, nterms, split=split)
    b = G.panels(surf, mp, np_, nterms, split=split)
    assert a["ntri"] == b["ntri"]
    _cmp(a, b)


@pytest.mark.parametrize("order,pairs,fs_bound", [(4, 137259, 4.0e-3), (6, 287821, 7.0e-3)])
def test_fixture_run_from_gpu_geometry_as_stgrf001(qol, orc, tmp_path, order, pairs, fs_bound):
    from qotential_b200 import geometry as G, stgrf
    z = np.load(os.path.join(HERE, "golden", f"grf_order{order}.npz"))
    P = qol.qol_surface_panels(G.BuiltinSurface(), 12, 36, order)
    sub = z["sub"]
    assert P["sw"].size == int(z["nsrc"])
    assert np.abs(P["sx"][sub] - z["sx_sub"]).max() < 1e-12   # the reference's gate (wasm-api-node.mjs:359)
    assert np.abs(P["snx"][sub] - z["snx_sub"]).max() < 1e-12
    assert np.abs(P["sw"][sub] - z["sw_sub"]).max() < 1e-12
    F = fixture_case(orc, order)  # density and chart boundary
    hd = F["hd"]
    x = P["sx"]
    ub = np.exp(0.5 * x[:, 0]) * np.cos(0.5 * x[:, 1])
    gr = np.stack([0.5 * ub, -0.5 * np.exp(0.5 * x[:, 0]) * np.sin(0.5 * x[:, 1]), 0 * ub], 1)
    ubn = (P["snx"] * gr).sum(1)
    uf = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], ub, ubn)
    u, nn, hist = qol.qol_grf_near(P["ntri"], order, order + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub,
                                   ubn, u=uf, xbuf=F["xbuf"])
    assert nn == pairs
    xyz, loge, tri = stgrf.render_lattice(G.BuiltinSurface(), 12, 36, order, u, ubn)
    path = tmp_path / f"order{order}.bin"
    stgrf.write(path, P["ntri"], P["sx"], P["snx"], P["sw"], ub, ubn, u, xyz, loge, tri)
    d = stgrf.read(path)
    assert d["ntri"] == int(z["ntri"]) and d["nsrc"] == int(z["nsrc"])
    assert np.abs(d["ubn"] - z["ubn"]).max() < 1e-11          # the reference's gate (:362-363)
    du = np.abs(d["u"] - z["u"])
    assert du.max() / max(1.0, np.abs(z["u"]).max()) < fs_bound


def test_adaptive_chart_panels_match_reference_fixture(qol):
    """the GPU generator over the reference's adaptive chart list
    (qol_surface_panels_charts) against the panels the reference's
    stellarator_geo_charts made of it (tests/golden/adaptive_charts.npz)"""
    from qotential_b200 import geometry as G
    z = np.load(os.path.join(HERE, "golden", "adaptive_charts.npz"))
    p = int(z["p"])
    a = qol.qol_surface_panels_charts(G.stellarator(), int(z["mp"]), int(z["np_"]), p, z["charts"])
    assert a["ntri"] == 2 * z["charts"].shape[0]
    sub = z["sub"]
    for k in ("sx", "snx", "sw", "rts", "rps"):
        x, y = np.asarray(a[k])[sub], z[k + "_sub"]
        assert np.abs(x - y).max() <= TOL * np.abs(y).max(), (k, np.abs(x - y).max())
