"""Adaptive charts (the reference's build_charts_adaptive,
utils/stellarator_geo_mex.c:427-546, the chart list of its W7-X-style runs):
the library's host builder (qol_surface_charts) against the reference's own
C, compiled from its source into oracle/_ref (exact equality, several
surfaces, grids and tolerances; skipped without that build), and against the
fixture that C wrote (tests/golden/adaptive_charts.npz, always)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_adaptive_charts_match_reference_fixture(qol):
    from qotential_b200 import geometry as G
    z = np.load(os.path.join(HERE, "golden", "adaptive_charts.npz"))
    cl = qol.qol_surface_charts(G.stellarator(), int(z["mp"]), int(z["np_"]), int(z["p"]), float(z["restol"]))
    assert np.array_equal(cl, z["charts"])


@pytest.mark.parametrize("case", ["stellarator", "builtin", "family"])
@pytest.mark.parametrize("mp,np_,p,restol", [(4, 12, 5, 0.0), (8, 24, 7, 0.0), (8, 24, 7, 1e-2), (8, 24, 7, 1e-3)])
def test_adaptive_charts_match_reference_build(qol, orc, case, mp, np_, p, restol):
    from qotential_b200 import geometry as G
    if orc.refgeo() is None:
        pytest.skip("oracle/_ref (the reference's geometry generator) not built")
    surf = {"stellarator": G.stellarator(), "builtin": G.BuiltinSurface(),
            "family": G.family_surface(np.random.default_rng(3))}[case]
    modes, nfp = surf.vmec_modes()
    a = qol.qol_surface_charts(surf, mp, np_, p, restol)
    b = orc.ref_charts(mp, np_, p, modes, nfp, restol)
    assert np.array_equal(a, b), (a.shape, b.shape)


def test_adaptive_charts_refine_and_cap(qol):
    """curvature refinement only adds charts (quarters); a cap below the
    count is refused with QOL_ERR_NNZ"""
    from qotential_b200 import geometry as G
    surf = G.stellarator()
    n0 = qol.qol_surface_charts(surf, 6, 16, 6, 0.0).shape[0]
    cl = qol.qol_surface_charts(surf, 6, 16, 6, 1e-2)
    assert cl.shape[0] > n0 and (cl.shape[0] - n0) % 3 == 0
    area = (cl[:, 0] * cl[:, 2]).sum()  # the charts tile the 6 x 16 parameter cells (each of area 1 in a1 a2 units)
    assert abs(area - 6 * 16) < 1e-9
    with pytest.raises(qol.QolError) as e:
        qol.qol_surface_charts(surf, 6, 16, 6, 1e-2, cap=100)
    assert e.value.code == 2
