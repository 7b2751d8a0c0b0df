"""The GPU GRF path on the inputs of the reference's frozen native fixtures
(web/stellarator/fixtures/native/order{4,6}-direct.bin: built-in surface,
mp 12 x np 36, nterms 4 and 6, Direct far field, ichart = 1, density
exp(x/2) cos(y/2)), compared with the reference's own output u (committed
under tests/golden/) and with the oracle on the same inputs.

Bounds against the reference's u: the oracle's measured agreement (fieldScaled
3.5e-3 / 6.5e-3, the reference's own cross-toolchain gate being 3e-3,
web/stellarator/test/wasm-api-node.mjs:364), the near-pair count exact.
Against the oracle: the near phase to TOL_U, as for the other GRF tests."""
import os

import numpy as np
import pytest

from conftest import fixture_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL_U = 1e-10


@pytest.mark.parametrize("order,pairs,fs_bound,mean_bound", [
    (4, 137259, 4.0e-3, 2.0e-4),
    (6, 287821, 7.0e-3, 2.0e-5),
])
def test_gpu_fixture_chart_boundary(qol, orc, order, pairs, fs_bound, mean_bound):
    z = np.load(os.path.join(HERE, "golden", f"grf_order{order}.npz"))
    F = fixture_case(orc, order)
    P = F["P"]
    assert P["sw"].size == int(z["nsrc"])
    uf = qol.qol_direct_farfield(P["sx"], P["snx"], P["sw"], F["ub"], F["ubn"])
    ug, nn, hist = qol.qol_grf_near(F["npan"], order, F["nq"], P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                    F["ub"], F["ubn"], u=uf, xbuf=F["xbuf"])
    assert nn == pairs and hist[5] > 0
    # against the reference's frozen output
    du = np.abs(ug - z["u"])
    assert du.max() / max(1.0, np.abs(z["u"]).max()) < fs_bound
    assert du.mean() < mean_bound
    # against the oracle on the same inputs (chart boundary included)
    uo_far = orc.direct_farfield(P["sx"], P["snx"], P["sw"], F["ub"], F["ubn"])
    offs, idx = orc.ballcsr(F["npan"], F["hd"], P["sx"], P["sw"])
    uo, _, histo = orc.grf_near(F["npan"], order, F["nq"], F["nq"], P["sx"], P["snx"], P["sw"], P["rts"], P["rps"],
                                F["ub"], F["ubn"], offs, idx, uo_far, xbuf=F["xbuf"])
    assert np.array_equal(hist, histo)
    err = np.abs(ug - uo).max() / np.abs(uo).max()
    assert err < TOL_U, err
