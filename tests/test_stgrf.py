"""STGRF001, the reference's GRF result file (written by
web/stellarator/native/stellarator_direct_main.f90:81-86, read by
web/stellarator/test/native-direct-parity.py:41-97): round trip, the reader's
checks, and the render lattice against the reference's own fixtures'
(tests/golden/render_order{4,6}.npz: every 11th render vertex of
order{4,6}-direct.bin)."""
import hashlib
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _blob_args(rng, ntri=3, hd=6):
    nsrc = ntri * hd
    from qotential_b200 import stgrf
    u = rng.normal(size=nsrc) * 1e-3
    return (ntri, rng.normal(size=(nsrc, 3)), rng.normal(size=(nsrc, 3)), rng.random(nsrc), rng.normal(size=nsrc),
            rng.normal(size=nsrc), u, rng.normal(size=(ntri * stgrf.NVR, 3)), -rng.random(ntri * stgrf.NVR),
            stgrf.render_faces(ntri))


def test_round_trip_and_checks(tmp_path):
    from qotential_b200 import stgrf
    rng = np.random.default_rng(1)
    args = _blob_args(rng)
    path = tmp_path / "a.bin"
    grf = stgrf.write(path, *args)
    d = stgrf.read(path)
    assert d["ntri"] == 3 and d["nsrc"] == 18 and d["nrender"] == 45 and d["nfaces"] == 48
    assert d["grf"] == grf == np.abs(args[6]).max() / np.abs(args[5]).max()
    for k, a in zip(("sx", "snx", "sw", "ub", "ubn", "u", "render_xyz", "render_log_error", "render_triangles"),
                    args[1:]):
        assert np.array_equal(d[k], np.asarray(a).reshape(d[k].shape))
    blob = path.read_bytes()
    bad = tmp_path / "b.bin"
    for corrupt, msg in ((b"STGRF002" + blob[8:], "magic"), (blob[:-8], "truncated"), (blob + b"\0" * 8, "trailing"),
                         (blob[:40] + np.float64(1.0).tobytes() + blob[48:], "GRF scalar")):
        bad.write_bytes(corrupt)
        with pytest.raises(ValueError, match=msg):
            stgrf.read(bad)
    tri = args[9].copy(); tri[0, 0] = 45
    stgrf.write(bad, *args[:9], tri)
    with pytest.raises(ValueError, match="out of range"):
        stgrf.read(bad)


def test_render_faces_cover_the_lattice():
    from qotential_b200 import stgrf
    f = stgrf.render_faces(2)
    assert f.shape == (32, 3) and f.min() == 0 and f.max() == 29
    assert len({tuple(sorted(t)) for t in f.tolist()}) == 32


@pytest.mark.parametrize("order", [4, 6])
def test_render_lattice_matches_reference_fixture(qol, order):
    """our lattice from the reference's own u: positions to 1e-13, log errors
    to 1e-10, the triangles' bytes identical (SHA-256)"""
    from qotential_b200 import geometry as G, stgrf
    z = np.load(os.path.join(HERE, "golden", f"grf_order{order}.npz"))
    r = np.load(os.path.join(HERE, "golden", f"render_order{order}.npz"))
    xyz, loge, tri = stgrf.render_lattice(G.BuiltinSurface(), 12, 36, order, z["u"], z["ubn"])
    assert xyz.shape[0] == int(r["nrender"]) and tri.shape[0] == int(r["nfaces"])
    sub = r["rsub"]
    assert np.abs(xyz[sub] - r["render_xyz_sub"]).max() < 1e-13
    assert np.abs(loge[sub] - r["render_log_error_sub"]).max() < 1e-10
    assert hashlib.sha256(tri.astype("<i8").tobytes()).hexdigest() == str(r["sha_render_triangles"])
