"""Extract the golden vectors the tests use from the reference's frozen native
fixtures (web/stellarator/fixtures/native/order{4,6}-direct.bin, format
STGRF001: header + f64 arrays sx, snx, sw, ub, ubn, u, ...; see
web/stellarator/test/native-direct-parity.py:41-97).

Writes tests/golden/grf_order{4,6}.npz with u, ub, ubn, the GRF scalar, a
strided subset of sx/snx/sw (every 7th node) and the SHA-256 of the full
f64 sx/snx/sw arrays, and tests/golden/render_order{4,6}.npz with the render
lattice's sizes, every 11th render vertex (position and log error) and the
SHA-256 of the render triangles, and tests/golden/adaptive_charts.npz: the
adaptive chart list of the reference's own geometry generator
(utils/stellarator_geo_mex.c stellarator_charts, compiled into oracle/_ref by
oracle/Makefile) for the stellarator surface, mp 6 x np 16, p 6, restol 1e-2,
and a strided subset of the panels its stellarator_geo_charts makes of that
list at nterms 6.  Run in a container that has the reference checkout,
naming its root (the argument, or the QOL_REFERENCE_DIR environment variable):
    python tests/golden/make_golden.py <reference checkout>
"""
import hashlib
import os
import struct
import sys

import numpy as np


def load(path):
    blob = open(path, "rb").read()
    magic, ntri, nsrc, nrender, nfaces, grf = struct.unpack_from("<8s4qd", blob)
    assert magic == b"STGRF001", magic
    off = 48
    out = dict(ntri=ntri, nsrc=nsrc, grf=grf, nrender=nrender, nfaces=nfaces)
    for name, cnt in [("sx", 3 * nsrc), ("snx", 3 * nsrc), ("sw", nsrc), ("ub", nsrc), ("ubn", nsrc), ("u", nsrc),
                      ("render_xyz", 3 * nrender), ("render_log_error", nrender)]:
        out[name] = np.frombuffer(blob, dtype="<f8", count=cnt, offset=off).copy()
        off += 8 * cnt
    out["render_triangles"] = np.frombuffer(blob, dtype="<i8", count=3 * nfaces, offset=off).copy()
    out["sha256"] = hashlib.sha256(blob).hexdigest()
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QOL_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set QOL_REFERENCE_DIR)")
    here = os.path.dirname(os.path.abspath(__file__))
    for order in (4, 6):
        f = load(os.path.join(ref, "web/stellarator/fixtures/native", f"order{order}-direct.bin"))
        sub = np.arange(0, f["nsrc"], 7)
        np.savez_compressed(
            os.path.join(here, f"grf_order{order}.npz"),
            ntri=f["ntri"], nsrc=f["nsrc"], grf=f["grf"], u=f["u"], ub=f["ub"], ubn=f["ubn"],
            sub=sub, sx_sub=f["sx"].reshape(-1, 3)[sub], snx_sub=f["snx"].reshape(-1, 3)[sub], sw_sub=f["sw"][sub],
            sha_sx=hashlib.sha256(f["sx"].tobytes()).hexdigest(),
            sha_snx=hashlib.sha256(f["snx"].tobytes()).hexdigest(),
            sha_sw=hashlib.sha256(f["sw"].tobytes()).hexdigest(),
            sha_bin=f["sha256"], mp=12, np_=36, order=order)
        rsub = np.arange(0, f["nrender"], 11)
        np.savez_compressed(
            os.path.join(here, f"render_order{order}.npz"), nrender=f["nrender"], nfaces=f["nfaces"], rsub=rsub,
            render_xyz_sub=f["render_xyz"].reshape(-1, 3)[rsub], render_log_error_sub=f["render_log_error"][rsub],
            sha_render_triangles=hashlib.sha256(f["render_triangles"].astype("<i8").tobytes()).hexdigest())
        print(order, f["sha256"])
    adaptive_charts(here)


def adaptive_charts(here, mp=6, np_=16, p=6, restol=1e-2):
    sys.path.insert(0, os.path.dirname(os.path.dirname(here)))
    import oracle as O
    from qotential_b200 import geometry as G
    modes, nfp = G.stellarator().vmec_modes()
    cl = O.ref_charts(mp, np_, p, modes, nfp, restol)
    geo = O.ref_geometry_charts(cl, mp, np_, p, modes, nfp)
    sub = np.arange(0, geo["sw"].size, 13)
    np.savez_compressed(os.path.join(here, "adaptive_charts.npz"), mp=mp, np_=np_, p=p, restol=restol, charts=cl,
                        sub=sub, sx_sub=geo["sx"].reshape(-1, 3)[sub], snx_sub=geo["snx"].reshape(-1, 3)[sub],
                        sw_sub=geo["sw"][sub], rts_sub=geo["rts"].reshape(-1, 3)[sub],
                        rps_sub=geo["rps"].reshape(-1, 3)[sub])
    print("adaptive charts", cl.shape[0])


if __name__ == "__main__":
    main()
