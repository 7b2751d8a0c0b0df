"""STGRF001: the reference's binary result format of a GRF run
(web/stellarator/native/stellarator_direct_main.f90:81-86 writes it,
web/stellarator/test/native-direct-parity.py:41-97 reads and validates it).

Layout, little-endian: the 8-byte magic "STGRF001"; ntri, nsrc, nrender,
nfaces (int64); the GRF scalar max|u| / max|du/dn| (f64); then the f64 arrays
sx (3 nsrc, node-major), snx (3 nsrc), sw, ub, ubn, u (nsrc each),
render_xyz (3 nrender), render_log_error (nrender) and the int64 array
render_triangles (3 nfaces, 0-based vertex indices).  The render lattice is the
reference's (build_render_lattice, stellarator_grf_core_mod.f90:976-1066): the
15 points (i/4, j/4), i + j <= 4, of every triangle mapped through its chart,
log10(max(|u interpolated| / max|du/dn|, 1e-16)) at each, and 16 faces a
triangle.

``write`` produces a file that the reference's parity script accepts; ``read``
applies the same checks as that script.
"""
import struct

import numpy as np

MAGIC = b"STGRF001"
KRENDER = 4
NVR = 15   # lattice points a triangle
NFR = 16   # lattice faces a triangle
FIELDS = ("sx", "snx", "sw", "ub", "ubn", "u", "render_xyz", "render_log_error", "render_triangles")


def render_uv():
    """The lattice points (i/4, j/4), i + j <= 4, in the reference's order."""
    return np.array([(i / KRENDER, j / KRENDER) for i in range(KRENDER + 1) for j in range(KRENDER + 1 - i)])


def _vertex(i, j):
    return 1 + i * 5 - i * (i - 1) // 2 + j


def render_faces(ntri):
    """Vertex indices (0-based) of the 16 lattice faces of every triangle."""
    one = []
    for i in range(KRENDER):
        for j in range(KRENDER - i):
            one.append((_vertex(i, j) - 1, _vertex(i + 1, j) - 1, _vertex(i, j + 1) - 1))
            if j < KRENDER - 1 - i:
                one.append((_vertex(i + 1, j) - 1, _vertex(i + 1, j + 1) - 1, _vertex(i, j + 1) - 1))
    one = np.array(one, dtype=np.int64)
    assert one.shape == (NFR, 3)
    return (one[None, :, :] + NVR * np.arange(ntri, dtype=np.int64)[:, None, None]).reshape(-1, 3)


def render_lattice(surface, mp, np_, nterms, u, ubn, split=True):
    """(render_xyz (ntri*15, 3), render_log_error (ntri*15,), render_triangles
    (ntri*16, 3)) of a run on ``surface`` (charts as geometry.panels)."""
    import qotential_b200 as qol
    from qotential_b200 import geometry as G
    uv = render_uv()
    xyz = G.panel_uv2x(surface, mp, np_, nterms, uv, split=split).reshape(-1, 3)
    ntri = xyz.shape[0] // NVR
    hd = nterms * (nterms + 1) // 2
    M = qol.qol_interp_matrix(nterms - 1, uv)           # NVR x hd
    ru = (np.asarray(u, np.float64).reshape(ntri, hd) @ M.T).ravel()
    if not np.all(np.isfinite(ru)) or np.abs(ru).max() > 1e300:
        raise ValueError("non-finite or overflowing interpolated u (status 32 of the reference)")
    scale = np.abs(np.asarray(ubn)).max()
    loge = np.log10(np.maximum(np.abs(ru) / scale, 1e-16))
    return xyz, loge, render_faces(ntri)


def write(path, ntri, sx, snx, sw, ub, ubn, u, render_xyz, render_log_error, render_triangles):
    """Write an STGRF001 file; the GRF scalar is max|u| / max|ubn|."""
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype="<f8").ravel())
    sw, ub, ubn, u = f64(sw), f64(ub), f64(ubn), f64(u)
    nsrc = sw.size
    xyz = f64(render_xyz)
    tri = np.ascontiguousarray(np.asarray(render_triangles, dtype="<i8").ravel())
    nrender, nfaces = xyz.size // 3, tri.size // 3
    grf = float(np.abs(u).max() / np.abs(ubn).max())
    with open(path, "wb") as fh:
        fh.write(struct.pack("<8s4qd", MAGIC, int(ntri), int(nsrc), int(nrender), int(nfaces), grf))
        for a in (f64(sx), f64(snx), sw, ub, ubn, u, xyz, f64(render_log_error)):
            fh.write(a.tobytes())
        fh.write(tri.tobytes())
    return grf


def read(path):
    """Read and validate an STGRF001 file (the checks of the reference's parity
    script): returns dict(ntri, nsrc, nrender, nfaces, grf, sx, snx, sw, ub,
    ubn, u, render_xyz, render_log_error, render_triangles)."""
    blob = open(path, "rb").read()
    if len(blob) < 48:
        raise ValueError(f"{path}: truncated header")
    magic, ntri, nsrc, nrender, nfaces, grf = struct.unpack_from("<8s4qd", blob)
    if magic != MAGIC:
        raise ValueError(f"{path}: bad magic {magic!r}")
    counts = {"sx": 3 * nsrc, "snx": 3 * nsrc, "sw": nsrc, "ub": nsrc, "ubn": nsrc, "u": nsrc,
              "render_xyz": 3 * nrender, "render_log_error": nrender, "render_triangles": 3 * nfaces}
    out = dict(ntri=ntri, nsrc=nsrc, nrender=nrender, nfaces=nfaces, grf=grf)
    off = 48
    for name in FIELDS:
        n = counts[name]
        if off + 8 * n > len(blob):
            raise ValueError(f"{path}: truncated {name}")
        dt = "<i8" if name == "render_triangles" else "<f8"
        out[name] = np.frombuffer(blob, dtype=dt, count=n, offset=off).copy()
        off += 8 * n
    if off != len(blob):
        raise ValueError(f"{path}: {len(blob) - off} trailing bytes")
    for name in FIELDS[:-1]:
        if not np.all(np.isfinite(out[name])):
            raise ValueError(f"{path}: non-finite value in {name}")
    tri = out["render_triangles"]
    if tri.size and (tri.min() < 0 or tri.max() >= nrender):
        raise ValueError(f"{path}: triangle index out of range")
    if out["render_log_error"].size and out["render_log_error"].min() < -16.0:
        raise ValueError(f"{path}: render log floor below -16")
    if np.abs(out["u"]).max() / np.abs(out["ubn"]).max() != grf:
        raise ValueError(f"{path}: GRF scalar {grf} != measured")
    for k in ("sx", "snx", "render_xyz"):
        out[k] = out[k].reshape(-1, 3)
    out["render_triangles"] = tri.reshape(-1, 3)
    return out
