"""qol_rrq_noalloc: the single-panel close correction for callers that cannot
allocate GPU memory (e.g. codes inside an application that owns all GPU
memory through its own pool, or on a path where cudaMalloc's implicit
synchronisation is not allowed).  Its workspace is a static 16 MiB device
array, so this test checks that two calls in a row reproduce the allocating
entry point qol_rrq, and that an oversized request is refused with
QOL_ERR_LIMIT.  Collected last on purpose: it runs after every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_RRQ = 1e-8  # the bound the other GPU parity tests use for RRQ rows


def _panel(nterms, k, mp=4, np_=10):
    from qotential_b200 import geometry as G
    P = G.panels(G.stellarator(), mp, np_, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    sl = slice(k * hd, (k + 1) * hd)
    return P, hd, tuple(np.ascontiguousarray(P[a][sl]) for a in ("sx", "snx", "sw", "rts", "rps"))


def _targets(P, hd, k, sx, snx, sw):
    rng = np.random.default_rng(11)
    diam = np.sqrt(sw.sum())
    tx = [sx, P["sx"][(k + 1) * hd:(k + 2) * hd]]
    for d in (1e-6, 1e-3, 0.05, 0.3, 1.5):
        j = rng.integers(0, hd, 5)
        tx.append(sx[j] + (d * diam * np.where(rng.random(5) < 0.5, -1, 1))[:, None] * snx[j])
    return np.ascontiguousarray(np.concatenate(tx))


def _call(qol, tx, geo, nterms, As, Ad):
    import torch
    L = qol.lib()
    L.qol_noalloc_last_error.restype = C.c_char_p
    d = [torch.as_tensor(a).cuda() for a in (tx,) + geo]
    p = lambda t: C.c_void_p(t.data_ptr())
    m = tx.shape[0]
    hd = nterms * (nterms + 1) // 2
    rc = L.qol_rrq_noalloc(C.c_longlong(m), p(d[0]), C.c_longlong(hd), p(d[1]), p(d[2]), p(d[3]), p(d[4]),
                           p(d[5]), C.c_longlong(nterms), C.c_longlong(nterms + 2), C.c_longlong(nterms + 2),
                           C.c_double(1.4), C.c_longlong(1), p(As), p(Ad), C.c_void_p(0))
    torch.cuda.synchronize()
    return rc, L.qol_noalloc_last_error().decode()


def test_noalloc_matches_qol_rrq_twice(qol):
    import torch
    nterms, k = 7, 11
    P, hd, geo = _panel(nterms, k)
    tx = _targets(P, hd, k, geo[0], geo[1], geo[2])
    m = tx.shape[0]
    Bs, Bd, _, _, _ = qol.qol_rrq(tx, *geo, nterms, nterms + 2, nterms + 2)
    for call in range(2):
        As = torch.full((m * hd,), float("nan"), dtype=torch.float64, device="cuda")
        Ad = torch.full((m * hd,), float("nan"), dtype=torch.float64, device="cuda")
        rc, msg = _call(qol, tx, geo, nterms, As, Ad)
        assert rc == 0, msg
        a = As.cpu().numpy().reshape(hd, m).T
        d = Ad.cpu().numpy().reshape(hd, m).T
        assert np.isfinite(a).all() and np.isfinite(d).all()
        assert np.abs(a - Bs).max() / np.abs(Bs).max() < TOL_RRQ, call
        assert np.abs(d - Bd).max() / np.abs(Bd).max() < TOL_RRQ, call


def test_noalloc_refuses_oversize(qol):
    import torch
    nterms, k = 13, 3
    P, hd, geo = _panel(nterms, k)
    m = 4000
    tx = np.ascontiguousarray(np.repeat(geo[0][:1], m, axis=0) + 10.0)
    As = torch.zeros(m * hd, dtype=torch.float64, device="cuda")
    Ad = torch.zeros(m * hd, dtype=torch.float64, device="cuda")
    rc, msg = _call(qol, tx, geo, nterms, As, Ad)
    assert rc == 9 and "scratch" in msg, (rc, msg)
