"""qol_rrq_noalloc: the single-panel close correction for callers that cannot
allocate GPU memory (e.g. codes inside an application that owns all GPU
memory through its own pool, or on a path where cudaMalloc's implicit
synchronisation is not allowed).  Its workspace is a static 16 MiB device
array, so this test checks that calls in a row reproduce the allocating
entry point qol_rrq byte for byte (the same kernels and tables), also after a
call of another order has replaced the tables in the array, that the calls
leave the device's free memory unchanged, that an oversized request is
refused with QOL_ERR_LIMIT and a host pointer with QOL_ERR_ARG.  Collected
last on purpose: it runs after every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def _prepare(nterms, k):
    """device copies of one panel's inputs and NaN-filled outputs"""
    import torch
    P, hd, geo = _panel(nterms, k)
    tx = _targets(P, hd, k, geo[0], geo[1], geo[2])
    m = tx.shape[0]
    dev = [torch.as_tensor(a).cuda() for a in (tx,) + geo]
    out = [torch.full((m * hd,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    return dict(nterms=nterms, hd=hd, m=m, tx=tx, geo=geo, dev=dev, out=out)


def _call_dev(qol, c):
    L = qol.lib()
    L.qol_noalloc_last_error.restype = C.c_char_p
    p = lambda t: C.c_void_p(t.data_ptr())
    n = c["nterms"]
    rc = L.qol_rrq_noalloc(C.c_longlong(c["m"]), p(c["dev"][0]), C.c_longlong(c["hd"]), *[p(t) for t in c["dev"][1:]],
                           C.c_longlong(n), C.c_longlong(n + 2), C.c_longlong(n + 2), C.c_double(1.4),
                           C.c_longlong(1), p(c["out"][0]), p(c["out"][1]), C.c_void_p(0))
    return rc, L.qol_noalloc_last_error().decode()


def _call(qol, tx, geo, nterms, As, Ad):
    import torch
    d = [torch.as_tensor(a).cuda() for a in (tx,) + geo]
    c = dict(nterms=nterms, hd=nterms * (nterms + 1) // 2, m=tx.shape[0], dev=d, out=[As, Ad])
    rc, msg = _call_dev(qol, c)
    torch.cuda.synchronize()
    return rc, msg


def test_noalloc_matches_qol_rrq_twice(qol):
    import torch
    first = _prepare(7, 11)
    rc, msg = _call_dev(qol, first)  # first call on this device: set-up (symbol address, constants)
    assert rc == 0, msg
    # order 7, order 9 (its tables replace order 7's in the array), order 7 again;
    # inputs and outputs allocated before the free memory is read
    cases = [_prepare(n, k) for n, k in ((7, 11), (9, 5), (7, 11))]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for c in cases:
        rc, msg = _call_dev(qol, c)
        assert rc == 0, msg
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0  # the calls took no device memory
    for c in cases:
        n, hd, m = c["nterms"], c["hd"], c["m"]
        a = c["out"][0].cpu().numpy().reshape(hd, m).T
        d = c["out"][1].cpu().numpy().reshape(hd, m).T
        Bs, Bd, _, _, _ = qol.qol_rrq(c["tx"], *c["geo"], n, n + 2, n + 2)
        assert np.isfinite(a).all() and np.isfinite(d).all()
        assert np.array_equal(a, Bs) and np.array_equal(d, Bd), n


def test_noalloc_refuses_host_pointer(qol):
    import torch
    nterms, k = 7, 11
    P, hd, geo = _panel(nterms, k)
    L = qol.lib()
    L.qol_noalloc_last_error.restype = C.c_char_p
    d = [torch.as_tensor(a).cuda() for a in geo]
    p = lambda t: C.c_void_p(t.data_ptr())
    host_tx = np.ascontiguousarray(geo[0][:4] + 1.0)  # pageable host memory
    As = torch.zeros(4 * hd, dtype=torch.float64, device="cuda")
    Ad = torch.zeros(4 * hd, dtype=torch.float64, device="cuda")
    rc = L.qol_rrq_noalloc(C.c_longlong(4), C.c_void_p(host_tx.ctypes.data), C.c_longlong(hd), *[p(t) for t in d],
                           C.c_longlong(nterms), C.c_longlong(nterms + 2), C.c_longlong(nterms + 2), C.c_double(1.4),
                           C.c_longlong(1), p(As), p(Ad), C.c_void_p(0))
    assert rc == 8 and "tx" in L.qol_noalloc_last_error().decode()  # QOL_ERR_ARG


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
