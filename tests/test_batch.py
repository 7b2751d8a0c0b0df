"""Batched near corrections (qotential_b200.batch): surfaces of one order in
one pipeline pass.  CPU: the combined numbering splits back to each surface's
own COO indices.  GPU: the batched values are each surface's own call's,
byte for byte (every panel and pair is computed independently)."""
import numpy as np
import pytest


def _problems(G, spec, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for nterms, mp, np_ in spec:
        surf = G.family_surface(rng)
        P = G.panels(surf, mp, np_, nterms, split=False)
        hd = nterms * (nterms + 1) // 2
        T = np.concatenate([P["sx"], G.off_surface_targets(P, 200, int(rng.integers(1 << 30)), hd)])
        tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
        out.append(dict(nterms=nterms, nquad=nterms + 2, orderff=nterms + 2, sx=P["sx"], snx=P["snx"], sw=P["sw"],
                        rts=P["rts"], rps=P["rps"], tcx=tcx, tcxrow=tcxrow, tcxi=tcxi))
    return out


def _coo_indices(hd, tcxrow, tcxi):
    """the reference's COO index layout: panel k's block (tcxi(k)-1) hd + (j-1) m + i"""
    si, sj = [], []
    for k in range(len(tcxi) - 1):
        a, b = tcxi[k] - 1, tcxi[k + 1] - 1
        for j in range(hd):
            si.append(tcxrow[a:b])
            sj.append(np.full(b - a, k * hd + j + 1))
    return np.concatenate(si), np.concatenate(sj)


def test_batch_numbering_round_trip():
    from qotential_b200 import batch as B
    from qotential_b200 import geometry as G
    probs = _problems(G, [(4, 4, 8), (4, 5, 10), (4, 4, 9)])
    comb, split = B.combine(probs)
    assert comb["npan"] * comb["hd"] == comb["nsrc"] and comb["tcxi"][-1] == comb["tcxrow"].size + 1
    si, sj = _coo_indices(comb["hd"], comb["tcxrow"], comb["tcxi"])
    z = np.zeros(si.size)
    for p, (ri, rj, _, _) in zip(probs, B.split_output(si, sj, z, z, split)):
        ei, ej = _coo_indices(comb["hd"], np.asarray(p["tcxrow"]), np.asarray(p["tcxi"]))
        assert np.array_equal(ri, ei) and np.array_equal(rj, ej)


@pytest.mark.gpu
def test_batch_matches_single_calls(qol):
    from qotential_b200 import batch as B
    from qotential_b200 import geometry as G
    probs = _problems(G, [(5, 4, 8), (6, 4, 9), (5, 5, 10), (6, 4, 8)], seed=4)
    res = B.getnearquad_batch(probs)
    for p, r in zip(probs, res):
        nt = p["nterms"]
        hd = nt * (nt + 1) // 2
        npan = p["sw"].size // hd
        one = qol.qol_getnearquad_lap_rrq(npan, nt, hd, p["nquad"], npan * hd, p["sx"], p["snx"], p["sw"], p["rts"],
                                          p["rps"], p["tcxrow"].size, p["tcx"], p["tcxrow"], p["tcxi"], p["orderff"],
                                          1.4, 30)
        for x, y in zip(r, one[:4]):
            assert np.asarray(x).tobytes() == np.asarray(y).tobytes()


@pytest.mark.gpu
def test_one_call_batch_matches_single_calls(qol):
    """surfaces of orders 4, 7 and 12 (one to three interpolation column
    blocks) in one qol_getnearquad_lap_rrq_batch_dev call, the level sums of
    all in one persistent launch: every job's COO and level histogram equal its
    own device call's, byte for byte"""
    import torch
    from qotential_b200 import batch as B
    from qotential_b200 import geometry as G
    probs = _problems(G, [(5, 4, 8), (8, 4, 9), (13, 3, 8), (5, 5, 10), (13, 3, 6)], seed=6)
    groups = {}
    for p in probs:
        groups.setdefault(B._key(p), []).append(p)
    combs = [B.combine(ps)[0] for ps in groups.values()]
    dev = torch.device("cuda", torch.cuda.current_device())
    Ds = [B.device_inputs(c, dev) for c in combs]

    def outbuf(c):
        n = int(c["tcxrow"].size) * c["hd"]
        return (torch.full((n,), -1, dtype=torch.int64, device=dev), torch.full((n,), -1, dtype=torch.int64, device=dev),
                torch.full((n,), np.nan, dtype=torch.float64, device=dev),
                torch.full((n,), np.nan, dtype=torch.float64, device=dev))

    batch_out = [outbuf(c) for c in combs]
    hist = B.run_device_batch(combs, Ds, batch_out)
    torch.cuda.synchronize()
    for c, D, bo, h in zip(combs, Ds, batch_out, hist):
        so = outbuf(c)
        hs = qol.qol_getnearquad_lap_rrq_dev(c["npan"], c["nterms"], c["nquad"], D["sx"], D["snx"], D["sw"], D["rts"],
                                             D["rps"], D["tcx"], D["tcxrow"], D["tcxi"], c["orderff"], 1.4, 30, so,
                                             want_hist=True)
        torch.cuda.synchronize()
        assert np.array_equal(np.asarray(h), np.asarray(hs))
        for x, y in zip(bo, so):
            assert x.cpu().numpy().tobytes() == y.cpu().numpy().tobytes()
