"""CUDA graphs of the device entry's back stage (no counterpart in the
reference): on a created stream a call captures its launches after the RRQ
count (level sums, RRQ phases, COO indices) and later calls with the same
arguments replay the graph; new arguments recapture it.  Every call's outputs
equal those of the same call on the legacy default stream, which cannot be
captured and so launches directly, byte for byte."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_replays_match_direct_launches(qol):
    import torch
    from qotential_b200 import geometry as G
    nterms = 7
    P = G.panels(G.stellarator(), 4, 12, nterms, split=False)
    hd = nterms * (nterms + 1) // 2
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 600, 3, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
    D = {k: t(P[k]) for k in ("sx", "snx", "sw", "rts", "rps")}
    q = (t(tcx), t(tcxrow, torch.int64), t(tcxi, torch.int64))
    npan, nq, nnz = P["sw"].size // hd, nterms + 2, tcxrow.size * hd

    def outputs():
        return (torch.zeros(nnz, dtype=torch.int64, device=dev), torch.zeros(nnz, dtype=torch.int64, device=dev),
                torch.zeros(nnz, dtype=torch.float64, device=dev), torch.zeros(nnz, dtype=torch.float64, device=dev))

    def call(out, stream):
        torch.cuda.synchronize()
        h = qol.qol_getnearquad_lap_rrq_dev(npan, nterms, nq, D["sx"], D["snx"], D["sw"], D["rts"], D["rps"], *q, nq,
                                            1.4, 30, out, stream=stream, sync=True, want_hist=True)
        return h, [o.cpu().numpy() for o in out]

    h0, ref = call(outputs(), 0)  # legacy default stream: direct launches
    s = torch.cuda.Stream(dev)
    out = outputs()
    c0, r0 = qol.qol_graph_stats()
    for _ in range(3):
        for o in out:
            o.zero_()
        h, got = call(out, s.cuda_stream)
        assert np.array_equal(h, h0)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    c1, r1 = qol.qol_graph_stats()
    assert (c1 - c0, r1 - r0) == (1, 2)  # one capture, then replays
    out2 = outputs()  # new buffers: new launch arguments, a new graph
    h, got = call(out2, s.cuda_stream)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    c2, r2 = qol.qol_graph_stats()
    assert (c2 - c1, r2 - r1) == (1, 0)
    qol.qol_set_graphs(0)  # switched off: direct launches, the same outputs
    try:
        h, got = call(out2, s.cuda_stream)
    finally:
        qol.qol_set_graphs(1)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    assert qol.qol_graph_stats() == (c2, r2)
