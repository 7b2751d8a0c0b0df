"""Re-entrancy of the device entry point per stream (no counterpart in the
reference, which is single-threaded): qol_getnearquad_lap_rrq_dev calls from
several host threads run concurrently when their streams differ, each on its
stream's own workspace, and in turn when they share a stream.  Their outputs
equal the same calls made one at a time, byte for byte."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = ((7, 4, 12, 600, 1), (9, 4, 10, 400, 2), (5, 6, 16, 800, 3), (7, 4, 12, 600, 4))  # nterms, mp, np, off, seed


class _Problem:
    """one getnearquad problem: device inputs and outputs"""

    def __init__(self, torch, dev, nterms, mp, np_, off, seed):
        from qotential_b200 import geometry as G
        P = G.panels(G.stellarator(), mp, np_, nterms, split=False)
        hd = nterms * (nterms + 1) // 2
        T = np.concatenate([P["sx"], G.off_surface_targets(P, off, seed, hd)])
        tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
        t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
        self.D = {k: t(P[k]) for k in ("sx", "snx", "sw", "rts", "rps")}
        self.q = (t(tcx), t(tcxrow, torch.int64), t(tcxi, torch.int64))
        self.npan, self.nterms = P["sw"].size // hd, nterms
        nnz = tcxrow.size * hd
        self.out = (torch.empty(nnz, dtype=torch.int64, device=dev), torch.empty(nnz, dtype=torch.int64, device=dev),
                    torch.empty(nnz, dtype=torch.float64, device=dev), torch.empty(nnz, dtype=torch.float64, device=dev))

    def run(self, qol, stream):
        nq = self.nterms + 2
        D = self.D
        return qol.qol_getnearquad_lap_rrq_dev(self.npan, self.nterms, nq, D["sx"], D["snx"], D["sw"], D["rts"],
                                               D["rps"], *self.q, nq, 1.4, 30, self.out, stream=stream, sync=True,
                                               want_hist=True)

    def result(self):
        return [o.cpu().numpy() for o in self.out]


def test_concurrent_calls_match_sequential(qol):
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    probs = [_Problem(torch, dev, *c) for c in CASES]
    streams = [torch.cuda.Stream(dev) for _ in range(2)]
    which = [0, 1, 0, 1]  # two threads on each stream
    ref, ref_hist = [], []
    for p, k in zip(probs, which):
        ref_hist.append(p.run(qol, streams[k].cuda_stream))
        ref.append(p.result())
    for _ in range(3):
        for p in probs:
            for o in p.out:
                o.zero_()
        torch.cuda.synchronize()
        errs, hists = [], [None] * len(probs)

        def work(i):
            try:
                hists[i] = probs[i].run(qol, streams[which[i]].cuda_stream)
            except Exception as e:  # reported below
                errs.append(e)

        threads = [threading.Thread(target=work, args=(i,)) for i in range(len(probs))]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        assert not errs, errs
        for p, r, h, rh in zip(probs, ref, hists, ref_hist):
            assert np.array_equal(h, rh)
            for a, b in zip(p.result(), r):
                assert np.array_equal(a, b)
