"""Batched near corrections: many surfaces in one pipeline pass per order.

Surfaces that share (nterms, nquad, orderff) are concatenated into one
qol_getnearquad_lap_rrq problem, so one set of kernel launches serves all of
them (the per-panel and per-pair work is independent, and every panel keeps
its own target list).  Numbering of the combined problem: all surfaces'
sources first, then all off-surface targets; an on-surface target keeps the
id of its node (so the self-pair masking of the naive block, row == source
node, holds), an off-surface one is numbered after every source.  The COO
output is split back per surface with its own numbering.

A problem is a dict with the getnearquad inputs of one surface: nterms, nquad,
orderff, sx, snx, sw, rts, rps (hd nodes a panel), tcx (ntcx x 3), tcxrow
(1-based ids: 1..nsrc nodes, above that off-surface targets), tcxi (npan+1,
1-based).  No counterpart in the reference (it has one surface per call).
"""
import numpy as np

from . import qol_getnearquad_lap_rrq, qol_getnearquad_lap_rrq_batch_dev, qol_getnearquad_lap_rrq_dev


def _key(p):
    return (int(p["nterms"]), int(p["nquad"]), int(p["orderff"]))


def combine(problems):
    """one problem from surfaces of one order, and the offsets to split its output"""
    nterms, nquad, orderff = _key(problems[0])
    hd = nterms * (nterms + 1) // 2
    nsrc = [np.asarray(p["sw"]).size for p in problems]
    src_off = np.concatenate([[0], np.cumsum(nsrc)])
    ntot = int(src_off[-1])
    noff = [int(max(0, np.asarray(p["tcxrow"]).max(initial=0) - n)) for p, n in zip(problems, nsrc)]
    off_off = np.concatenate([[0], np.cumsum(noff)])
    rows, xis, pair_off = [], [np.array([1], np.int64)], [0]
    for s, p in enumerate(problems):
        r = np.asarray(p["tcxrow"], np.int64)
        on = r <= nsrc[s]
        rows.append(np.where(on, r + src_off[s], r - nsrc[s] + ntot + off_off[s]))
        xi = np.asarray(p["tcxi"], np.int64)
        xis.append(xi[1:] - 1 + pair_off[-1] + 1)
        pair_off.append(pair_off[-1] + int(xi[-1] - 1))
    cat = lambda k, shape: np.concatenate([np.asarray(p[k], np.float64).reshape(shape) for p in problems])
    comb = dict(nterms=nterms, nquad=nquad, orderff=orderff, npan=ntot // hd, hd=hd, nsrc=ntot,
                sx=cat("sx", (-1, 3)), snx=cat("snx", (-1, 3)), sw=cat("sw", (-1,)), rts=cat("rts", (-1, 3)),
                rps=cat("rps", (-1, 3)), tcx=cat("tcx", (-1, 3)), tcxrow=np.concatenate(rows),
                tcxi=np.concatenate(xis))
    split = dict(hd=hd, nsrc=nsrc, src_off=src_off, ntot=ntot, off_off=off_off, pair_off=pair_off)
    return comb, split


def split_output(si, sj, vs, vd, split):
    """per-surface (sparsei, sparsej, sparsevs, sparsevd) in each surface's numbering"""
    hd, out = split["hd"], []
    for s in range(len(split["nsrc"])):
        a, b = split["pair_off"][s] * hd, split["pair_off"][s + 1] * hd
        r = np.asarray(si[a:b], np.int64)
        on = r <= split["ntot"]
        rl = np.where(on, r - split["src_off"][s], r - split["ntot"] - split["off_off"][s] + split["nsrc"][s])
        out.append((rl, np.asarray(sj[a:b], np.int64) - split["src_off"][s], vs[a:b], vd[a:b]))
    return out


def getnearquad_batch(problems, distff=1.4, iside=30):
    """near corrections of every surface, one host-entry call per order group;
    a list of (sparsei, sparsej, sparsevs, sparsevd) in the input order"""
    groups = {}
    for i, p in enumerate(problems):
        groups.setdefault(_key(p), []).append(i)
    res = [None] * len(problems)
    for key, idx in groups.items():
        comb, split = combine([problems[i] for i in idx])
        si, sj, vs, vd, _ = qol_getnearquad_lap_rrq(comb["npan"], comb["nterms"], comb["hd"], comb["nquad"],
                                                    comb["nsrc"], comb["sx"], comb["snx"], comb["sw"], comb["rts"],
                                                    comb["rps"], comb["tcxrow"].size, comb["tcx"], comb["tcxrow"],
                                                    comb["tcxi"], comb["orderff"], distff, iside)
        for i, r in zip(idx, split_output(si, sj, vs, vd, split)):
            res[i] = r
    return res


def device_inputs(comb, dev):
    """the combined problem's inputs as CUDA tensors (device entry point)"""
    import torch
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)
    D = {k: t(comb[k]) for k in ("sx", "snx", "sw", "rts", "rps", "tcx")}
    D["tcxrow"] = t(comb["tcxrow"], torch.int64)
    D["tcxi"] = t(comb["tcxi"], torch.int64)
    return D


def run_device(comb, D, out, stream=0, sync=False, distff=1.4, iside=30):
    """one device-entry pass of a combined (or single) problem"""
    return qol_getnearquad_lap_rrq_dev(comb["npan"], comb["nterms"], comb["nquad"], D["sx"], D["snx"], D["sw"],
                                       D["rts"], D["rps"], D["tcx"], D["tcxrow"], D["tcxi"], comb["orderff"], distff,
                                       iside, out, stream=stream, sync=sync)


def run_device_batch(combs, Ds, outs, stream=0, distff=1.4, iside=30):
    """every combined problem (any orders) in ONE library call: the level sums
    of all of them in one persistent launch fed by a level-binned work queue;
    returns the level histograms"""
    jobs = [dict(npan=c["npan"], nterms=c["nterms"], nquad=c["nquad"], orderff=c["orderff"], distff=distff,
                 iside=iside, out=o, **{k: D[k] for k in ("sx", "snx", "sw", "rts", "rps", "tcx", "tcxrow", "tcxi")})
            for c, D, o in zip(combs, Ds, outs)]
    return qol_getnearquad_lap_rrq_batch_dev(jobs, stream=stream)
