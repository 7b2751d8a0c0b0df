"""Work split of the near-field path over GPUs, one process per GPU.

The (target, panel) pairs are independent, so the panels are cut into
contiguous ranges, one per rank, balanced by an estimate of each panel's cost
(its near pairs, those close enough to land on the RRQ branch weighted by the
measured RRQ-to-direct cost ratio).  Source geometry is replicated.  Two
callers:

- ``getnearquad_shard``: one rank's part of qol_getnearquad_lap_rrq.  The
  rank passes only its panels; target rows are renumbered relative to the
  range (so the self-pair mask of the naive block compares rows with the
  range's own nodes) and the COO indices are shifted back, so the ranks'
  outputs concatenated in rank order are the single call's output.
- ``grf_near_sharded``: the GRF driver's near phase
  (web/stellarator/fortran/stellarator_grf_core_mod.f90:652-899) and its
  Direct far field (:566-606) with every node a target: each rank computes
  the near corrections of its panel range (qol_grf_near_range) and the far
  field of a target range (qol_direct_farfield_range), and one all-reduce
  (sum) over the process group adds the ranks' contributions.  The reference
  has no counterpart (one host, serial scatter at :892-896); the sum over
  ranks changes only the order in which a node's corrections are added.
"""
import numpy as np

# cost of an RRQ pair relative to a level-resolved one: the bench workload at
# order 12 spends 51 ms on 0.54 M RRQ pairs and 29 ms on 1.91 M direct pairs
RRQ_WEIGHT = 6.0
# pairs closer to the panel's node mean than this fraction of sqrt(area)
# resolve on the RRQ branch or the finest level (the cost estimate only)
NEAR_FRACTION = 0.6


def panel_costs(tcxi, tcx, sx, sw, hd):
    """Estimated work of each panel's near pairs (CSR tcxi 1-based, targets tcx)."""
    tcxi = np.asarray(tcxi, np.int64)
    npan = tcxi.size - 1
    sx = np.asarray(sx, np.float64).reshape(-1, 3)[:npan * hd]
    sw = np.asarray(sw, np.float64).ravel()[:npan * hd]
    cen = sx.reshape(npan, hd, 3).mean(1)
    rad = np.sqrt(sw.reshape(npan, hd).sum(1))
    tcx = np.asarray(tcx, np.float64).reshape(-1, 3)
    counts = np.diff(tcxi)
    pan = np.repeat(np.arange(npan), counts)
    d = np.linalg.norm(tcx[:tcxi[-1] - 1] - cen[pan], axis=1) / rad[pan]
    w = np.where(d < NEAR_FRACTION, RRQ_WEIGHT, 1.0)
    return np.bincount(pan, weights=w, minlength=npan)


def balanced_ranges(cost, world):
    """Contiguous panel ranges [lo, hi), one per rank in rank order, covering
    every panel, each near a 1/world share of the total cost."""
    cost = np.asarray(cost, np.float64)
    n = cost.size
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.concatenate([[0.0], np.cumsum(cost)])
    cuts = [0]
    for r in range(1, world):
        k = int(np.searchsorted(c, c[-1] * r / world))
        cuts.append(min(max(k, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def shard_inputs(rank, world, hd, sx, snx, sw, rts, rps, tcx, tcxrow, tcxi, ranges=None):
    """One rank's panels and near lists: panel arrays of its range, its CSR
    (1-based, from 1) and its rows renumbered relative to the range
    (row - lo hdim).  Returns (dict of arrays, (lo, hi), row_shift)."""
    tcxi = np.asarray(tcxi, np.int64)
    npan = tcxi.size - 1
    if ranges is None:
        ranges = balanced_ranges(panel_costs(tcxi, tcx, sx, sw, hd), world)
    a, b = ranges[rank]
    sl = slice(a * hd, b * hd)
    lo, hi = tcxi[a] - 1, tcxi[b] - 1
    shift = a * hd
    arr = lambda x, n: np.ascontiguousarray(np.asarray(x, np.float64).reshape(-1, n)[sl])
    S = dict(sx=arr(sx, 3), snx=arr(snx, 3), sw=np.ascontiguousarray(np.asarray(sw, np.float64).ravel()[sl]),
             rts=arr(rts, 3), rps=arr(rps, 3),
             tcx=np.ascontiguousarray(np.asarray(tcx, np.float64).reshape(-1, 3)[lo:hi]),
             tcxrow=np.ascontiguousarray(np.asarray(tcxrow, np.int64)[lo:hi] - shift),
             tcxi=np.ascontiguousarray(tcxi[a:b + 1] - lo))
    assert b <= npan
    return S, (a, b), shift


def getnearquad_shard(rank, world, npan, nterms, hd, nquad, sx, snx, sw, rts, rps, tcx, tcxrow, tcxi, orderff,
                      distff=1.4, iside=30, ranges=None):
    """This rank's part of qol_getnearquad_lap_rrq: (sparsei, sparsej,
    sparsevs, sparsevd) of its panel range with the single call's global
    numbering; the ranks' outputs concatenated in rank order are the single
    call's."""
    import qotential_b200 as qol
    S, (a, b), shift = shard_inputs(rank, world, hd, sx, snx, sw, rts, rps, tcx, tcxrow, tcxi, ranges)
    n = b - a
    si, sj, vs, vd, _ = qol.qol_getnearquad_lap_rrq(n, nterms, hd, nquad, n * hd, S["sx"], S["snx"], S["sw"],
                                                    S["rts"], S["rps"], S["tcxrow"].size, S["tcx"], S["tcxrow"],
                                                    S["tcxi"], orderff, distff, iside)
    return si + shift, sj + shift, vs, vd


def grf_near_sharded(npan, nterms, nquad, sx, snx, sw, rts, rps, ub, ubn, group=None, rank=None, world=None,
                     orderff=None, distff=1.4, iside=30, xbuf=None, near=None, far=None):
    """u = far field + near corrections of the GRF driver over all ranks of a
    torch.distributed process group, every node a target.  Rank r computes
    the far field of the r-th block of targets and the near corrections of
    the r-th cost-balanced panel range; one all-reduce (sum) of u.  ``near``
    and ``far`` stand in for qol_grf_near_range / qol_direct_farfield_range
    (same arguments and meaning) so the split can be exercised without a GPU.
    Returns (u, this rank's panel range)."""
    import torch
    import torch.distributed as dist
    import qotential_b200 as qol
    if group is not None or dist.is_initialized():
        rank = dist.get_rank(group) if rank is None else rank
        world = dist.get_world_size(group) if world is None else world
    rank = 0 if rank is None else rank
    world = 1 if world is None else world
    hd = nterms * (nterms + 1) // 2
    nsrc = npan * hd
    near = near or qol.qol_grf_near_range
    far = far or qol.qol_direct_farfield_range
    # near lists are computed inside the library; the cost estimate uses the
    # ball test's geometry on the host
    from qotential_b200 import geometry as G
    tcxi, _, tcx = G.near_lists(sx, sw, hd)
    ranges = balanced_ranges(panel_costs(tcxi, tcx, sx, sw, hd), world)
    plo, phi = ranges[rank]
    tlo, thi = (rank * nsrc) // world, ((rank + 1) * nsrc) // world
    u = np.zeros(nsrc)
    far(sx, snx, sw, ub, ubn, tlo, thi, u)
    u = near(npan, nterms, nquad, sx, snx, sw, rts, rps, ub, ubn, plo, phi, u=u,
             orderff=orderff, distff=distff, iside=iside, xbuf=xbuf)
    if world > 1:
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.as_tensor(u, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        u = t.cpu().numpy()
    return u, (plo, phi)
