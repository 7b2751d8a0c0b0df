"""The multi-GPU split of the near-field path (qotential_b200.sharding) on
CPU: cost-balanced contiguous panel ranges, per-rank inputs renumbered so the
ranks' outputs concatenate to the single call's, and the GRF split's one
all-reduce of u over two gloo ranks, with stand-ins for the two GPU range
entry points that record which panels and targets each rank was given."""
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_balanced_ranges_partition_and_balance():
    from qotential_b200 import sharding as S
    rng = np.random.default_rng(0)
    cost = rng.uniform(1.0, 10.0, 1000)
    for world in (1, 2, 3, 8):
        r = S.balanced_ranges(cost, world)
        assert r[0][0] == 0 and r[-1][1] == cost.size
        assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
        shares = [cost[a:b].sum() for a, b in r]
        assert max(shares) - min(shares) <= 2 * cost.max() + 1e-9


def test_shard_inputs_concatenate_to_the_whole():
    from qotential_b200 import geometry as G
    from qotential_b200 import sharding as S
    nterms = 4
    hd = nterms * (nterms + 1) // 2
    P = G.panels(G.torus(), 6, 12, nterms, split=False)
    T = np.concatenate([P["sx"], G.off_surface_targets(P, 40, 3, hd)])
    tcxi, tcxrow, tcx = G.near_lists(P["sx"], P["sw"], hd, targets=T)
    npan = P["sw"].size // hd
    cost = S.panel_costs(tcxi, tcx, P["sx"], P["sw"], hd)
    assert cost.shape == (npan,) and np.all(cost >= np.diff(tcxi))  # at least one unit a pair
    rows, sws = [], []
    for rank in range(3):
        Sh, (a, b), shift = S.shard_inputs(rank, 3, hd, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], tcx,
                                           tcxrow, tcxi)
        assert shift == a * hd and Sh["tcxi"][0] == 1 and Sh["tcxi"][-1] == Sh["tcxrow"].size + 1
        # rows of the range's own nodes are 1..(b - a) hd in the shard's numbering
        own = (Sh["tcxrow"] >= 1) & (Sh["tcxrow"] <= (b - a) * hd)
        assert np.array_equal(own, (Sh["tcxrow"] + shift > a * hd) & (Sh["tcxrow"] + shift <= b * hd))
        rows.append(Sh["tcxrow"] + shift)
        sws.append(Sh["sw"])
    assert np.array_equal(np.concatenate(rows), tcxrow)
    assert np.array_equal(np.concatenate(sws), P["sw"])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _grf_rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    from qotential_b200 import geometry as G
    from qotential_b200 import sharding as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nterms = 4
        hd = nterms * (nterms + 1) // 2
        P = G.panels(G.torus(), 6, 12, nterms, split=False)
        npan = P["sw"].size // hd
        ub = np.cos(P["sx"][:, 0]); ubn = np.sin(P["sx"][:, 1])
        seen = {}

        def far(sx, snx, sw, ub_, ubn_, tlo, thi, u):  # stand-in: target i gets 1000 + i
            seen["far"] = (tlo, thi)
            u[tlo:thi] = 1000.0 + np.arange(tlo, thi)

        def near(npan_, nterms_, nquad, sx, snx, sw, rts, rps, ub_, ubn_, plo, phi, u=None, **kw):
            seen["near"] = (plo, phi)  # stand-in: panel k adds k to the targets of its nodes
            u = u.copy()
            for k in range(plo, phi):
                u[k * hd:(k + 1) * hd] += k
            return u

        u, rng_ = S.grf_near_sharded(npan, nterms, nterms + 2, P["sx"], P["snx"], P["sw"], P["rts"], P["rps"], ub,
                                     ubn, near=near, far=far)
        q.put((rank, u.tolist(), seen["far"], seen["near"], rng_))
    finally:
        dist.destroy_process_group()


def test_grf_split_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grf_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(2):
            r = q.get(timeout=300)
            res[r[0]] = r
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    nterms = 4
    hd = nterms * (nterms + 1) // 2
    npan = 2 * 6 * 12
    nsrc = npan * hd
    want = 1000.0 + np.arange(nsrc) + np.repeat(np.arange(npan), hd)
    for r in range(2):
        assert np.array_equal(np.asarray(res[r][1]), want)  # every rank holds the reduced u
    assert res[0][2] == (0, nsrc // 2) and res[1][2] == (nsrc // 2, nsrc)
    assert res[0][3][0] == 0 and res[0][3][1] == res[1][3][0] and res[1][3][1] == npan
    assert tuple(res[0][3]) == tuple(res[0][4])
