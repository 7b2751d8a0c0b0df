"""The N > 1 path of bench.py on CPU: two gloo ranks, each building its panel
shard of the workload (bench.workload(rank, world): a cost-balanced panel
range, qotential_b200.sharding) and taking the step time as the maximum over
ranks (all_reduce MAX), as the GPU run does over NCCL.  The shards must
partition the single-rank workload exactly: panels, near pairs (rows shifted
back by each shard's row shift) and their CSR, in order."""
import os
import socket
import sys

import numpy as np
import pytest

ORDER = 4  # small panels: the shard logic does not depend on the order


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        W = bench.workload(rank, world, order=ORDER)
        sizes = torch.tensor([W["npan"], W["pairs"]], dtype=torch.int64)
        every = [torch.zeros_like(sizes) for _ in range(world)]
        dist.all_gather(every, sizes)
        ms = torch.tensor([10.0 * (rank + 1)])
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        dist.barrier()
        q.put((rank, [e.tolist() for e in every], float(ms.item()), (W["tcxrow"] + W["row_shift"]).tolist(),
               W["tcxi"].tolist(), W["sw"].tolist(), W["panel_range"]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_the_workload():
    import multiprocessing as mp
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
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
    full = bench.workload(0, 1, order=ORDER)
    every = res[0][1]
    assert every == res[1][1]
    assert sum(e[0] for e in every) == full["npan"] and sum(e[1] for e in every) == full["pairs"]
    assert res[0][2] == res[1][2] == 20.0  # the step time of the job: the slowest rank's
    rows = np.concatenate([np.asarray(res[r][3]) for r in range(2)])
    assert np.array_equal(rows, full["tcxrow"])
    sw = np.concatenate([np.asarray(res[r][5]) for r in range(2)])
    assert np.array_equal(sw, full["sw"])
    assert res[0][6][0] == 0 and res[0][6][1] == res[1][6][0] and res[1][6][1] == full["npan"]
    for r in range(2):  # each shard's CSR is one-based and covers its own pairs
        xi = np.asarray(res[r][4])
        assert xi[0] == 1 and xi[-1] == len(res[r][3]) + 1 and np.all(np.diff(xi) >= 0)
