"""Multi-rank logic on CPU ranks (gloo, world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from vtp.dist import lpt_assign


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "vt-physics_b200")]
    import torch.distributed as dist
    from vtp.dist import aggregate_throughput, lpt_assign
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # each rank "processes" its LPT share of 7 scenes; time = its cost
    costs = [5, 3, 8, 1, 4, 4, 2]
    mine = lpt_assign(costs, world)[rank]
    units, ms = aggregate_throughput(sum(costs[i] for i in mine) * 10, float(sum(costs[i] for i in mine)))
    q.put((rank, sorted(mine), units, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_assignment_balances_and_covers():
    costs = [5, 3, 8, 1, 4, 4, 2]
    parts = lpt_assign(costs, 2)
    assert sorted(i for p in parts for i in p) == list(range(7))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert lpt_assign(costs, 1) == [[2, 0, 4, 5, 1, 6, 3]]


def test_two_rank_aggregation_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shares = [r[1] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(7))
    # units summed over ranks, time = max over ranks, same on every rank
    assert res[0][2] == res[1][2] == 270.0
    assert res[0][3] == res[1][3] == max(sum([5, 3, 8, 1, 4, 4, 2][i] for i in s) for s in shares)
