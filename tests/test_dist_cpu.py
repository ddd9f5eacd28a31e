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


def _mix():
    from vtp import scenes
    return [scenes.dam_break("PBF", 700, seed=61), scenes.dam_break("DFSPH", 1200, seed=62),
            scenes.dam_break("PBF", 400, seed=63), scenes.dam_break("DFSPH", 600, seed=64),
            scenes.dam_break("PBF", 1000, seed=65)]


def _advance(scene, steps):
    """One scene of the mix through the FP64 CPU oracle: final state and iteration counts."""
    from oracle import oracle as O
    o = O.OracleSolver(scene)
    iters = []
    for _ in range(steps):
        o.step(1)
        if scene.solver == "DFSPH":
            iters.append((o.last.div_iters, o.last.inc_iters))
    return o.pos.copy(), o.vel.copy(), iters


def _shard_worker(rank, world, port, steps, q):
    import datetime
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "vt-physics_b200")]
    import torch.distributed as dist
    from vtp.dist import gather_scene_results, scene_share
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    mix = _mix()
    mine = scene_share(mix, world, rank)
    local = {k: _advance(mix[k], steps) for k in mine}
    merged = gather_scene_results(local)
    q.put((rank, mine, merged if rank == 0 else sorted(merged)))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_matches_single_rank_run():
    """Each of two gloo ranks advances its LPT share of a small batched mix
    (3 PBF + 2 DFSPH scenes) through the FP64 CPU oracle; the gathered
    per-scene results equal a single-rank run of every scene."""
    import numpy as np
    steps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, steps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(2)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mix = _mix()
    shares = [r[1] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(len(mix))) and shares[0] and shares[1]
    merged = res[0][2]
    assert sorted(merged) == res[1][2] == list(range(len(mix)))
    for k, sc in enumerate(mix):
        pos, vel, iters = _advance(sc, steps)
        gp, gv, gi = merged[k]
        assert gi == iters
        assert np.allclose(gp, pos, rtol=0, atol=1e-12) and np.allclose(gv, vel, rtol=0, atol=1e-12)
