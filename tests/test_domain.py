"""Single-scene domain decomposition of DFSPH and PBF (vtp/domain.py, csrc/domain.cu).

The decomposed run must reproduce the whole-scene run bit for bit: every owned row
sees the whole-scene neighbour list and neighbour values.  On CPU the stages are
the FP64 oracle's (the functions or_dfsph_step is made of), run as threads of one
process and as gloo ranks; on the GPU they are the library's, against the library
solver holding the whole scene.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from vtp import domain, scenes

FORCED = {"forceDivIterations": 3, "forceIncompIterations": 2}


def _whole_oracle(sc, steps, force=(0, 0)):
    from oracle import oracle as O
    o = O.OracleSolver(sc, force_div=force[0], force_inc=force[1])
    iters = []
    for _ in range(steps):
        o.step(1)
        iters.append((o.last.div_iters, o.last.inc_iters))
    fl = o.mat == 0
    return o.pos[fl], o.vel[fl], iters


# ----------------------------------------------------------------------------- host logic

def test_slab_plan_splits_fluid_evenly_and_owns_every_coordinate():
    a = domain.scene_arrays(scenes.dam_break("DFSPH", 3000, seed=11))
    for ranks in (1, 2, 3, 5):
        plan = domain.plan_slabs(a, ranks)
        assert plan.ranks == ranks
        size = a.config["DFSPH"]["Required"]["simSpaceSize"]
        assert plan.axis == int(np.argmax(size))
        own = plan.owner(a.fluid_pos[:, plan.axis])
        counts = np.bincount(own, minlength=ranks)
        assert counts.sum() == len(a.fluid_gid)
        assert counts.max() - counts.min() <= a.fluid_pos.shape[0] // 20 + 40   # lattice layers tie
        for k in range(ranks):
            lo, hi = plan.slab(k)
            x = a.fluid_pos[own == k, plan.axis]
            assert np.all(x >= lo) and np.all(x < hi)
    assert domain.plan_slabs(a, 4).ghost == pytest.approx(1.01 * a.h)


def test_scene_arrays_keep_attach_ids_and_reject_interleaved_ids():
    sc = scenes.colliding_blocks()
    a = domain.scene_arrays(sc)
    n0 = sc.objects[0].n
    assert a.fluid_gid.tolist() == list(range(sc.n_fluid))
    assert a.bnd_gid[0] == sc.n_fluid and not a.boundary_first
    assert a.fluid_obj[:n0].max() == 0 and a.fluid_obj[n0:].min() == 1
    assert a.obj_count.tolist() == [sc.objects[0].n, sc.objects[1].n]
    assert np.allclose(a.fluid_vel[:n0], [1.5, 0, 0]) and np.allclose(a.fluid_vel[n0:], [-1.5, 0, 0])
    sc.objects = [sc.objects[0], sc.objects[2], sc.objects[1]]   # fluid, box, fluid
    with pytest.raises(ValueError, match="fluid ids all below or all above"):
        domain.scene_arrays(sc)
    with pytest.raises(ValueError, match="DFSPH and PBF"):
        domain.scene_arrays(scenes.layered_mixture("IMMCT", 6, seed=1))


@pytest.mark.parametrize("ranks", [1, 2, 4])
def test_decomposed_oracle_with_the_adaptive_step(oracle_lib, ranks):
    """The CFL step (cfl 0.05 binds at 1.5 m/s: dt ~3.3e-4 against the 1 ms cap, changing every
    substep): one max all-reduce of the owned |v|^2 per substep gives every rank the
    whole-scene step, and the trajectories stay bit-identical."""
    from oracle import oracle as O
    sc = scenes.colliding_blocks()
    sc.config = dict(sc.config, B200={"cfl": 0.05})
    o = O.OracleSolver(sc)
    o.step(10)
    fl = o.mat == 0
    assert max(o.dts) < 1e-3 and len(set(o.dts)) > 3
    out = domain.run_local(sc, ranks, 10, make_stages=oracle_lib.DfsphDomainStages)
    assert np.array_equal(out["pos"], o.pos[fl]) and np.array_equal(out["vel"], o.vel[fl])


# ----------------------------------------------------------------------------- oracle stages

@pytest.mark.parametrize("ranks", [1, 2, 3])
@pytest.mark.parametrize("forced", [True, False])
def test_decomposed_oracle_equals_whole_scene_oracle(oracle_lib, ranks, forced):
    sc = scenes.dam_break("DFSPH", 3000, seed=11)
    force = (3, 2) if forced else (0, 0)
    pos, vel, iters = _whole_oracle(sc, 4, force)
    out = domain.run_local(sc, ranks, 4, make_stages=oracle_lib.DfsphDomainStages,
                           extra=FORCED if forced else None)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)
    assert sum(out["owned"]) == sc.n_fluid and min(out["owned"]) > 0


@pytest.mark.parametrize("ranks", [2, 4])
def test_decomposed_oracle_with_migration_tension_and_two_objects(oracle_lib, ranks):
    """Blocks thrown at each other across slab bounds: particles migrate every few substeps,
    ghosts carry surface normals for the tension pass, residuals are per fluid object."""
    sc = scenes.colliding_blocks()
    steps = 25
    pos, vel, iters = _whole_oracle(sc, steps)
    out = domain.run_local(sc, ranks, steps, make_stages=oracle_lib.DfsphDomainStages)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)
    plan = out["plan"]
    start = np.bincount(plan.owner(domain.scene_arrays(sc).fluid_pos[:, plan.axis]), minlength=ranks)
    assert out["owned"] != start.tolist()   # ownership moved with the particles


@pytest.mark.parametrize("speculate", [False, True])
def test_queued_solve_a_changes_nothing(oracle_lib, speculate):
    """The solve loop queues the next iteration's solve_a before it waits for the summed
    residual and drops it when the solve stops; without the queued pass the run is the same."""
    sc = scenes.colliding_blocks()
    pos, vel, iters = _whole_oracle(sc, 6)
    out = domain.run_local(sc, 2, 6, make_stages=oracle_lib.DfsphDomainStages, speculate=speculate)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


def _whole_oracle_fields(sc, steps):
    from oracle import oracle as O
    o = O.OracleSolver(sc)
    o.step(steps)
    fl = o.mat == 0
    return o.pos[fl], o.vel[fl]


@pytest.mark.parametrize("ranks", [1, 2, 3])
def test_decomposed_pbf_oracle_equals_whole_scene_oracle(oracle_lib, ranks):
    """PBF: lambda and the corrected positions / velocities go to the ghosts every constraint
    iteration; the external force is applied to owned and ghost rows alike."""
    sc = scenes.pbf_dam_break_m1()
    pos, vel = _whole_oracle_fields(sc, 4)
    out = domain.run_local(sc, ranks, 4, make_stages=oracle_lib.PbfDomainStages)
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)
    assert out["iters"] == [(4, 0)] * 4


@pytest.mark.parametrize("ranks", [2, 4])
def test_decomposed_pbf_oracle_follows_a_collapsing_column(oracle_lib, ranks):
    """80 substeps of a mass-1 dam break split across its height: the column collapses through
    the slab bounds (ownership moves), speeds reach ~5 m/s and ghosts are chosen with the
    external-force reach added."""
    sc = scenes.dam_break("PBF", 3000, seed=21, spacing=0.1)
    pos, vel = _whole_oracle_fields(sc, 80)
    out = domain.run_local(sc, ranks, 80, make_stages=oracle_lib.PbfDomainStages)
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)
    plan = out["plan"]
    start = np.bincount(plan.owner(domain.scene_arrays(sc).fluid_pos[:, plan.axis]), minlength=ranks)
    assert out["owned"] != start.tolist()


@pytest.mark.parametrize("kind", ["DFSPH", "PBF"])
def test_decomposed_oracle_with_an_empty_slab(oracle_lib, kind):
    """A slab that holds no fluid (nor boundary) and one that holds no owned fluid but ghosts:
    every stage runs on zero rows and the others are unaffected."""
    if kind == "DFSPH":
        sc, stages = scenes.dam_break("DFSPH", 3000, seed=11), oracle_lib.DfsphDomainStages
    else:
        sc, stages = scenes.dam_break("PBF", 3000, seed=21, spacing=0.1), oracle_lib.PbfDomainStages
    a = domain.scene_arrays(sc)
    ax = domain.plan_slabs(a, 2).axis
    lo = float(a.fluid_pos[:, ax].min())
    h = a.h
    # slab 0 far below everything, slab 1 a sliver of ghosts only, slab 2 the rest
    plan = domain.SlabPlan(ax, (lo - 50 * h, lo - 0.5 * h), domain.GHOST_MARGIN * h)
    pos, vel = _whole_oracle_fields(sc, 3)
    out = domain.run_local(sc, 3, 3, make_stages=stages, plan=plan)
    assert out["owned"][:2] == [0, 0]
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _gloo_rank(rank, world, port, steps, q, kind="DFSPH"):
    import datetime
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "vt-physics_b200")]
    import torch.distributed as dist
    from oracle import oracle as O
    from vtp import domain as D, scenes as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        sc = S.colliding_blocks() if kind == "DFSPH" else S.dam_break("PBF", 3000, seed=21, spacing=0.1)
        arrays = D.scene_arrays(sc)
        plan = D.plan_slabs(arrays, world)
        stages = O.DfsphDomainStages if kind == "DFSPH" else O.PbfDomainStages
        r = D.DomainRank(arrays, plan, D.TorchComm(), stages)
        r.step(steps)
        parts = [None] * world
        dist.all_gather_object(parts, r.state())
        if rank == 0:
            q.put(D.merge_states(arrays, parts))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kind", [(2, "DFSPH"), (3, "DFSPH"), (2, "PBF")])
def test_gloo_ranks_equal_whole_scene_oracle(oracle_lib, world, kind):
    steps = 12
    if kind == "DFSPH":
        pos, vel, iters = _whole_oracle(scenes.colliding_blocks(), steps)
    else:
        pos, vel = _whole_oracle_fields(scenes.dam_break("PBF", 3000, seed=21, spacing=0.1), steps)
        iters = [(4, 0)] * steps
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, steps, q, kind)) for r in range(world)]
    for p in procs:
        p.start()
    out = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


# ----------------------------------------------------------------------------- library stages

def _whole_library(sc, steps, extra):
    import vtp
    s = vtp.solver_from_scene(sc, extra=extra)
    assert s.initialize()
    iters = []
    for _ in range(steps):
        assert s.tickNsteps(1)
        st = s.stats()
        iters.append((st["last_div_iters"], st["last_incomp_iters"]))
    fl = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    pos, vel = s.get_field("pos")[fl], s.get_field("vel")[fl]
    s.destroy()
    return pos, vel, iters


@pytest.mark.gpu
@pytest.mark.parametrize("ranks", [1, 2, 4])
@pytest.mark.parametrize("halo", ["peer", "exchange"])
def test_library_domains_equal_whole_scene_library(vtp_gpu, ranks, halo):
    """Ghost values by peer stores (the owners' stage kernels write into the other slabs'
    ghost rows) and by pack / exchange / unpack give the whole-scene run."""
    sc = scenes.dam_break("DFSPH", 8000, seed=22)
    for extra in (FORCED, {}):
        pos, vel, iters = _whole_library(sc, 5, extra)
        out = domain.run_local(sc, ranks, 5, extra=extra, halo=halo)
        assert out["iters"] == iters
        assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
@pytest.mark.parametrize("halo", ["peer", "exchange"])
def test_library_domains_with_migration_tension_and_two_objects(vtp_gpu, halo):
    sc = scenes.colliding_blocks()
    pos, vel, iters = _whole_library(sc, 25, {})
    out = domain.run_local(sc, 4, 25, halo=halo)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
def test_library_domains_follow_the_decomposed_oracle(vtp_gpu, oracle_lib):
    """The library's decomposed run against the oracle's decomposed run: FP32 vs FP64 after
    three substeps with forced iterations (the bars of the whole-scene DFSPH parity test)."""
    sc = scenes.colliding_blocks()
    lib_out = domain.run_local(sc, 3, 3, extra=FORCED)
    ora = domain.run_local(sc, 3, 3, make_stages=oracle_lib.DfsphDomainStages, extra=FORCED)
    assert np.abs(lib_out["pos"] - ora["pos"]).max() < 1e-6
    assert np.abs(lib_out["vel"] - ora["vel"]).max() < 1e-4


def _ipc_rank(rank, world, port, steps, q, kind):
    """One process of the CUDA IPC test: the library's stages on cuda:0, peer-store halos
    linked through IPC handles, exchanges over gloo (device tensors staged through the host,
    the device synchronised before every collective, so a collective orders the ranks' kernels
    as NCCL's on the stream would)."""
    import datetime
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "vt-physics_b200")]
    import torch
    import torch.distributed as dist
    from vtp import domain as D, scenes as S

    class GlooDeviceComm(D.TorchComm):
        def exchange(self, sends, recvs):
            torch.cuda.synchronize()
            cs = {k: t.cpu() for k, t in sends.items()}
            cr = {k: torch.empty(t.shape, dtype=t.dtype) for k, t in recvs.items()}
            super().exchange(cs, cr)
            for k, t in cr.items():
                recvs[k].copy_(t)
            return recvs

        def counts(self, send_counts, device):
            return super().counts(send_counts, "cpu")

        def _reduce(self, t, op):
            torch.cuda.synchronize()
            c = t.cpu()
            dist.all_reduce(c, op=op)
            t.copy_(c)
            return t

        def allreduce_sum(self, t):
            return self._reduce(t, dist.ReduceOp.SUM)

        def allreduce_max(self, t):
            return self._reduce(t, dist.ReduceOp.MAX)

        def fence(self, device):
            torch.cuda.synchronize()
            dist.barrier()

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(0)
    r = None
    try:
        sc = S.colliding_blocks() if kind == "DFSPH" else S.dam_break("PBF", 8000, seed=21, spacing=0.1)
        arrays = D.scene_arrays(sc)
        plan = D.plan_slabs(arrays, world)
        with torch.cuda.stream(torch.cuda.Stream()):
            r = D.DomainRank(arrays, plan, GlooDeviceComm(), halo="peer")
            assert r.peer_mode
            r.step(steps)
            state = r.state()
        torch.cuda.synchronize()
        parts = [None] * world
        dist.all_gather_object(parts, state)
        if rank == 0:
            q.put(D.merge_states(arrays, parts))
    finally:
        # every rank's kernels (and their stores into the peers) have finished before any
        # worker, and the memory its peers map, is released
        torch.cuda.synchronize()
        dist.barrier()
        if r is not None:
            r.close()
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["DFSPH", "PBF"])
def test_two_processes_store_halos_through_cuda_ipc(vtp_gpu, kind):
    """Two ranks as two processes on one GPU, each worker's stage kernels storing the ghost
    values into the other process's buffers through CUDA IPC mappings (the multi-GPU path,
    without NVLink): the merged result equals the whole-scene library run bit for bit."""
    steps = 25 if kind == "DFSPH" else 40
    sc = scenes.colliding_blocks() if kind == "DFSPH" else scenes.dam_break("PBF", 8000, seed=21, spacing=0.1)
    pos, vel, iters = _whole_library(sc, steps, {})
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ipc_rank, args=(r, 2, port, steps, q, kind)) for r in range(2)]
    for p in procs:
        p.start()
    out = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    if kind == "DFSPH":
        assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
def test_dfsph_1m_in_four_slabs_equals_the_whole_scene(vtp_gpu):
    sc = scenes.dfsph_1m()
    pos, vel, iters = _whole_library(sc, 2, FORCED)
    out = domain.run_local(sc, 4, 2, extra=FORCED)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
@pytest.mark.parametrize("ranks", [1, 2, 4])
@pytest.mark.parametrize("halo", ["peer", "exchange"])
def test_library_pbf_domains_equal_whole_scene_library(vtp_gpu, ranks, halo):
    """PBF at mass-1 particles, the collapsing column over 40 substeps: the decomposed library
    run equals the whole-scene library run bit for bit, with the ghosts' lambda, positions and
    velocities stored by the owners' kernels or exchanged."""
    sc = scenes.dam_break("PBF", 8000, seed=21, spacing=0.1)
    pos, vel, _ = _whole_library(sc, 40, {})
    out = domain.run_local(sc, ranks, 40, halo=halo)
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["DFSPH", "PBF"])
def test_library_domains_with_an_empty_slab(vtp_gpu, kind):
    sc = scenes.dam_break("DFSPH", 8000, seed=22) if kind == "DFSPH" else \
        scenes.dam_break("PBF", 8000, seed=21, spacing=0.1)
    a = domain.scene_arrays(sc)
    ax = domain.plan_slabs(a, 2).axis
    lo = float(a.fluid_pos[:, ax].min())
    plan = domain.SlabPlan(ax, (lo - 50 * a.h, lo - 0.5 * a.h), domain.GHOST_MARGIN * a.h)
    pos, vel, _ = _whole_library(sc, 3, FORCED if kind == "DFSPH" else {})
    out = domain.run_local(sc, 3, 3, plan=plan, extra=FORCED if kind == "DFSPH" else None)
    assert out["owned"][:2] == [0, 0]
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
def test_dfsph_1m_in_eight_slabs_over_25_free_substeps(vtp_gpu):
    """The benchmark scene from rest, the residual deciding (up to 60 iterations a solve in
    the first substeps): eight slabs take the whole scene's iteration counts and end on its
    trajectory bit for bit."""
    sc = scenes.dfsph_1m()
    pos, vel, iters = _whole_library(sc, 25, {})
    out = domain.run_local(sc, 8, 25)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)


@pytest.mark.gpu
@pytest.mark.parametrize("halo", ["peer", "exchange"])
def test_library_domains_with_the_adaptive_step(vtp_gpu, halo):
    """The library's adaptive step computed on the device for the whole scene and on the host
    from the all-reduced |v|^2 for the slabs: the same steps, the same trajectory."""
    sc = scenes.colliding_blocks()
    extra = {"cfl": 0.05}
    pos, vel, iters = _whole_library(sc, 10, extra)
    out = domain.run_local(sc, 4, 10, extra=extra, halo=halo)
    assert out["iters"] == iters
    assert np.array_equal(out["pos"], pos) and np.array_equal(out["vel"], vel)
