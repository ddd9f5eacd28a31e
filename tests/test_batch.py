"""Scene batching: one solver advancing several independent scenes.

Each scene of a batched solver must produce exactly (bit for bit, iteration
counts included) what a solver holding that scene alone produces: the scenes
share kernel launches, never arithmetic.  CPU tests cover the host-side
validation of vtp_solver_add_scene.
"""
import json

import numpy as np
import pytest

import vtp
from vtp import scenes


def _pbf_mix():
    return [scenes.dam_break("PBF", n, seed=70 + k, gravity_y=g)
            for k, (n, g) in enumerate([(2000, -9.0), (5500, -11.5), (3100, -8.2), (8000, -10.0)])]


def _dfsph_mix():
    return [scenes.dam_break("DFSPH", n, seed=90 + k, gravity_y=g)
            for k, (n, g) in enumerate([(3000, -9.81), (6000, -8.5), (12000, -11.0)])]


# ---------------------------------------------------------------- CPU: host-side validation

def test_add_scene_requires_matching_shared_parameters():
    a, b = _pbf_mix()[:2]
    s = vtp.PBFSolver()
    assert s.setConfig(a.config)
    assert s.addScene(b.config) == 1
    bad = json.loads(json.dumps(b.config))
    bad["PBF"]["Required"]["timeStep"] = 0.002
    with pytest.raises(vtp.VtpError, match="timeStep"):
        s.addScene(bad)
    bad = json.loads(json.dumps(b.config))
    bad["PBF"]["Required"]["iterationNum"] = 7
    with pytest.raises(vtp.VtpError, match="iterationNum"):
        s.addScene(bad)
    s.destroy()


def test_add_scene_rejects_mixture_solvers_and_bad_scene_index():
    sc = scenes.layered_mixture("IMMCT", 8, seed=1)
    s = vtp.IMMCTSolver()
    assert s.setConfig(sc.config)
    with pytest.raises(vtp.VtpError, match="PBF and DFSPH"):
        s.addScene(sc.config)
    s.destroy()
    p = vtp.PBFSolver()
    a = _pbf_mix()[0]
    assert p.setConfig(a.config)
    o = vtp.Object(vtp.Particle_Common)
    o.pos = a.objects[0].pos
    o.getObjectComponentConfig()["epmMaterial"] = 0
    o.attachSpecificSolverObjectComponentConfig({"solverType": 0, "exportFlag": False, "velocityStart": [0, 0, 0],
                                                 "colorStart": [0, 0, 0]})
    assert not p.attachObject(o, scene=1)
    assert "scene index" in p.last_error
    p.destroy()


def test_set_config_drops_added_scenes():
    a, b = _pbf_mix()[:2]
    s = vtp.PBFSolver()
    s.setConfig(a.config)
    assert s.addScene(b.config) == 1
    s.setConfig(a.config)
    assert s.addScene(b.config) == 1
    s.destroy()


def test_batched_scene_generator():
    mix = scenes.batched_scenes()
    assert len(mix) == 64
    assert [m.solver for m in mix].count("PBF") == 48
    nf = np.array([m.n_fluid for m in mix])
    assert nf.min() >= 4000 * 0.8 and nf.max() <= 256000 * 1.1
    g = np.array([m.config[m.solver]["Optional"]["gravity"][1] for m in mix])
    assert np.all((g >= -12) & (g <= -8))


# ---------------------------------------------------------------- GPU: batched == alone

def _run_alone(sc, steps, extra):
    s = vtp.solver_from_scene(sc, extra)
    assert s.initialize()
    assert s.tickNsteps(steps), s.last_error
    out = (s.get_field("pos"), s.get_field("vel"), s.stats())
    s.destroy()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("kind,steps,extra", [
    ("PBF", 6, None),
    ("PBF", 6, {"rowLanes": 8}),
    ("DFSPH", 4, None),
    ("DFSPH", 3, {"deviceLoop": False}),
    ("DFSPH", 3, {"useGraphs": False, "blockSize": 64}),
])
def test_batched_scenes_match_each_scene_alone(vtp_gpu, kind, steps, extra):
    mix = _pbf_mix() if kind == "PBF" else _dfsph_mix()
    b, ranges = vtp.solver_from_scenes(mix, extra)
    assert b.initialize()
    assert b.tickNsteps(steps), b.last_error
    pos, vel = b.get_field("pos"), b.get_field("vel")
    for k, sc in enumerate(mix):
        lo, hi = ranges[k]
        p1, v1, st1 = _run_alone(sc, steps, extra)
        assert np.array_equal(pos[lo:hi], p1), f"scene {k} positions"
        assert np.array_equal(vel[lo:hi], v1), f"scene {k} velocities"
        if kind == "DFSPH":
            sk = b.scene_stats(k)
            assert (sk["total_div_iters"], sk["total_incomp_iters"]) == (st1["total_div_iters"],
                                                                          st1["total_incomp_iters"])
            assert sk["last_incomp_residual"] == st1["last_incomp_residual"]
    b.destroy()


@pytest.mark.gpu
def test_batched_neighbor_lists_are_per_scene(vtp_gpu):
    mix = _dfsph_mix()[:2]
    b, ranges = vtp.solver_from_scenes(mix)
    assert b.initialize() and b.tickNsteps(2)
    maxnbr = int(mix[0].config["DFSPH"]["Required"]["maxNeighborNum"])
    cnt, nb = b.get_neighbors(maxnbr)
    for k, sc in enumerate(mix):
        lo, hi = ranges[k]
        s = vtp.solver_from_scene(sc)
        assert s.initialize() and s.tickNsteps(2)
        c1, n1 = s.get_neighbors(maxnbr)
        s.destroy()
        sub = nb[lo:hi].astype(np.int64)
        sub = np.where(sub == 0xFFFFFFFF, -1, sub - lo)
        assert np.array_equal(cnt[lo:hi], c1)
        assert np.array_equal(sub, np.where(n1 == 0xFFFFFFFF, -1, n1.astype(np.int64)))
    b.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_batched_scenes_follow_the_fp64_oracle(vtp_gpu, oracle_lib, kind):
    """Each scene of a batch of the benchmark's mix (log-uniform sizes, per-scene gravity, PBF
    particles of mass 1) against the FP64 oracle advancing that scene alone, not only against
    the library's own per-scene runs: positions within 1e-5 and velocities within 1e-4 of the
    largest value after three substeps (DFSPH with forced iterations, so the comparison does
    not hinge on the stop test)."""
    mix = scenes.batched_scenes(count=8, n_pbf=4, n_min=2e3, n_max=1.6e4, pbf_spacing=0.1)
    part = [m for m in mix if m.solver == kind]
    force = (2, 3) if kind == "DFSPH" else (0, 0)
    extra = {"forceDivIterations": force[0], "forceIncompIterations": force[1]} if kind == "DFSPH" else None
    b, ranges = vtp.solver_from_scenes(part, extra)
    assert b.initialize()
    assert b.tickNsteps(3), b.last_error
    pos, vel = b.get_field("pos"), b.get_field("vel")
    b.destroy()
    for k, sc in enumerate(part):
        lo, hi = ranges[k]
        o = oracle_lib.OracleSolver(sc, force_div=force[0], force_inc=force[1])
        o.step(3)
        fm = np.concatenate([np.full(ob.n, ob.material == 0) for ob in sc.objects])
        req = sc.config[kind]["Required"]
        v_floor = 1e-3 * 2 * float(req["particleRadius"]) / float(req["timeStep"])
        dp = np.abs(pos[lo:hi][fm] - o.pos[fm]).max() / np.abs(o.pos[fm]).max()
        dv = np.abs(vel[lo:hi][fm] - o.vel[fm]).max() / max(np.abs(o.vel[fm]).max(), v_floor)
        print(f"{kind} scene {k} ({sc.n_fluid} fluid): pos {dp:.2e} vel {dv:.2e}")
        assert dp < 1e-5 and dv < 1e-4, f"scene {k}"


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_multi_range_frame_equals_per_range_calls(vtp_gpu, kind):
    """vtp_solver_step_state_ranges on the fluid objects of every scene of a batch (ranges
    separated by the scenes' boundaries, held back to back on the host) gives what
    set_state_range per range, tickNsteps and get_state_range per range give."""
    mix = _pbf_mix() if kind == "PBF" else _dfsph_mix()
    a, ranges = vtp.solver_from_scenes(mix)
    b, _ = vtp.solver_from_scenes(mix)
    assert a.initialize() and b.initialize() and a.tickNsteps(2) and b.tickNsteps(2)
    fl = []
    for sc, (lo, _) in zip(mix, ranges):
        start = lo
        for o in sc.objects:
            if o.material == 0:
                fl.append((start, o.n))
            start += o.n
    total = sum(c for _, c in fl)
    pa, va = vtp.HostBuffer((total, 3)), vtp.HostBuffer((total, 3))
    off = 0
    for first, count in fl:
        a.get_state_range_ptr(first, count, pa.ptr + 12 * off, va.ptr + 12 * off)
        off += count
    pb, vb = pa.array.copy(), va.array.copy()
    for frame in range(3):
        va.array[::7] *= 0.5
        vb[::7] *= 0.5
        assert a.step_state_ranges_ptr(fl, pa.ptr, va.ptr, 1, pa.ptr, va.ptr), a.last_error
        off = 0
        for first, count in fl:
            b.set_state_range_ptr(first, count, pb[off:off + count].ctypes.data, vb[off:off + count].ctypes.data)
            off += count
        assert b.tickNsteps(1), b.last_error
        off = 0
        for first, count in fl:
            pc, vc = np.empty((count, 3), np.float32), np.empty((count, 3), np.float32)
            b.get_state_range_ptr(first, count, pc.ctypes.data, vc.ctypes.data)
            pb[off:off + count], vb[off:off + count] = pc, vc
            off += count
        assert np.array_equal(pa.array, pb) and np.array_equal(va.array, vb), frame
    assert np.array_equal(a.get_field("pos"), b.get_field("pos"))
    a.strict = True
    with pytest.raises(vtp.VtpError, match="ascending and disjoint"):
        a.step_state_ranges_ptr(fl[::-1], pa.ptr, va.ptr, 1, pa.ptr, va.ptr)
    with pytest.raises(vtp.VtpError, match="ascending and disjoint"):
        a.step_state_ranges_ptr([fl[1], (fl[1][0], 1)], pa.ptr, va.ptr, 1, pa.ptr, va.ptr)   # overlapping
    pa.free()
    va.free()
    a.destroy()
    b.destroy()
