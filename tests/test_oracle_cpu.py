"""CPU oracle known-answer tests (test infrastructure checks)."""
import numpy as np
import pytest

from vtp import scenes


def brute_force_lists(pos, grid):
    """O(n^2) neighbour sets with the reference's FP32 membership test."""
    pos = pos.astype(np.float32)
    n = pos.shape[0]
    h = np.float32(grid.cell)
    out = []
    for i in range(n):
        d = (pos[i] - pos).astype(np.float32)
        d2 = np.float32(d[:, 2] * d[:, 2]) + np.float32(d[:, 1] * d[:, 1]) + np.float32(d[:, 0] * d[:, 0])
        r = np.sqrt(d2.astype(np.float64))  # only used for a far-from-boundary check below
        out.append(set(np.flatnonzero((r > 0) & (r <= float(h) * (1 - 1e-6))).tolist()))
    return out


def test_neighbor_sets_contain_all_clear_pairs(oracle_lib):
    rng = np.random.default_rng(3)
    pos = rng.random((600, 3)).astype(np.float32) * 0.3
    req = {"particleRadius": 0.01, "simSpaceLB": [-0.1] * 3, "simSpaceSize": [0.5] * 3, "maxNeighborNum": 600}
    grid = oracle_lib.make_grid(req)
    cnt, nb, ids, keys = oracle_lib.neighbors(pos, grid)
    bf = brute_force_lists(pos, grid)
    for i in range(pos.shape[0]):
        got = set(nb[i, 1:cnt[i]].tolist())
        assert nb[i, 0] == i
        assert bf[i] <= got                       # every pair clearly inside h is found
        d = np.linalg.norm(pos[list(got)].astype(np.float64) - pos[i], axis=1) if got else np.zeros(0)
        assert np.all(d <= 0.04 * (1 + 1e-6))      # nothing outside h is accepted
    # stable (cell, id) order
    order = np.lexsort((ids, keys))
    assert np.array_equal(order, np.arange(ids.size))


def test_lattice_has_33_neighbors_with_exact_arithmetic(oracle_lib):
    # spacing 0.25 and h = 0.5 are exact binary fractions: the 2-spacing pairs are exactly at h.
    p = np.stack(np.meshgrid(*[np.arange(9, dtype=np.float32) * 0.25] * 3, indexing="ij"), -1).reshape(-1, 3)
    req = {"particleRadius": 0.125, "simSpaceLB": [-1.0] * 3, "simSpaceSize": [5.0] * 3, "maxNeighborNum": 60}
    grid = oracle_lib.make_grid(req)
    cnt, nb, _, _ = oracle_lib.neighbors(p, grid)
    centre = int(np.flatnonzero(np.all(p == 1.0, axis=1))[0])
    assert cnt[centre] == 33


def test_max_neighbor_truncation(oracle_lib):
    p = np.stack(np.meshgrid(*[np.arange(9, dtype=np.float32) * 0.25] * 3, indexing="ij"), -1).reshape(-1, 3)
    req = {"particleRadius": 0.125, "simSpaceLB": [-1.0] * 3, "simSpaceSize": [5.0] * 3, "maxNeighborNum": 10}
    cnt, nb, _, _ = oracle_lib.neighbors(p, oracle_lib.make_grid(req))
    assert cnt.max() == 10 and np.all(nb[:, :1] != 0xFFFFFFFF)


def test_outside_particles_have_no_lists(oracle_lib):
    p = np.array([[0.1, 0.1, 0.1], [0.12, 0.1, 0.1], [5.0, 5.0, 5.0]], np.float32)
    req = {"particleRadius": 0.01, "simSpaceLB": [0.0] * 3, "simSpaceSize": [1.0] * 3, "maxNeighborNum": 8}
    cnt, nb, ids, _ = oracle_lib.neighbors(p, oracle_lib.make_grid(req))
    assert cnt.tolist() == [2, 2, 0] and ids.tolist() == [0, 1]


def test_oracle_is_thread_count_independent(oracle_lib):
    sc = scenes.dam_break("DFSPH", 3000, seed=4)
    outs = []
    for t in (1, 4):
        oracle_lib.set_threads(t)
        o = oracle_lib.OracleSolver(sc)
        o.step(2)
        outs.append((o.pos.copy(), o.vel.copy(), o.last.div_iters, o.last.inc_iters))
    oracle_lib.set_threads(0)
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2:] == outs[1][2:]


def test_dfsph_forced_iterations(oracle_lib):
    sc = scenes.dam_break("DFSPH", 3000, seed=5)
    o = oracle_lib.OracleSolver(sc, force_div=3, force_inc=2)
    o.step(1)
    assert (o.last.div_iters, o.last.inc_iters) == (3, 2)


def test_pbf_free_fall_without_neighbours(oracle_lib):
    # a single fluid particle far from everything falls ballistically: v = g t, x = x0 + sum v dt
    cfg = scenes.pbf_config(dt=0.01, r=0.01, lb=(-1, -1, -1), size=(2, 2, 2))
    sc = scenes.Scene("PBF", cfg, [scenes.SceneObject("p", np.array([[0.0, 0.5, 0.0]], np.float32), 0)])
    o = oracle_lib.OracleSolver(sc)
    o.step(3)
    g = -9.81
    assert o.vel[0, 1] == pytest.approx(3 * g * 0.01, rel=1e-6)
    assert o.pos[0, 1] == pytest.approx(0.5 + g * 0.01 * 0.01 * (1 + 2 + 3), rel=1e-6)


def test_standard_pbf_keeps_the_fluid_in_the_box(oracle_lib):
    # The reference's PBF constraint gradients leave out the particle mass (consistent only for
    # m = 1); at r = 0.01 (m = 8e-3) the correction is ~125x too weak and the dam-break fluid
    # passes through the 2-layer floor.  The standard formulation holds it.
    sc = scenes.pbf_dam_break()
    ref = oracle_lib.OracleSolver(sc)
    sc.config["B200"] = {"pbfFormulation": "standard", "pbfEpsilon": 100.0}
    std = oracle_lib.OracleSolver(sc)
    f = ref.mat == 0
    ref.step(90)
    std.step(90)
    assert (ref.pos[f, 1] < 0).sum() > 5000
    assert (std.pos[f, 1] < 0).sum() < 50
    assert abs(std.density[f].mean() / 1000.0 - 1.0) < 0.02


def test_oracle_adaptive_step_follows_the_cfl_rule(oracle_lib):
    """The oracle's adaptive step (the library's "cfl" extension) is
    min(timeStep, cfl * 2r / max|v_fluid|) on the substep's velocities."""
    from vtp import scenes
    sc = scenes.dam_break("DFSPH", 1500, seed=44)
    for o in sc.objects:
        if o.material == 0:
            o.velocity_start = (6.0, 0.0, 0.0)
    sc.config["B200"] = {"cfl": 0.4}
    o = oracle_lib.OracleSolver(sc, force_div=1, force_inc=1)
    fluid = o.mat == 0
    for _ in range(2):
        vmax = float(np.sqrt((o.vel[fluid] ** 2).sum(axis=1).max()))
        o.step(1)
        expect = min(1e-3, 0.4 * 0.01 / vmax)
        assert abs(o.dts[-1] - expect) <= 1e-5 * expect
    assert o.dts[0] < 1e-3
