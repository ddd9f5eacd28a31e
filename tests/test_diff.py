"""Differentiable PBF: the sm_100a adjoint against the FP64 CPU adjoint and FP64
central finite differences, both with the neighbour lists frozen to the ones the
GPU forward built (tolerance: 1e-3 relative, the differentiable-PBF target)."""
import numpy as np
import pytest

from vtp import scenes

TOL = 1e-3
TARGET = np.array([0.8, 0.2, 0.6])


def small_case(seed=7):
    sc = scenes.dam_break("PBF", 400, seed=seed)
    f = sc.objects[0]
    rng = np.random.default_rng(seed)
    f.velocity = rng.normal(0.0, 0.1, (f.n, 3)).astype(np.float32)
    return sc


def loss_grad(pos, mask, target):
    m = pos[mask].astype(np.float64).mean(0)
    g = np.zeros(pos.shape, np.float64)
    g[mask] = 2.0 * (m - target) / mask.sum()
    return float(((m - target) ** 2).sum()), g


# ---------------------------------------------------------------- CPU: the FP64 adjoint itself

def test_oracle_adjoint_matches_finite_differences(oracle_lib):
    sc = small_case(3)
    d = oracle_lib.PbfDiff(sc)
    f = d.fluid
    x0, v0 = d.base.pos.copy(), d.base.vel.copy()
    T = 6
    target = TARGET * 0.1
    xT, _, states, used = d.rollout(x0, v0, T, record=True)
    _, xbar = loss_grad(xT, f, target)
    gx, gv, gk = d.adjoint(states, used, xbar, np.zeros_like(xbar))
    rng = np.random.default_rng(11)
    k0 = d.p.xsph_k
    for _ in range(3):
        dv = np.zeros_like(v0)
        dv[f] = rng.normal(size=(f.sum(), 3))
        dk = rng.normal()
        nrm = np.sqrt((dv ** 2).sum() + dk * dk)
        dv, dk = dv / nrm, dk / nrm

        def L(s):
            d.p.xsph_k = k0 + s * dk
            x, _, _, _ = d.rollout(x0, v0 + s * dv, T, lists=used)
            d.p.xsph_k = k0
            return loss_grad(x, f, target)[0]
        fd = (L(1e-4) - L(-1e-4)) / 2e-4
        ad = float((gv * dv).sum() + gk * dk)
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-14


# ---------------------------------------------------------------- GPU: the library's adjoint

@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [1, 8])
def test_gpu_adjoint_matches_fp64_adjoint_and_fd(vtp_gpu, oracle_lib, lanes):
    from vtp import diff
    sc = small_case(7)
    mask = diff.fluid_mask(sc)
    T, every = 10, 4
    s = diff.pbf_solver(sc, extra={"rowLanes": lanes})
    maxnbr = int(sc.config["PBF"]["Required"]["maxNeighborNum"])
    diff.diff_forward(s, T, every, keep_lists=True)
    lists = [diff.diff_lists(s, t, maxnbr) for t in range(T)]
    target = TARGET * 0.1
    _, dl = loss_grad(s.get_field("pos"), mask, target)
    gx, gv, gk = diff.diff_backward(s, dl.astype(np.float32), None)
    s.destroy()

    d = oracle_lib.PbfDiff(sc)
    x0, v0 = d.base.pos.copy(), d.base.vel.copy()
    xT, _, states, used = d.rollout(x0, v0, T, lists=lists, record=True)
    _, xbar = loss_grad(xT, mask, target)
    ox, ov, ok = d.adjoint(states, used, xbar, np.zeros_like(xbar))
    rel_v = np.linalg.norm(gv[mask] - ov[mask]) / np.linalg.norm(ov[mask])
    rel_x = np.linalg.norm(gx[mask] - ox[mask]) / np.linalg.norm(ox[mask])
    print(f"adjoint vs FP64 adjoint: vel {rel_v:.2e} pos {rel_x:.2e} k {abs(gk - ok) / abs(ok):.2e}")
    assert rel_v < TOL and rel_x < TOL
    assert abs(gk - ok) <= TOL * abs(ok)

    rng = np.random.default_rng(5006)
    k0 = d.p.xsph_k
    for _ in range(4):
        dv = np.zeros_like(v0)
        dv[mask] = rng.normal(size=(mask.sum(), 3))
        dk = rng.normal()
        nrm = np.sqrt((dv ** 2).sum() + dk * dk)
        dv, dk = dv / nrm, dk / nrm

        def L(e):
            d.p.xsph_k = k0 + e * dk
            x, _, _, _ = d.rollout(x0, v0 + e * dv, T, lists=lists)
            d.p.xsph_k = k0
            return loss_grad(x, mask, target)[0]
        fd = (L(1e-4) - L(-1e-4)) / 2e-4
        ad = float((gv.astype(np.float64) * dv).sum() + gk * dk)
        print(f"directional: fd {fd:.6e} adjoint {ad:.6e}")
        assert abs(ad - fd) <= TOL * abs(fd)


@pytest.mark.gpu
def test_gpu_adjoint_same_with_and_without_programmatic_launch(vtp_gpu):
    """Programmatic dependent launch ("pdl") between the forward and adjoint
    kernels changes when blocks start, not what they read: the forward state
    and every gradient are bit-identical with it on and off."""
    from vtp import diff
    sc = small_case(10)
    mask = diff.fluid_mask(sc)
    out = []
    for pdl in (True, False):
        s = diff.pbf_solver(sc, extra={"pdl": pdl})
        diff.diff_forward(s, 8, 3)
        pos = s.get_field("pos")
        _, dl = loss_grad(pos, mask, TARGET)
        out.append((pos, diff.diff_backward(s, dl.astype(np.float32), None)))
        s.destroy()
    (pa, (xa, va, ka)), (pb, (xb, vb, kb)) = out
    assert np.array_equal(pa, pb)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb) and ka == kb


@pytest.mark.gpu
def test_gpu_adjoint_independent_of_checkpoint_interval(vtp_gpu):
    from vtp import diff
    sc = small_case(9)
    mask = diff.fluid_mask(sc)
    out = []
    for every in (1, 3, 8):
        s = diff.pbf_solver(sc)
        diff.diff_forward(s, 8, every)
        pos = s.get_field("pos")
        _, dl = loss_grad(pos, mask, TARGET)
        out.append((pos, diff.diff_backward(s, dl.astype(np.float32), None)))
        # the solver is back at the forward's final state
        assert np.array_equal(s.get_field("pos"), pos)
        s.destroy()
    for pos, (gx, gv, gk) in out[1:]:
        assert np.array_equal(pos, out[0][0])
        assert np.array_equal(gv, out[0][1][1]) and np.array_equal(gx, out[0][1][0]) and gk == out[0][1][2]


@pytest.mark.gpu
def test_gpu_adjoint_same_with_segment_graphs_and_reused_buffers(vtp_gpu):
    """The backward replays each full checkpoint segment as captured graphs
    ("useGraphs", default on), the forward keeps as many segments' tapes
    resident as "tapeBudgetMB" allows (the backward recomputes the others), and
    a rollout of the same shape as the last reuses its checkpoints and tapes:
    none of it changes the forward state or any gradient, bit for bit."""
    from vtp import diff
    sc = small_case(13)
    mask = diff.fluid_mask(sc)
    out = []
    # tapeBudgetMB 0: one resident tape (the forward's last segment; the other is recomputed);
    # the default budget holds both segments' tapes (no recompute)
    for graphs, budget in ((True, None), (False, None), (True, 0), (False, 0)):
        extra = {"useGraphs": graphs}
        if budget is not None:
            extra["tapeBudgetMB"] = budget
        s = diff.pbf_solver(sc, extra=extra)
        x0, v0 = s.get_field("pos"), s.get_field("vel")
        runs = []
        for _ in range(2):   # the second rollout restarts from the initial state on reused buffers
            s.set_field("pos", x0)
            s.set_field("vel", v0)
            diff.diff_forward(s, 8, 4)
            pos = s.get_field("pos")
            _, dl = loss_grad(pos, mask, TARGET)
            runs.append((pos,) + tuple(diff.diff_backward(s, dl.astype(np.float32), None)))
        s.destroy()
        for a, b in zip(runs[0], runs[1]):
            assert np.array_equal(a, b)
        out.append(runs[0])
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_torch_autograd_wrapper(vtp_gpu):
    import torch
    from vtp import diff
    sc = small_case(12)
    f = sc.objects[0]
    roll = diff.make_rollout(sc, steps=6, checkpoint_every=3)
    v0 = torch.tensor(f.velocity, requires_grad=True)
    k = torch.tensor(0.01, requires_grad=True)
    x = roll(v0, k)
    loss = ((x.double().mean(0) - torch.tensor(TARGET)) ** 2).sum()
    loss.backward()
    s = diff.pbf_solver(sc, f.velocity, 0.01)
    diff.diff_forward(s, 6, 3)
    mask = diff.fluid_mask(sc)
    _, dl = loss_grad(s.get_field("pos"), mask, TARGET)
    _, gv, gk = diff.diff_backward(s, dl.astype(np.float32), None)
    s.destroy()
    assert np.allclose(v0.grad.numpy(), gv[mask], rtol=1e-5, atol=1e-12)
    assert k.grad.item() == pytest.approx(gk, rel=1e-5)


# ---------------------------------------------------------------- DFSPH pressure solve as an operator

def _dfsph_case(vtp, seed=4):
    sc = scenes.dam_break("DFSPH", 3000, seed=seed)
    s = vtp.solver_from_scene(sc)
    assert s.initialize() and s.tickNsteps(3)
    return sc, s


def test_oracle_dfsph_solve_adjoint_matches_finite_differences(oracle_lib):
    sc = scenes.dam_break("DFSPH", 3000, seed=4)
    o = oracle_lib.OracleSolver(sc)
    o.step(3)
    cnt, nb, _, _ = oracle_lib.neighbors(o.pos.astype(np.float32), o.grid)
    f = o.mat == 0
    rng = np.random.default_rng(1)
    v = o.vel.copy()
    v[f] += rng.normal(0, 0.05, (f.sum(), 3))
    u = np.zeros_like(v)
    u[f] = rng.normal(size=(f.sum(), 3))
    _, vb = oracle_lib.dfsph_solve_op(o, cnt, nb, 5, v, u)
    for _ in range(2):
        d = np.zeros_like(v)
        d[f] = rng.normal(size=(f.sum(), 3))
        fp, _ = oracle_lib.dfsph_solve_op(o, cnt, nb, 5, v + 1e-6 * d)
        fm, _ = oracle_lib.dfsph_solve_op(o, cnt, nb, 5, v - 1e-6 * d)
        fd = float(((fp - fm) / 2e-6 * u).sum())
        assert abs(float((vb * d).sum()) - fd) <= 1e-7 * abs(fd)


@pytest.mark.gpu
def test_gpu_dfsph_solve_vjp_matches_fp64_and_fd(vtp_gpu, oracle_lib):
    from vtp import diff
    sc, s = _dfsph_case(vtp_gpu)
    n = s.counts()["total"]
    mask = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    rng = np.random.default_rng(2)
    v = s.get_field("vel")
    v[mask] += rng.normal(0, 0.05, (mask.sum(), 3)).astype(np.float32)
    iters = 5
    vo, it = diff.dfsph_solve(s, v, 0, iters)
    assert it == iters
    u = np.zeros((n, 3), np.float32)
    u[mask] = rng.normal(size=(mask.sum(), 3))
    vb = diff.dfsph_solve_vjp(s, u)
    # FP64 oracle operator on the same positions, volumes and lists
    o = oracle_lib.OracleSolver(sc)
    o.pos = s.get_field("pos").astype(np.float64)
    o.vol = s.get_field("volume").astype(np.float64)
    cnt, nb = s.get_neighbors(int(sc.config["DFSPH"]["Required"]["maxNeighborNum"]))
    ov, ob = oracle_lib.dfsph_solve_op(o, cnt, nb, iters, v.astype(np.float64), u.astype(np.float64))
    dv0 = np.linalg.norm(ov[mask] - v[mask])
    rel_out = np.linalg.norm(vo[mask] - ov[mask]) / dv0
    rel_vjp = np.linalg.norm(vb[mask] - ob[mask]) / np.linalg.norm(ob[mask])
    print(f"solve output vs FP64 (relative to the solve's change) {rel_out:.2e}, vjp {rel_vjp:.2e}")
    assert rel_out < TOL and rel_vjp < TOL
    # directional derivatives: FP64 central differences of the oracle operator
    for _ in range(3):
        d = np.zeros((n, 3), np.float64)
        d[mask] = rng.normal(size=(mask.sum(), 3))
        fp, _ = oracle_lib.dfsph_solve_op(o, cnt, nb, iters, v.astype(np.float64) + 1e-6 * d)
        fm, _ = oracle_lib.dfsph_solve_op(o, cnt, nb, iters, v.astype(np.float64) - 1e-6 * d)
        fd = float(((fp - fm) / 2e-6 * u).sum())
        ad = float((vb.astype(np.float64) * d).sum())
        print(f"directional: fd {fd:.6e} vjp {ad:.6e}")
        assert abs(ad - fd) <= TOL * abs(fd)
    s.destroy()


@pytest.mark.gpu
def test_gpu_dfsph_solve_leaves_solver_state_unchanged(vtp_gpu):
    from vtp import diff
    sc, a = _dfsph_case(vtp_gpu, seed=6)
    b = vtp_gpu.solver_from_scene(sc)
    assert b.initialize() and b.tickNsteps(3)
    diff.dfsph_solve(a, a.get_field("vel") * 1.1, 1)
    assert a.tickNsteps(2) and b.tickNsteps(2)
    assert np.array_equal(a.get_field("pos"), b.get_field("pos"))
    assert np.array_equal(a.get_field("vel"), b.get_field("vel"))
    with pytest.raises(vtp_gpu.VtpError, match="advanced"):
        diff.dfsph_solve_vjp(a, np.zeros((a.counts()["total"], 3), np.float32))
    a.destroy()
    b.destroy()
