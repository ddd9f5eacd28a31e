"""Differentiable DFSPH rollout: the substep's hand-written adjoint (lists frozen per
substep, pressure-solve iteration counts and clamp patterns of the forward held fixed).

CPU: the FP64 adjoint of the oracle against FP64 central differences of the oracle's
frozen-list rollout.  GPU: the library's adjoint against the FP64 adjoint of the same
discrete map and against FP64 central differences, with the GPU's lists and iteration
counts (tolerance 1e-3 relative, the differentiable-rollout target)."""
import numpy as np
import pytest

from vtp import scenes

TOL = 1e-3


def _linear_loss(shape, mask, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=shape) * mask[:, None]
    b = rng.normal(size=shape) * mask[:, None]
    return a, b


# ---------------------------------------------------------------- CPU: the FP64 adjoint itself

def test_oracle_dfsph_rollout_adjoint_matches_finite_differences(oracle_lib):
    sc = scenes.dam_break("DFSPH", 800, seed=7)
    # viscosity 1e-2 instead of the scenes' 1e-6, so that the viscosity term's share of the
    # gradient is far above the FP64 rounding of the central differences
    d = oracle_lib.DfsphDiff(sc, viscosity=1e-2)
    f = d.fluid
    rng = np.random.default_rng(1)
    x0, v0 = d.base.pos.copy(), d.base.vel.copy()
    v0[f] += rng.normal(0, 0.1, (f.sum(), 3))
    T, iters = 3, [(3, 2)] * 3
    _, _, states, used = d.rollout(x0, v0, T, iters, record=True)
    lists = [(u[0], u[1]) for u in used]
    A, B = _linear_loss(x0.shape, f, 2)

    def L(x, v, vis=None):
        vis0 = d.p.vis
        if vis is not None:
            d.p.vis = vis
        xT, vT, _, _ = d.rollout(x, v, T, iters, lists=lists)
        d.p.vis = vis0
        return float((A * xT).sum() + (B * vT).sum())

    gx, gv, gvis = d.adjoint(states, used, A, B)
    # eps 1e-8: a position step of 1e-7 already moves some particles across a clamp
    # (delta = max(delta, 0)) of the pressure solves, where the map has a kink
    for _ in range(2):
        dx = rng.normal(size=x0.shape) * f[:, None]
        dv = rng.normal(size=x0.shape) * f[:, None]
        fd = (L(x0 + 1e-8 * dx, v0) - L(x0 - 1e-8 * dx, v0)) / 2e-8
        assert abs(float((gx * dx).sum()) - fd) <= 1e-6 * abs(fd)
        fd = (L(x0, v0 + 1e-7 * dv) - L(x0, v0 - 1e-7 * dv)) / 2e-7
        assert abs(float((gv * dv).sum()) - fd) <= 1e-6 * abs(fd)
    e = d.p.vis * 1e-4
    fd = (L(x0, v0, d.p.vis + e) - L(x0, v0, d.p.vis - e)) / (2 * e)
    assert abs(gvis - fd) <= 1e-6 * abs(fd)


# ---------------------------------------------------------------- GPU: the library's adjoint

T_GPU, EVERY = 4, 2


def gpu_case(seed=5, n=3000, vis=1e-2, threshold=None):
    sc = scenes.dam_break("DFSPH", n, seed=seed)
    sc.config["DFSPH"]["Required"]["fPartRestViscosity"] = vis
    if threshold is not None:
        sc.config["DFSPH"]["Required"]["divFreeThreshold"] = threshold
        sc.config["DFSPH"]["Required"]["incompThreshold"] = threshold
    f = sc.objects[0]
    rng = np.random.default_rng(seed)
    f.velocity = rng.normal(0.0, 0.1, (f.n, 3)).astype(np.float32)
    return sc


def _rollout_gradients(vtp, sc, A, B, keep_lists, extra=None):
    from vtp import diff
    s = vtp.solver_from_scene(sc, extra=extra)
    assert s.initialize()
    x0, v0 = s.get_field("pos"), s.get_field("vel")
    diff.diff_forward(s, T_GPU, EVERY, keep_lists=keep_lists)
    out = diff.diff_backward(s, A.astype(np.float32), B.astype(np.float32))
    return s, x0, v0, out


@pytest.mark.gpu
@pytest.mark.parametrize("threshold", [None, 1e-5])
def test_gpu_dfsph_rollout_adjoint_matches_fp64_adjoint_and_fd(vtp_gpu, oracle_lib, threshold):
    """threshold 1e-5 makes the solves run many more iterations than the recording's first
    speculative chunk, so the segment is restored from its checkpoint and recorded again with
    host-driven solves; the forward must still equal ordinary substeps bit for bit."""
    from vtp import diff
    sc = gpu_case(threshold=threshold)
    mask = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    n = mask.size
    A, B = _linear_loss((n, 3), mask, 3)
    s, x0, v0, (gx, gv, gvis) = _rollout_gradients(vtp_gpu, sc, A, B, keep_lists=True)
    M = int(sc.config["DFSPH"]["Required"]["maxNeighborNum"])
    lists = [diff.diff_lists(s, t, M) for t in range(T_GPU)]
    iters = [diff.diff_iterations(s, t) for t in range(T_GPU)]
    print("iterations per substep", iters)
    assert all(1 <= a <= 101 and 1 <= b <= 101 for a, b in iters)
    # the recording forward advanced the solver exactly as ordinary substeps do
    b = vtp_gpu.solver_from_scene(sc)
    assert b.initialize() and b.tickNsteps(T_GPU)
    assert np.array_equal(s.get_field("pos"), b.get_field("pos"))
    assert np.array_equal(s.get_field("vel"), b.get_field("vel"))
    b.destroy()
    # FP64 adjoint of the same discrete map: the GPU's lists and iteration counts
    d = oracle_lib.DfsphDiff(sc)
    xd, vd = x0.astype(np.float64), v0.astype(np.float64)
    _, _, states, used = d.rollout(xd, vd, T_GPU, iters, lists=lists, record=True)
    ox, ov, ovis = d.adjoint(states, used, A, B)
    ex = np.linalg.norm(gx[mask] - ox[mask]) / np.linalg.norm(ox[mask])
    ev = np.linalg.norm(gv[mask] - ov[mask]) / np.linalg.norm(ov[mask])
    evis = abs(gvis - ovis) / abs(ovis)
    print(f"GPU vs FP64 adjoint: positions {ex:.2e}, velocities {ev:.2e}, viscosity {evis:.2e}")
    assert ex < TOL and ev < TOL and evis < TOL

    def L(x, v):
        xT, vT, _, _ = d.rollout(x, v, T_GPU, iters, lists=lists)
        return float((A * xT).sum() + (B * vT).sum())

    rng = np.random.default_rng(8)
    for _ in range(2):
        dv = rng.normal(size=(n, 3)) * mask[:, None]
        fd = (L(xd, vd + 1e-7 * dv) - L(xd, vd - 1e-7 * dv)) / 2e-7
        ad = float((gv.astype(np.float64) * dv).sum())
        print(f"velocity direction: fd {fd:.6e} adjoint {ad:.6e}")
        assert abs(ad - fd) <= TOL * abs(fd)
        dx = rng.normal(size=(n, 3)) * mask[:, None]
        fd = (L(xd + 1e-8 * dx, vd) - L(xd - 1e-8 * dx, vd)) / 2e-8
        ad = float((gx.astype(np.float64) * dx).sum())
        print(f"position direction: fd {fd:.6e} adjoint {ad:.6e}")
        assert abs(ad - fd) <= TOL * abs(fd)
    s.destroy()


@pytest.mark.gpu
def test_gpu_dfsph_rollout_adjoint_same_with_recomputed_segments(vtp_gpu):
    """One resident tape (tapeBudgetMB 0): every earlier segment is recomputed from its
    checkpoint, and the gradient is the bits of the all-resident run."""
    sc = gpu_case(seed=6)
    mask = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    A, B = _linear_loss((mask.size, 3), mask, 4)
    s1, _, _, g1 = _rollout_gradients(vtp_gpu, sc, A, B, keep_lists=True)
    s2, _, _, g2 = _rollout_gradients(vtp_gpu, sc, A, B, keep_lists=False, extra={"tapeBudgetMB": 0})
    assert np.array_equal(g1[0], g2[0]) and np.array_equal(g1[1], g2[1]) and g1[2] == g2[2]
    assert np.array_equal(s1.get_field("pos"), s2.get_field("pos"))
    for s in (s1, s2):
        s.destroy()


@pytest.mark.gpu
def test_gpu_dfsph_rollout_rejects_unsupported_settings(vtp_gpu):
    from vtp import diff
    sc = gpu_case(seed=7, n=1000)
    s = vtp_gpu.solver_from_scene(sc)
    with pytest.raises(vtp_gpu.VtpError, match="before diff_forward"):
        diff.diff_backward(s, np.zeros((s.counts()["total"], 3), np.float32))
    s.destroy()
    s = vtp_gpu.solver_from_scene(sc, extra={"cfl": 0.4})
    with pytest.raises(vtp_gpu.VtpError, match="fixed time step"):
        diff.diff_forward(s, 2, 1)
    s.destroy()
    sc.config["DFSPH"]["Required"]["surfaceTensionCoefficient"] = 0.001
    s = vtp_gpu.solver_from_scene(sc)
    with pytest.raises(vtp_gpu.VtpError, match="surface-tension"):
        diff.diff_forward(s, 2, 1)
    s.destroy()


@pytest.mark.gpu
def test_torch_autograd_dfsph_rollout(vtp_gpu):
    """The torch wrapper's gradients are the C ABI's for the same loss."""
    import torch
    from vtp import diff
    sc = gpu_case(seed=9, n=2000)
    mask = diff.fluid_mask(sc)
    f = sc.objects[0]
    roll = diff.make_dfsph_rollout(sc, steps=4, checkpoint_every=2)
    x0 = torch.tensor(f.pos, requires_grad=True)
    v0 = torch.tensor(f.velocity, requires_grad=True)
    w = torch.linspace(-1.0, 1.0, 3, dtype=torch.float64)

    def loss_of(x, v):
        return (x.double().mean(0) * w).sum() + (v.double() ** 2).sum() * 1e-3

    x, v = roll(x0, v0)
    loss_of(x, v).backward()
    # the same loss through the C ABI: dL/d(output) from torch, then the library's backward
    s = vtp_gpu.solver_from_scene(sc)
    assert s.initialize()
    diff.diff_forward(s, 4, 2)
    xo = torch.tensor(s.get_field("pos")[mask], requires_grad=True)
    vo = torch.tensor(s.get_field("vel")[mask], requires_grad=True)
    assert torch.equal(xo, x.detach()) and torch.equal(vo, v.detach())
    loss_of(xo, vo).backward()
    n = mask.size
    gx = np.zeros((n, 3), np.float32)
    gv = np.zeros((n, 3), np.float32)
    gx[mask] = xo.grad.numpy()
    gv[mask] = vo.grad.numpy()
    ox, ov, _ = diff.diff_backward(s, gx, gv)
    s.destroy()
    assert np.array_equal(x0.grad.numpy(), ox[mask])
    assert np.array_equal(v0.grad.numpy(), ov[mask])
