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
