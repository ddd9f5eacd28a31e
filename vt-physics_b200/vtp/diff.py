"""Differentiable PBF and DFSPH through the C ABI, and their torch.autograd wrappers.

The adjoint itself is the library's (vtp_solver_diff_forward / _backward:
checkpointed forward, per-segment recompute into a tape with the substep
kernels, hand-written adjoint passes in reverse).  This module moves arrays
across the boundary and exposes the rollout to torch.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from ._lib import check, lib
from .solver import Object, Particle_Common, PBFSolver


def diff_forward(s, steps: int, checkpoint_every: int = 20, keep_lists: bool = False):
    check(lib().vtp_solver_diff_forward(s._h, int(steps), int(checkpoint_every), 1 if keep_lists else 0),
          "diff_forward")


def diff_backward(s, dl_dpos=None, dl_dvel=None):
    """dL/d(final pos, vel) (n x 3, attach order) -> (dL/dpos0, dL/dvel0, dL/dparam), the
    parameter being XSPH_k (PBF) or fPartRestViscosity (DFSPH)."""
    n = s.counts()["total"]

    def arr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, np.float32).reshape(n, 3)
        return a

    gp, gv = arr(dl_dpos), arr(dl_dvel)
    op = np.zeros((n, 3), np.float32)
    ov = np.zeros((n, 3), np.float32)
    gk = C.c_double()
    check(lib().vtp_solver_diff_backward(s._h, None if gp is None else gp.ctypes.data,
                                         None if gv is None else gv.ctypes.data, op.ctypes.data, ov.ctypes.data,
                                         C.byref(gk)), "diff_backward")
    return op, ov, gk.value


def diff_lists(s, step: int, max_nbr: int):
    n = s.counts()["total"]
    cnt = np.empty(n, np.uint32)
    nb = np.empty((n, max_nbr), np.uint32)
    check(lib().vtp_solver_diff_lists(s._h, int(step), cnt.ctypes.data, nb.ctypes.data, int(max_nbr)), "diff_lists")
    return cnt, nb


def diff_iterations(s, step: int):
    """DFSPH: (divergence, density) pressure-solve iterations of recorded substep `step`."""
    di, ii = C.c_uint32(), C.c_uint32()
    check(lib().vtp_solver_diff_iterations(s._h, int(step), C.byref(di), C.byref(ii)), "diff_iterations")
    return di.value, ii.value


def pbf_solver(scene, v0_fluid=None, xsph_k=None, extra=None):
    """A PBF solver of `scene` with per-particle initial fluid velocities and an XSPH coefficient."""
    cfg = json.loads(json.dumps(scene.config))
    if xsph_k is not None:
        cfg["PBF"]["Required"]["XSPH_k"] = float(xsph_k)
    if extra:
        cfg["B200"] = dict(extra)
    s = PBFSolver(strict=True)
    s.setConfig(cfg)
    k = 0
    for o in scene.objects:
        obj = Object(Particle_Common, o.name)
        obj.getObjectComponentConfig()["epmMaterial"] = o.material
        obj.attachSpecificSolverObjectComponentConfig({"solverType": 0, "exportFlag": o.export_flag,
                                                       "velocityStart": list(o.velocity_start),
                                                       "colorStart": list(o.color_start)})
        obj.pos = o.pos
        obj.velocity = o.velocity
        if o.material == 0 and v0_fluid is not None:
            obj.velocity = np.asarray(v0_fluid[k:k + o.n], np.float32)
            k += o.n
        s.attachObject(obj)
    s.initialize()
    return s


def fluid_mask(scene) -> np.ndarray:
    return np.concatenate([np.full(o.n, o.material == 0) for o in scene.objects])


def make_rollout(scene, steps: int, checkpoint_every: int = 20, extra=None):
    """torch.autograd.Function: (v0 of the fluid [nf, 3], XSPH_k []) -> fluid positions after `steps`."""
    import torch

    mask = fluid_mask(scene)

    class PbfRollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, v0, k):
            s = pbf_solver(scene, v0.detach().cpu().numpy(), float(k.item()), extra)
            diff_forward(s, steps, checkpoint_every)
            pos = s.get_field("pos")
            ctx.solver = s
            return torch.from_numpy(pos[mask].copy()).to(v0.device)

        @staticmethod
        def backward(ctx, g):
            s = ctx.solver
            n = s.counts()["total"]
            dl = np.zeros((n, 3), np.float32)
            dl[mask] = g.detach().cpu().numpy()
            _, gv, gk = diff_backward(s, dl, None)
            s.destroy()
            ctx.solver = None
            dev = g.device
            return torch.from_numpy(gv[mask].copy()).to(dev), torch.tensor(gk, dtype=torch.float32, device=dev)

    return PbfRollout.apply


def make_dfsph_rollout(scene, steps: int, checkpoint_every: int = 10, extra=None):
    """torch.autograd.Function: (fluid positions x0 [nf, 3], fluid velocities v0 [nf, 3]) ->
    (fluid positions, fluid velocities) after `steps` DFSPH substeps; the backward is the
    library's adjoint of the rollout (lists, iteration counts and clamps of the forward)."""
    import torch

    mask = fluid_mask(scene)

    class DfsphRollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x0, v0):
            from .solver import solver_from_scene
            s = solver_from_scene(scene, extra=extra)
            if not s.initialize():
                raise RuntimeError(s.last_error)
            for name, val in (("pos", x0), ("vel", v0)):
                full = s.get_field(name)
                full[mask] = val.detach().cpu().numpy()
                s.set_field(name, full)
            diff_forward(s, steps, checkpoint_every)
            ctx.solver = s
            dev = x0.device
            return (torch.from_numpy(s.get_field("pos")[mask].copy()).to(dev),
                    torch.from_numpy(s.get_field("vel")[mask].copy()).to(dev))

        @staticmethod
        def backward(ctx, gx, gv):
            s = ctx.solver
            n = s.counts()["total"]
            dx = np.zeros((n, 3), np.float32)
            dv = np.zeros((n, 3), np.float32)
            if gx is not None:
                dx[mask] = gx.detach().cpu().numpy()
            if gv is not None:
                dv[mask] = gv.detach().cpu().numpy()
            ox, ov, _ = diff_backward(s, dx, dv)
            s.destroy()
            ctx.solver = None
            dev = (gx if gx is not None else gv).device
            return torch.from_numpy(ox[mask].copy()).to(dev), torch.from_numpy(ov[mask].copy()).to(dev)

    return DfsphRollout.apply


def dfsph_solve(s, v_in, which: int = 0, force_iters: int = 0):
    """One DFSPH pressure solve on the solver's current positions: (v* out, iterations)."""
    n = s.counts()["total"]
    vi = np.ascontiguousarray(v_in, np.float32).reshape(n, 3)
    vo = np.zeros((n, 3), np.float32)
    it = C.c_uint32()
    check(lib().vtp_solver_dfsph_solve_forward(s._h, int(which), vi.ctypes.data, vo.ctypes.data, int(force_iters),
                                               C.byref(it)), "dfsph_solve_forward")
    return vo, it.value


def dfsph_solve_vjp(s, vbar_out):
    """dL/d(v* in) of the last dfsph_solve, given dL/d(v* out)."""
    n = s.counts()["total"]
    vb = np.ascontiguousarray(vbar_out, np.float32).reshape(n, 3)
    out = np.zeros((n, 3), np.float32)
    check(lib().vtp_solver_dfsph_solve_backward(s._h, vb.ctypes.data, out.ctypes.data), "dfsph_solve_backward")
    return out


def make_dfsph_solve(s, which: int = 0, force_iters: int = 0):
    """torch.autograd.Function over the pressure solve of solver `s` at its current state."""
    import torch

    class DfsphSolve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, v):
            out, _ = dfsph_solve(s, v.detach().cpu().numpy(), which, force_iters)
            return torch.from_numpy(out).to(v.device)

        @staticmethod
        def backward(ctx, g):
            return torch.from_numpy(dfsph_solve_vjp(s, g.detach().cpu().numpy())).to(g.device)

    return DfsphSolve.apply
