"""Python front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, always as the checker: it is never a fallback for the CUDA path.
State is kept in attach order in FP64; neighbour search runs in FP32 with the
reference's arithmetic (UGNSCudaImpl.cu:28-203).
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None


class OrGrid(C.Structure):
    _fields_ = [("lb", C.c_float * 3), ("cell", C.c_float), ("dims", C.c_int32 * 3), ("maxnbr", C.c_uint32)]


class OrPbf(C.Structure):
    _fields_ = [("dt", C.c_double), ("h", C.c_double), ("rho0", C.c_double), ("rho_b", C.c_double),
                ("xsph_k", C.c_double), ("eps", C.c_double), ("g", C.c_double * 3), ("iterations", C.c_int32),
                ("form", C.c_int32)]


class OrDfsph(C.Structure):
    _fields_ = [("dt", C.c_double), ("h", C.c_double), ("rho0", C.c_double), ("rho_b", C.c_double),
                ("vis", C.c_double), ("div_thr", C.c_double), ("inc_thr", C.c_double), ("gamma", C.c_double),
                ("g", C.c_double * 3), ("force_div", C.c_int32), ("force_inc", C.c_int32),
                ("max_iters", C.c_int32)]


class OrImm(C.Structure):
    _fields_ = [("dt", C.c_double), ("h", C.c_double), ("vol0", C.c_double), ("gamma", C.c_double),
                ("Cf", C.c_double), ("Cd0", C.c_double), ("g", C.c_double * 3), ("P", C.c_int32),
                ("ct", C.c_int32), ("rho", C.c_double * 8), ("mu", C.c_double * 8), ("vis_base", C.c_double),
                ("vis_max", C.c_double), ("relax", C.c_double), ("thin0", C.c_double), ("theta", C.c_double),
                ("div_thr", C.c_double), ("inc_thr", C.c_double), ("force_div", C.c_int32),
                ("force_inc", C.c_int32), ("max_iters", C.c_int32)]


class OrImmOut(C.Structure):
    _fields_ = [("div_iters", C.c_int32), ("inc_iters", C.c_int32), ("div_residual", C.c_double),
                ("inc_residual", C.c_double), ("retries", C.c_int32), ("crashed", C.c_int32)]


class OrSolveOut(C.Structure):
    _fields_ = [("div_iters", C.c_int32), ("inc_iters", C.c_int32), ("div_residual", C.c_double),
                ("inc_residual", C.c_double), ("crashed", C.c_int32)]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            from . import build as _b  # type: ignore
            _b.build()
        L = C.CDLL(str(path))
        P = C.c_void_p
        L.or_neighbors.restype = C.c_uint32
        L.or_neighbors.argtypes = [C.c_uint32, P, C.POINTER(OrGrid), P, P, P, P]
        L.or_pbf_init.argtypes = [C.c_uint32, P, P, P, P, C.POINTER(OrGrid), C.POINTER(OrPbf)]
        L.or_pbf_step.argtypes = [C.c_uint32, P, P, P, P, P, C.POINTER(OrGrid), C.POINTER(OrPbf), P, P]
        L.or_dfsph_init.argtypes = [C.c_uint32, P, P, P, P, C.POINTER(OrGrid), C.POINTER(OrDfsph)]
        L.or_dfsph_step.argtypes = [C.c_uint32, P, P, C.c_int32, P, P, P, P, P, C.POINTER(OrGrid),
                                    C.POINTER(OrDfsph), C.POINTER(OrSolveOut), P, P]
        L.or_pbf_step_frozen.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrPbf)]
        L.or_pbf_step_adjoint.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrPbf), P, P,
                                          C.POINTER(C.c_double)]
        L.or_dfsph_solve_op.argtypes = [C.c_uint32, P, P, P, P, P, P, C.c_uint32, C.c_double, C.c_double, C.c_int,
                                         P, P]
        L.or_dfsph_step_frozen.restype = None
        L.or_dfsph_step_frozen.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrDfsph),
                                           C.c_int, C.c_int]
        L.or_dfsph_step_adjoint.restype = None
        L.or_dfsph_step_adjoint.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrDfsph),
                                            C.c_int, C.c_int, P, P, C.POINTER(C.c_double)]
        L.or_imm_init.argtypes = [C.c_uint32, P, P, P, C.POINTER(OrGrid), C.POINTER(OrImm)]
        L.or_imm_step.argtypes = [C.c_uint32, P, P, C.c_int32, P, P, P, P, P, P, P, P, C.POINTER(OrGrid),
                                  C.POINTER(OrImm), C.POINTER(OrImmOut)]
        for name in ("or_dfsph_ratio_alpha", "or_dfsph_solve_a", "or_dfsph_solve_b", "or_dfsph_forces",
                     "or_dfsph_tension"):
            getattr(L, name).restype = None
        L.or_dfsph_ratio_alpha.argtypes = [C.c_uint32, P, P, P, P, P, P, C.c_uint32, C.c_double, P, P]
        L.or_dfsph_solve_a.argtypes = [C.c_uint32, P, P, P, P, P, P, P, P, C.c_uint32, C.c_double, C.c_double, P, P]
        L.or_dfsph_solve_b.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.c_double, C.c_double, P]
        L.or_dfsph_pressure_apply.argtypes = [C.c_uint32, P, P, P, C.c_double]
        L.or_dfsph_forces.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrDfsph), P, P]
        L.or_dfsph_tension.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrDfsph), P]
        L.or_dfsph_accelerate.argtypes = [C.c_uint32, P, P, P, P, C.c_double]
        for name in ("or_pbf_apply_force", "or_pbf_lambda", "or_pbf_dx", "or_pbf_xsph"):
            getattr(L, name).restype = None
        L.or_pbf_apply_force.argtypes = [C.c_uint32, P, P, P, C.POINTER(OrPbf)]
        L.or_pbf_lambda.argtypes = [C.c_uint32, P, P, P, P, P, C.c_uint32, C.POINTER(OrPbf), P, P]
        L.or_pbf_dx.argtypes = [C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrPbf), P]
        L.or_pbf_xsph.argtypes = [C.c_uint32, P, P, P, P, P, P, C.c_uint32, C.POINTER(OrPbf), P]
        L.or_dfsph_advance.argtypes = [C.c_uint32, P, P, P, P, C.c_double]
        L.or_num_threads.restype = C.c_int
        L.or_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data if a is not None else None


def make_grid(required: dict) -> OrGrid:
    """Grid of UniformGirdNeighborSearcher::setConfig: cell = h = 4 r, dims = ceil(size / h) in FP32."""
    r = np.float32(required["particleRadius"])
    h = np.float32(r * np.float32(4))
    g = OrGrid()
    for a in range(3):
        g.lb[a] = float(np.float32(required["simSpaceLB"][a]))
        g.dims[a] = int(math.ceil(float(np.float32(np.float32(required["simSpaceSize"][a]) / h))))
    g.cell = float(h)
    g.maxnbr = int(required["maxNeighborNum"])
    return g


def neighbors(pos: np.ndarray, grid: OrGrid):
    """Reference-layout neighbour lists, stable (cell, id) order and cell keys."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    n = pos.shape[0]
    cnt = np.empty(n, np.uint32)
    nb = np.empty((n, grid.maxnbr), np.uint32)
    ids = np.empty(n, np.uint32)
    keys = np.empty(n, np.uint32)
    alive = lib().or_neighbors(n, _ptr(pos), C.byref(grid), _ptr(cnt), _ptr(nb), _ptr(ids), _ptr(keys))
    return cnt, nb, ids[:alive], keys[:alive]


def set_threads(n: int):
    lib().or_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().or_num_threads())


class OracleSolver:
    """FP64 state machine for one scene (PBF or DFSPH), attach order."""

    def __init__(self, scene, force_div: int = 0, force_inc: int = 0):
        self.kind = scene.solver
        req = scene.config[self.kind]["Required"]
        opt = scene.config[self.kind]["Optional"]
        self.grid = make_grid(req)
        objs = scene.objects
        self.pos = np.concatenate([o.pos for o in objs]).astype(np.float64)
        vels = []
        for o in objs:
            if o.velocity is not None:
                vels.append(np.asarray(o.velocity, np.float32))
            else:
                vels.append(np.tile(np.asarray(o.velocity_start, np.float32), (o.n, 1)))
        self.vel = np.concatenate(vels).astype(np.float64)
        self.mat = np.concatenate([np.full(o.n, o.material, np.int32) for o in objs])
        self.obj = np.concatenate([np.full(o.n, k, np.int32) for k, o in enumerate(objs)])
        self.obj_is_fluid = np.array([1 if o.material == 0 else 0 for o in objs], np.int32)
        self.n = self.pos.shape[0]
        r = np.float32(req["particleRadius"])
        h = float(np.float32(r * np.float32(4)))
        vol0 = float(np.float32(np.float32(2) * r) ** np.float32(3))
        g = [0.0, -9.8, 0.0]
        if opt["enable"]:
            g = [float(np.float32(v)) for v in opt["gravity"]]
        self.vol = np.full(self.n, vol0, np.float64)
        self.steps = 0
        if self.kind == "PBF":
            p = OrPbf()
            p.dt = float(np.float32(req["timeStep"]))
            p.h = h
            p.rho0 = float(np.float32(req["fPartRestDensity"]))
            p.rho_b = float(np.float32(req["bPartRestDensity"]))
            p.xsph_k = float(np.float32(req["XSPH_k"]))
            p.eps = float(np.float32(1e-6))
            for a in range(3):
                p.g[a] = g[a]
            p.iterations = int(req["iterationNum"])
            ext = scene.config.get("B200", {})
            if ext.get("pbfFormulation", "reference") == "standard":
                p.form = 1
                p.eps = float(np.float32(ext.get("pbfEpsilon", 100.0)))
            self.p = p
            self.mass = np.full(self.n, p.rho0 * vol0, np.float64)
            lib().or_pbf_init(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.mass), _ptr(self.vol),
                              C.byref(self.grid), C.byref(p))
            self.density = np.zeros(self.n)
            self.lam = np.zeros(self.n)
        elif self.kind == "DFSPH":
            p = OrDfsph()
            p.dt = float(np.float32(req["timeStep"]))
            p.h = h
            p.rho0 = float(np.float32(req["fPartRestDensity"]))
            p.rho_b = float(np.float32(req["bPartRestDensity"]))
            p.vis = float(np.float32(req["fPartRestViscosity"]))
            p.div_thr = float(np.float32(req["divFreeThreshold"]))
            p.inc_thr = float(np.float32(req["incompThreshold"]))
            p.gamma = float(np.float32(req["surfaceTensionCoefficient"]))
            for a in range(3):
                p.g[a] = g[a]
            p.force_div = force_div
            p.force_inc = force_inc
            p.max_iters = 101
            self.p = p
            # adaptive step (the library's "cfl" extension): dt = min(timeStep, cfl * 2r / max |v|)
            self.cfl = float(scene.config.get("B200", {}).get("cfl", 0.0))
            self.dt_max = np.float32(req["timeStep"])
            self.diameter = np.float32(2) * np.float32(req["particleRadius"])
            self.dts = []
            self.rest_density = np.where(self.mat == 0, p.rho0, 0.0).astype(np.float64)
            lib().or_dfsph_init(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vol), _ptr(self.rest_density),
                                C.byref(self.grid), C.byref(p))
            self.ratio = np.zeros(self.n)
            self.alpha = np.zeros(self.n)
            self.last = OrSolveOut()
        else:
            raise NotImplementedError(self.kind)

    def set_forced_iterations(self, div: int, inc: int):
        self.p.force_div = int(div)
        self.p.force_inc = int(inc)

    def step(self, n: int = 1):
        L = lib()
        for _ in range(n):
            if self.kind == "PBF":
                L.or_pbf_step(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vel), _ptr(self.mass),
                              _ptr(self.vol), C.byref(self.grid), C.byref(self.p), _ptr(self.density),
                              _ptr(self.lam))
            else:
                if self.cfl > 0:
                    # the library's formula in FP32 on the fluid velocities of this substep
                    v = self.vel[self.mat == 0].astype(np.float32)
                    v2 = (v * v).sum(axis=1, dtype=np.float32)
                    vmax = np.sqrt(np.float32(v2.max())) if v2.size else np.float32(0)
                    dt = self.dt_max
                    if vmax > 0:
                        dt = max(min(self.dt_max, np.float32(np.float32(self.cfl) * self.diameter) / vmax),
                                 np.float32(self.dt_max * np.float32(1e-4)))
                    self.p.dt = float(np.float32(dt))
                    self.dts.append(self.p.dt)
                out = OrSolveOut()
                L.or_dfsph_step(self.n, _ptr(self.mat), _ptr(self.obj), len(self.obj_is_fluid),
                                _ptr(self.obj_is_fluid), _ptr(self.pos), _ptr(self.vel), _ptr(self.vol),
                                _ptr(self.rest_density), C.byref(self.grid), C.byref(self.p), C.byref(out),
                                _ptr(self.ratio), _ptr(self.alpha))
                self.last = out
            self.steps += 1


class ImmOracle:
    """FP64 state machine for one IMM or IMM-CT scene (attach order): positions,
    mixture and phase velocities, volume fractions, conformation tensor and Cd
    (IMMCTSolver.cpp:408-477, IMMSolver.cpp:400-466; or_imm_step)."""

    def __init__(self, scene, force_div: int = 0, force_inc: int = 0):
        self.kind = scene.solver
        req = scene.config[self.kind]["Required"]
        opt = scene.config[self.kind]["Optional"]
        self.grid = make_grid(req)
        objs = scene.objects
        self.pos = np.concatenate([o.pos for o in objs]).astype(np.float64)
        vels = [np.asarray(o.velocity, np.float32) if o.velocity is not None
                else np.tile(np.asarray(o.velocity_start, np.float32), (o.n, 1)) for o in objs]
        self.vel = np.concatenate(vels).astype(np.float64)
        self.mat = np.concatenate([np.full(o.n, o.material, np.int32) for o in objs])
        self.obj = np.concatenate([np.full(o.n, k, np.int32) for k, o in enumerate(objs)])
        self.obj_is_fluid = np.array([1 if o.material == 0 else 0 for o in objs], np.int32)
        self.n = self.pos.shape[0]
        f32 = lambda v: float(np.float32(v))
        p = OrImm()
        r = np.float32(req["particleRadius"])
        p.dt = f32(req["timeStep"])
        p.h = f32(r * np.float32(4))
        p.vol0 = f32((np.float32(2) * r) ** np.float32(3))
        p.gamma = f32(req["surfaceTensionCoefficient"])
        p.Cf = f32(req["diffusionCoefficientCf"])
        g = [0.0, -9.8, 0.0]
        if opt["enable"]:
            g = [f32(v) for v in opt["gravity"]]
        for a in range(3):
            p.g[a] = g[a]
        rho = [f32(v) for v in req["phaseRestDensity"]]
        p.P = len(rho)
        for k, v in enumerate(rho):
            p.rho[k] = v
        p.ct = 1 if self.kind == "IMMCT" else 0
        if p.ct:
            for k in range(p.P):   # IMMCTSolver::setConfig copies solventViscosity to every phase
                p.mu[k] = f32(req["solventViscosity"])
            p.Cd0 = f32(req["momentumExchangeCoefficientCd0"])
            p.vis_base = f32(np.float32(req["solutionBasicViscosity"]) * np.float32(1000))
            p.vis_max = f32(np.float32(req["solutionMaxViscosity"]) * np.float32(1000))
            p.relax = f32(req["relaxationTime"])
            p.thin0 = f32(req["shearThinningBasicFactor"])
            p.theta = f32(req["rheologicalThreshold"])
        else:
            for k, v in enumerate(req["phaseRestViscosity"]):
                p.mu[k] = f32(v)
            p.Cd0 = f32(req["momentumExchangeCoefficientCd"])
        p.div_thr = f32(req["divFreeThreshold"])
        p.inc_thr = f32(req["incompThreshold"])
        p.force_div, p.force_inc, p.max_iters = force_div, force_inc, 101
        self.p = p
        P = p.P
        self.frac = np.concatenate([np.tile(np.asarray(o.phase_fraction, np.float32)[:P], (o.n, 1))
                                    for o in objs]).astype(np.float64)
        self.vph = np.repeat(self.vel[:, None, :], P, axis=1).copy()   # init_data_cuda: v_k = v
        self.Q = np.tile(np.eye(3).reshape(1, 9), (self.n, 1))
        self.cd = np.full(self.n, p.Cd0, np.float64)
        self.vol = np.zeros(self.n)
        lib().or_imm_init(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vol), C.byref(self.grid), C.byref(p))
        self.steps = 0
        self.last = OrImmOut()

    def set_forced_iterations(self, div: int, inc: int):
        self.p.force_div = int(div)
        self.p.force_inc = int(inc)

    def step(self, n: int = 1):
        for _ in range(n):
            out = OrImmOut()
            lib().or_imm_step(self.n, _ptr(self.mat), _ptr(self.obj), len(self.obj_is_fluid), _ptr(self.obj_is_fluid),
                              _ptr(self.pos), _ptr(self.vel), _ptr(self.vph), _ptr(self.frac), _ptr(self.Q),
                              _ptr(self.cd), _ptr(self.vol), C.byref(self.grid), C.byref(self.p), C.byref(out))
            self.last = out
            self.steps += 1


class PbfDiff:
    """FP64 differentiable PBF rollout with frozen neighbour lists (test infrastructure).

    ``rollout`` advances (pos, vel) ``steps`` substeps; the lists of substep t are either
    given (``lists[t]`` = (counts, nbrs) in the reference layout, e.g. the GPU's lists of the
    same trajectory) or built from the FP32-rounded positions after the external force, as
    the reference builds them.  ``adjoint`` runs or_pbf_step_adjoint backwards over a recorded
    rollout and returns dL/d(pos0, vel0, XSPH_k).
    """

    def __init__(self, scene, xsph_k: float | None = None):
        self.base = OracleSolver(scene)
        if xsph_k is not None:
            self.base.p.xsph_k = float(xsph_k)
        self.p = self.base.p
        self.maxnbr = int(self.base.grid.maxnbr)

    @property
    def fluid(self):
        return self.base.mat == 0

    def _lists_after_force(self, pos, vel):
        x = pos.copy()
        v = vel.copy()
        f = self.fluid
        g = np.array([self.p.g[a] for a in range(3)])
        v[f] += g * self.p.dt
        x[f] += v[f] * self.p.dt
        cnt, nb, _, _ = neighbors(x.astype(np.float32), self.base.grid)
        return cnt, nb

    def rollout(self, pos0, vel0, steps: int, lists=None, record: bool = False):
        b = self.base
        pos = np.ascontiguousarray(pos0, np.float64).copy()
        vel = np.ascontiguousarray(vel0, np.float64).copy()
        states, used = [], []
        for t in range(steps):
            cnt, nb = lists[t] if lists is not None else self._lists_after_force(pos, vel)
            cnt = np.ascontiguousarray(cnt, np.uint32)
            nb = np.ascontiguousarray(nb, np.uint32)
            if record:
                states.append((pos.copy(), vel.copy()))
                used.append((cnt, nb))
            lib().or_pbf_step_frozen(b.n, _ptr(b.mat), _ptr(pos), _ptr(vel), _ptr(b.mass), _ptr(b.vol), _ptr(cnt),
                                     _ptr(nb), self.maxnbr, C.byref(self.p))
        return pos, vel, states, used

    def adjoint(self, states, used, xbar, vbar):
        b = self.base
        xb = np.ascontiguousarray(xbar, np.float64).copy()
        vb = np.ascontiguousarray(vbar, np.float64).copy()
        kb = C.c_double(0.0)
        for t in range(len(states) - 1, -1, -1):
            pos, vel = states[t]
            cnt, nb = used[t]
            lib().or_pbf_step_adjoint(b.n, _ptr(b.mat), _ptr(pos), _ptr(vel), _ptr(b.mass), _ptr(b.vol), _ptr(cnt),
                                      _ptr(nb), self.maxnbr, C.byref(self.p), _ptr(xb), _ptr(vb), C.byref(kb))
        return xb, vb, kb.value


class DfsphDiff:
    """FP64 differentiable DFSPH rollout with frozen neighbour lists and iteration counts
    (test infrastructure; no counterpart in the reference).

    ``rollout`` advances (pos, vel) ``steps`` substeps (DFSPHSolver.cpp:339-406, surface
    tension off); substep t uses ``lists[t]`` = (counts, nbrs) in the reference layout (e.g.
    the GPU's lists of the same trajectory) or lists built from the FP32-rounded positions,
    and exactly ``iters[t]`` = (divergence, density) pressure-solve iterations.  ``adjoint``
    runs or_dfsph_step_adjoint backwards over a recorded rollout and returns
    dL/d(pos0, vel0, fPartRestViscosity).
    """

    def __init__(self, scene, viscosity: float | None = None):
        self.base = OracleSolver(scene)
        if viscosity is not None:
            self.base.p.vis = float(viscosity)
        self.p = self.base.p
        self.maxnbr = int(self.base.grid.maxnbr)
        b = self.base
        self.mass = np.where(b.mat == 0, b.rest_density * b.vol, 0.0).astype(np.float64)

    @property
    def fluid(self):
        return self.base.mat == 0

    def lists_of(self, pos):
        cnt, nb, _, _ = neighbors(np.asarray(pos).astype(np.float32), self.base.grid)
        return cnt, nb

    def rollout(self, pos0, vel0, steps: int, iters, lists=None, record: bool = False):
        b = self.base
        pos = np.ascontiguousarray(pos0, np.float64).copy()
        vel = np.ascontiguousarray(vel0, np.float64).copy()
        states, used = [], []
        for t in range(steps):
            cnt, nb = lists[t] if lists is not None else self.lists_of(pos)
            cnt = np.ascontiguousarray(cnt, np.uint32)
            nb = np.ascontiguousarray(nb, np.uint32)
            di, ii = (int(x) for x in iters[t])
            if record:
                states.append((pos.copy(), vel.copy()))
                used.append((cnt, nb, di, ii))
            lib().or_dfsph_step_frozen(b.n, _ptr(b.mat), _ptr(pos), _ptr(vel), _ptr(b.vol), _ptr(self.mass),
                                       _ptr(cnt), _ptr(nb), self.maxnbr, C.byref(self.p), di, ii)
        return pos, vel, states, used

    def adjoint(self, states, used, xbar, vbar):
        b = self.base
        xb = np.ascontiguousarray(xbar, np.float64).copy()
        vb = np.ascontiguousarray(vbar, np.float64).copy()
        kb = C.c_double(0.0)
        for t in range(len(states) - 1, -1, -1):
            pos, vel = states[t]
            cnt, nb, di, ii = used[t]
            lib().or_dfsph_step_adjoint(b.n, _ptr(b.mat), _ptr(pos), _ptr(vel), _ptr(b.vol), _ptr(self.mass),
                                        _ptr(cnt), _ptr(nb), self.maxnbr, C.byref(self.p), di, ii, _ptr(xb),
                                        _ptr(vb), C.byref(kb))
        return xb, vb, kb.value


def dfsph_solve_op(o: "OracleSolver", cnt, nbr, iters: int, vadv, vbar=None):
    """FP64 pressure-solve operator on the oracle's current positions with the given lists:
    returns (v* after `iters` iterations, dL/dv* in or None)."""
    v = np.ascontiguousarray(vadv, np.float64).copy()
    vb = None if vbar is None else np.ascontiguousarray(vbar, np.float64).copy()
    cnt = np.ascontiguousarray(cnt, np.uint32)
    nbr = np.ascontiguousarray(nbr, np.uint32)
    lib().or_dfsph_solve_op(o.n, _ptr(o.mat), _ptr(o.pos), _ptr(o.vol), _ptr(o.rest_density), _ptr(cnt), _ptr(nbr),
                            int(o.grid.maxnbr), float(o.p.h), float(o.p.dt), int(iters), _ptr(v), _ptr(vb))
    return v, vb


class DfsphDomainStages:
    """FP64 DFSPH stages over one rank's particles of a slab-decomposed scene (test
    infrastructure: the checker of the decomposed run, in the stage interface of
    ``vtp.domain.LibraryStages``).

    The rank's particles (owned and ghost fluid rows in load-slot order, then its boundary
    band) are kept sorted by scene-wide id, so the oracle's lists, stable in (cell, index),
    are the whole-scene lists in the whole-scene order; the stages are the functions
    ``or_dfsph_step`` is made of (DFSPHSolver.cpp:339-406).  Exchanged values are FP64.
    """

    def __init__(self, config: dict, fluid_pos0, bnd_pos, bnd_gid, boundary_first: bool, capacity: int,
                 n_objects: int):
        import torch
        self.torch = torch
        self.device = torch.device("cpu")
        self.dtype = torch.float64
        req = config["DFSPH"]["Required"]
        opt = config["DFSPH"]["Optional"]
        self.grid = make_grid(req)
        r = np.float32(req["particleRadius"])
        self.vol0 = float(np.float32(np.float32(2) * r) ** np.float32(3))
        p = OrDfsph()
        p.dt = float(np.float32(req["timeStep"]))
        p.h = float(np.float32(r * np.float32(4)))
        p.rho0 = float(np.float32(req["fPartRestDensity"]))
        p.rho_b = float(np.float32(req["bPartRestDensity"]))
        p.vis = float(np.float32(req["fPartRestViscosity"]))
        p.gamma = float(np.float32(req["surfaceTensionCoefficient"]))
        g = [float(np.float32(v)) for v in opt["gravity"]] if opt["enable"] else [0.0, -9.8, 0.0]
        for a in range(3):
            p.g[a] = g[a]
        p.max_iters = 101
        self.p = p
        self.nobj = int(n_objects)
        self.boundary_first = bool(boundary_first)
        # Boundary volumes of the band with the rank's initial fluid present, as a solver holding
        # the whole scene computes them at initialize (or_dfsph_init over every particle).
        fp0 = np.asarray(fluid_pos0, np.float64).reshape(-1, 3)
        bp = np.asarray(bnd_pos, np.float64).reshape(-1, 3)
        parts = [bp, fp0] if boundary_first else [fp0, bp]
        mats = [np.ones(len(bp), np.int32), np.zeros(len(fp0), np.int32)]
        if not boundary_first:
            mats = mats[::-1]
        pos = np.ascontiguousarray(np.concatenate(parts))
        mat = np.concatenate(mats)
        vol = np.full(len(pos), self.vol0)
        rest = np.where(mat == 0, p.rho0, 0.0)
        lib().or_dfsph_init(len(pos), _ptr(mat), _ptr(pos), _ptr(vol), _ptr(rest), C.byref(self.grid), C.byref(p))
        sel = mat == 1
        self.bnd_pos = bp
        self.bnd_gid = np.asarray(bnd_gid, np.int64)
        self.bnd_vol = vol[sel]
        self.bnd_rest = rest[sel]

    def empty(self, field: int, count: int):
        shape = (count,) if field == 0 else (count, 3)
        return self.torch.empty(shape, dtype=self.torch.float64)

    def load(self, n_own, pos, vel, gid, obj):
        nf = pos.shape[0]
        nb = len(self.bnd_gid)
        all_gid = np.concatenate([gid.numpy().astype(np.int64), self.bnd_gid])
        order = np.argsort(all_gid, kind="stable")
        inv = np.empty_like(order)
        inv[order] = np.arange(len(order))
        self.local_of_slot = inv[:nf]
        self.n_own = int(n_own)
        cat = lambda f, b: np.ascontiguousarray(np.concatenate([f, b])[order])
        self.pos = cat(pos.numpy().astype(np.float64), self.bnd_pos)
        self.vel = cat(vel.numpy().astype(np.float64), np.zeros((nb, 3)))
        self.mat = cat(np.zeros(nf, np.int32), np.ones(nb, np.int32))
        self.vol = cat(np.full(nf, self.vol0), self.bnd_vol)
        self.rest = cat(np.full(nf, self.p.rho0), self.bnd_rest)
        self.mass = np.where(self.mat == 0, self.rest * self.vol, 0.0)
        obj_all = np.full(nf + nb, -1, np.int32)
        obj_all[self.local_of_slot[: self.n_own]] = obj.numpy()[: self.n_own]
        self.obj = obj_all
        self.n = nf + nb

    def prepare(self):
        cnt, nbr, _, _ = neighbors(self.pos.astype(np.float32), self.grid)
        self.cnt, self.nbr = cnt, nbr
        n, M = self.n, int(self.grid.maxnbr)
        self.M = M
        self.ratio = np.zeros(n)
        self.alpha = np.zeros(n)
        lib().or_dfsph_ratio_alpha(n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vol), _ptr(self.mass), _ptr(cnt),
                                   _ptr(nbr), M, self.p.h, _ptr(self.ratio), _ptr(self.alpha))
        self.vadv = self.vel.copy()
        self.kappa = np.zeros(n)
        self.delta = np.zeros(n)
        self.acc = np.zeros((n, 3))
        self.nrm = np.zeros((n, 3))

    def vmax2(self) -> float:
        """Largest |v|^2 of the owned rows, as OracleSolver forms it for the adaptive step."""
        idx = self.local_of_slot[: self.n_own]
        if idx.size == 0:
            return 0.0
        v = self.vel[idx].astype(np.float32)
        return float((v * v).sum(axis=1, dtype=np.float32).max())

    def set_dt(self, dt: float):
        self.p.dt = float(np.float32(dt))

    def solve_begin(self, which: int):
        pass

    def solve_a(self):
        lib().or_dfsph_solve_a(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vol), _ptr(self.ratio),
                               _ptr(self.alpha), _ptr(self.vadv), _ptr(self.cnt), _ptr(self.nbr), self.M, self.p.h,
                               self.p.dt, _ptr(self.delta), _ptr(self.kappa))
        sums = np.zeros(self.nobj)
        for i in np.nonzero(self.obj >= 0)[0]:   # owned rows, ascending id
            sums[self.obj[i]] += self.delta[i]
        return self.torch.tensor(sums, dtype=self.torch.float64)

    def solve_b(self):
        lib().or_dfsph_solve_b(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vol), _ptr(self.mass),
                               _ptr(self.kappa), _ptr(self.cnt), _ptr(self.nbr), self.M, self.p.h, self.p.dt,
                               _ptr(self.vadv))

    def forces(self):
        L = lib()
        L.or_dfsph_pressure_apply(self.n, _ptr(self.mat), _ptr(self.vel), _ptr(self.vadv), self.p.dt)
        L.or_dfsph_forces(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vel), _ptr(self.mass), _ptr(self.rest),
                          _ptr(self.cnt), _ptr(self.nbr), self.M, C.byref(self.p), _ptr(self.acc), _ptr(self.nrm))
        if self.p.gamma == 0.0:
            L.or_dfsph_accelerate(self.n, _ptr(self.mat), _ptr(self.vel), _ptr(self.vadv), _ptr(self.acc), self.p.dt)

    def tension(self):
        L = lib()
        L.or_dfsph_tension(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.mass), _ptr(self.rest), _ptr(self.nrm),
                           _ptr(self.cnt), _ptr(self.nbr), self.M, C.byref(self.p), _ptr(self.acc))
        L.or_dfsph_accelerate(self.n, _ptr(self.mat), _ptr(self.vel), _ptr(self.vadv), _ptr(self.acc), self.p.dt)

    def finalize(self):
        lib().or_dfsph_advance(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vel), _ptr(self.vadv), self.p.dt)

    def _field(self, field: int):
        return (self.kappa, self.vadv, self.vel, self.nrm)[field]

    def pack(self, field: int, slots):
        idx = self.local_of_slot[slots.numpy()]
        return self.torch.from_numpy(self._field(field)[idx].copy())

    def unpack(self, field: int, first: int, values):
        idx = self.local_of_slot[first: first + values.shape[0]]
        v = values.numpy()
        self._field(field)[idx] = v
        if field == 2:   # velocities after the forces: v* = v
            self.vadv[idx] = v

    def read(self):
        idx = self.local_of_slot[: self.n_own]
        return self.torch.from_numpy(self.pos[idx].copy()), self.torch.from_numpy(self.vel[idx].copy())


class PbfDomainStages:
    """FP64 PBF stages over one rank's particles of a slab-decomposed scene (test
    infrastructure: the checker of the decomposed run, in the stage interface of
    ``vtp.domain.LibraryStages``).  Particles are kept sorted by scene-wide id as in
    ``DfsphDomainStages``; the stages are the functions ``or_pbf_step`` is made of
    (PBFSolver.cpp:326-376)."""

    def __init__(self, config: dict, fluid_pos0, bnd_pos, bnd_gid, boundary_first: bool, capacity: int,
                 n_objects: int):
        import torch
        self.torch = torch
        self.device = torch.device("cpu")
        self.dtype = torch.float64
        req = config["PBF"]["Required"]
        opt = config["PBF"]["Optional"]
        self.grid = make_grid(req)
        r = np.float32(req["particleRadius"])
        self.vol0 = float(np.float32(np.float32(2) * r) ** np.float32(3))
        p = OrPbf()
        p.dt = float(np.float32(req["timeStep"]))
        p.h = float(np.float32(r * np.float32(4)))
        p.rho0 = float(np.float32(req["fPartRestDensity"]))
        p.rho_b = float(np.float32(req["bPartRestDensity"]))
        p.xsph_k = float(np.float32(req["XSPH_k"]))
        p.eps = float(np.float32(1e-6))
        g = [float(np.float32(v)) for v in opt["gravity"]] if opt["enable"] else [0.0, -9.8, 0.0]
        for a in range(3):
            p.g[a] = g[a]
        p.iterations = int(req["iterationNum"])
        ext = config.get("B200", {})
        if ext.get("pbfFormulation", "reference") == "standard":
            p.form = 1
            p.eps = float(np.float32(ext.get("pbfEpsilon", 100.0)))
        self.p = p
        self.mass0 = p.rho0 * self.vol0
        # boundary mass / volume of the band with the rank's initial fluid present (or_pbf_init)
        fp0 = np.asarray(fluid_pos0, np.float64).reshape(-1, 3)
        bp = np.asarray(bnd_pos, np.float64).reshape(-1, 3)
        parts = [bp, fp0] if boundary_first else [fp0, bp]
        mats = [np.ones(len(bp), np.int32), np.zeros(len(fp0), np.int32)]
        if not boundary_first:
            mats = mats[::-1]
        pos = np.ascontiguousarray(np.concatenate(parts))
        mat = np.concatenate(mats)
        mass = np.full(len(pos), self.mass0)
        vol = np.full(len(pos), self.vol0)
        lib().or_pbf_init(len(pos), _ptr(mat), _ptr(pos), _ptr(mass), _ptr(vol), C.byref(self.grid), C.byref(p))
        sel = mat == 1
        self.bnd_pos = bp
        self.bnd_gid = np.asarray(bnd_gid, np.int64)
        self.bnd_mass = mass[sel]
        self.bnd_vol = vol[sel]

    def empty(self, field: int, count: int):
        return self.torch.empty((count,) if field == 4 else (count, 6), dtype=self.torch.float64)

    def load(self, n_own, pos, vel, gid, obj):
        nf = pos.shape[0]
        nb = len(self.bnd_gid)
        order = np.argsort(np.concatenate([gid.numpy().astype(np.int64), self.bnd_gid]), kind="stable")
        inv = np.empty_like(order)
        inv[order] = np.arange(len(order))
        self.local_of_slot = inv[:nf]
        self.n_own = int(n_own)
        cat = lambda f, b: np.ascontiguousarray(np.concatenate([f, b])[order])
        self.pos = cat(pos.numpy().astype(np.float64), self.bnd_pos)
        self.vel = cat(vel.numpy().astype(np.float64), np.zeros((nb, 3)))
        self.mat = cat(np.zeros(nf, np.int32), np.ones(nb, np.int32))
        self.mass = cat(np.full(nf, self.mass0), self.bnd_mass)
        self.vol = cat(np.full(nf, self.vol0), self.bnd_vol)
        self.n = nf + nb

    def prepare(self):
        lib().or_pbf_apply_force(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vel), C.byref(self.p))
        self.cnt, self.nbr, _, _ = neighbors(self.pos.astype(np.float32), self.grid)
        self.M = int(self.grid.maxnbr)
        self.rho = np.zeros(self.n)
        self.lam = np.zeros(self.n)
        self.dx = np.zeros((self.n, 3))

    def pbf_lambda(self):
        lib().or_pbf_lambda(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.mass), _ptr(self.cnt), _ptr(self.nbr),
                            self.M, C.byref(self.p), _ptr(self.rho), _ptr(self.lam))

    def pbf_dx(self):
        lib().or_pbf_dx(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vel), _ptr(self.mass), _ptr(self.lam),
                        _ptr(self.cnt), _ptr(self.nbr), self.M, C.byref(self.p), _ptr(self.dx))

    def pbf_xsph(self):
        lib().or_pbf_xsph(self.n, _ptr(self.mat), _ptr(self.pos), _ptr(self.vel), _ptr(self.vol), _ptr(self.cnt),
                          _ptr(self.nbr), self.M, C.byref(self.p), _ptr(self.dx))

    def pack(self, field: int, slots):
        idx = self.local_of_slot[slots.numpy()]
        if field == 4:
            return self.torch.from_numpy(self.lam[idx].copy())
        return self.torch.from_numpy(np.concatenate([self.pos[idx], self.vel[idx]], axis=1))

    def unpack(self, field: int, first: int, values):
        idx = self.local_of_slot[first: first + values.shape[0]]
        v = values.numpy()
        if field == 4:
            self.lam[idx] = v
        else:
            self.pos[idx] = v[:, :3]
            self.vel[idx] = v[:, 3:]

    def read(self):
        idx = self.local_of_slot[: self.n_own]
        return self.torch.from_numpy(self.pos[idx].copy()), self.torch.from_numpy(self.vel[idx].copy())
