"""Single-scene domain decomposition of DFSPH and PBF: one slab of the scene per rank.

The reference runs a scene on one device (SolverManager.cpp:11-17).  Here a
DFSPH or PBF scene too large for one GPU, or wanted faster than one GPU runs it, is
split along one axis into slabs, one per rank, by fluid-particle quantiles at
the start.  Rank k owns the fluid particles whose coordinate on that axis
lies in [bounds[k], bounds[k+1]) and holds

* ghosts: copies of the fluid particles other ranks own within ``ghost``
  (h plus a margin) of its slab, refreshed every substep;
* a boundary band: the boundary particles within ``2 * ghost`` of its slab
  (those within one ghost width are neighbours of owned rows, the outer half
  completes their own neighbourhoods for the boundary volumes).

A substep (DFSPHSolver::tick, DFSPHSolver.cpp:339-406) runs as the stages of
the rank's worker (``vtp_domain_*`` in include/vtp.h) with exchanges between:

1. migration: owned particles whose new position lies in another slab move
   to that slab's rank (from the second substep on);
2. ghosts: positions, velocities and ids of the owned particles within
   ``ghost`` of each peer's slab go to that peer;
3. load and prepare: sort, neighbour lists, compression ratio and alpha;
4. the divergence solve, then after step 5 the density solve; every iteration
   runs solve_a, sends kappa to the ghosts, runs solve_b, sends v* to the
   ghosts, adds the ranks' per-object FP64 residual sums and applies the
   reference's stop test (vfsph_div / vfsph_incomp, DFSPHCudaImpl.cu:449-503)
   to the sum, identically on every rank;
5. forces (pressure applied, viscosity, gravity; surface normals, then the
   tension pass with the ghosts' normals, when the tension coefficient is not
   0), then the ghosts' velocities;
6. finalize (positions advanced) and the owned rows read back.

A PBF substep (PBFSolver::tick, PBFSolver.cpp:326-376) has no residual: after
migration and the ghosts (chosen with twice the largest move under the
external force added to the ghost width, since PBF builds its lists on the
positions after that force), every constraint iteration runs the lambda pass,
sends lambda to the ghosts, runs the correction pass and sends the corrected
positions and velocities to the ghosts; XSPH follows.

Rows keep their scene-wide attach ids and a rank holds every particle within
h of its owned rows, so an owned row's neighbour list, in the reference's
order, is the one a solver holding the whole scene builds, and every value it
gathers equals the whole-scene value: with the same iteration counts the
decomposed run gives the whole-scene trajectory bit for bit.  Only the
residual's FP64 sum is associated differently (per rank, then across ranks),
which moves it by rounding.

Exchanges go through a ``comm`` object: ``TorchComm`` over an initialised
torch.distributed group (NCCL point-to-point and all-reduce between GPUs,
gloo on CPU tensors) or ``LoopbackComm``, which runs several domains in one
process (threads, one CUDA stream each) for tests and for emulating a
decomposition on one device.  The stage backend is pluggable: ``LibraryStages``
runs the sm_100a library; the tests plug in the FP64 oracle's stages.
Bounds stay fixed after the start (no rebalancing).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import threading
from dataclasses import dataclass

import numpy as np

FIELD_KAPPA, FIELD_VADV, FIELD_VEL, FIELD_NORMAL = 0, 1, 2, 3   # DFSPH exchanges
FIELD_LAMBDA, FIELD_POSVEL = 4, 5                               # PBF exchanges
GHOST_MARGIN = 1.01   # ghost width / h: covers the FP32 rounding of the membership test r <= h


# ----------------------------------------------------------------------------- scene and slabs

@dataclass
class SceneArrays:
    """A DFSPH or PBF scene in the attach order of a solver holding all of it (ids = attach
    index)."""
    solver: str                # "DFSPH" | "PBF"
    config: dict
    fluid_pos: np.ndarray      # (nf, 3) float32
    fluid_vel: np.ndarray      # (nf, 3) float32
    fluid_gid: np.ndarray      # (nf,) int64, ascending
    fluid_obj: np.ndarray      # (nf,) int32: ordinal of the particle's fluid object
    obj_count: np.ndarray      # (n_objects,) int64
    bnd_pos: np.ndarray        # (nb, 3) float32
    bnd_gid: np.ndarray        # (nb,) int64, ascending
    boundary_first: bool       # boundary ids all below the fluid ids
    h: float                   # support radius 4 r (FP32)


def scene_arrays(scene) -> SceneArrays:
    """Split a ``vtp.scenes.Scene`` (DFSPH or PBF) into fluid and boundary arrays with attach ids."""
    if scene.solver not in ("DFSPH", "PBF"):
        raise ValueError("domain decomposition runs DFSPH and PBF scenes")
    fp, fv, fg, fo, bp, bg, counts = [], [], [], [], [], [], []
    start = 0
    for o in scene.objects:
        ids = np.arange(start, start + o.n, dtype=np.int64)
        start += o.n
        if o.material == 0:
            fp.append(np.asarray(o.pos, np.float32))
            v = (np.asarray(o.velocity, np.float32) if o.velocity is not None
                 else np.tile(np.asarray(o.velocity_start, np.float32), (o.n, 1)))
            fv.append(v)
            fg.append(ids)
            fo.append(np.full(o.n, len(counts), np.int32))
            counts.append(o.n)
        else:
            bp.append(np.asarray(o.pos, np.float32))
            bg.append(ids)
    if not counts:
        raise ValueError("scene has no fluid")
    cat = lambda xs, shape, dt: np.concatenate(xs) if xs else np.zeros(shape, dt)
    fgid, bgid = cat(fg, (0,), np.int64), cat(bg, (0,), np.int64)
    if bgid.size and not (bgid.max() < fgid.min() or bgid.min() > fgid.max()):
        raise ValueError("domain decomposition needs fluid ids all below or all above the boundary ids")
    if start >= 2 ** 31:
        raise ValueError("more than 2^31 particles")
    req = scene.config[scene.solver]["Required"]
    h = float(np.float32(np.float32(req["particleRadius"]) * np.float32(4)))
    return SceneArrays(scene.solver, scene.config, cat(fp, (0, 3), np.float32), cat(fv, (0, 3), np.float32), fgid,
                       cat(fo, (0,), np.int32), np.asarray(counts, np.int64), cat(bp, (0, 3), np.float32), bgid,
                       bool(bgid.size and bgid.max() < fgid.min()), h)


@dataclass
class SlabPlan:
    """Slabs along `axis`: rank k owns [bounds[k-1], bounds[k]) with -inf / +inf at the ends."""
    axis: int
    bounds: tuple              # inner bounds, ascending, len = ranks - 1 (FP32 values)
    ghost: float

    @property
    def ranks(self) -> int:
        return len(self.bounds) + 1

    def slab(self, k: int) -> tuple:
        lo = -math.inf if k == 0 else self.bounds[k - 1]
        hi = math.inf if k == self.ranks - 1 else self.bounds[k]
        return lo, hi

    def owner(self, x):
        """Owning rank of each coordinate (torch tensor or numpy array)."""
        try:
            import torch
            if isinstance(x, torch.Tensor):
                b = torch.tensor(self.bounds, dtype=x.dtype, device=x.device)
                return torch.searchsorted(b, x.contiguous(), right=True)
        except ImportError:
            pass
        return np.searchsorted(np.asarray(self.bounds, dtype=np.asarray(x).dtype), x, side="right")


def plan_slabs(arrays: SceneArrays, ranks: int, axis: int | None = None) -> SlabPlan:
    """Equal fluid counts per slab at the start, along the longest axis of the simulation space."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    if axis is None:
        size = arrays.config[arrays.solver]["Required"]["simSpaceSize"]
        axis = int(np.argmax(np.asarray(size, np.float64)))
    x = np.sort(arrays.fluid_pos[:, axis])
    n = x.size
    bounds = tuple(float(x[min(n - 1, (k * n) // ranks)]) for k in range(1, ranks))
    return SlabPlan(axis, bounds, GHOST_MARGIN * arrays.h)


# ----------------------------------------------------------------------------- exchanges

class TorchComm:
    """Exchanges over the default torch.distributed group: point-to-point sends and receives
    and all-reduce (NCCL on CUDA tensors, gloo on CPU tensors)."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()

    def exchange(self, sends: dict, recvs: dict) -> dict:
        """sends {peer: tensor}; recvs {peer: tensor to fill}; both sides agree on the counts."""
        d = self.dist
        ops = [d.P2POp(d.isend, sends[q].contiguous(), q) for q in sorted(sends)]
        ops += [d.P2POp(d.irecv, recvs[q], q) for q in sorted(recvs)]
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()
        return recvs

    def counts(self, send_counts: list, device) -> list:
        """send_counts[q]: rows this rank sends to q; returns the rows each peer sends here."""
        import torch
        mine = torch.tensor(send_counts, dtype=torch.int64, device=device)
        parts = [torch.empty_like(mine) for _ in range(self.size)]
        self.dist.all_gather(parts, mine)
        return [int(p[self.rank].item()) for p in parts]

    def allreduce_sum(self, t):
        self.dist.all_reduce(t)
        return t

    def share(self, obj) -> list:
        """Every rank's `obj` (host objects, e.g. IPC handles), in rank order."""
        out = [None] * self.size
        self.dist.all_gather_object(out, obj)
        return out

    def fence(self, device):
        """Orders every rank's later stream work after every rank's earlier stream work (a
        one-element all-reduce on the stream)."""
        import torch
        if getattr(self, "_one", None) is None or self._one.device != device:
            self._one = torch.zeros(1, dtype=torch.float32, device=device)
        self.dist.all_reduce(self._one)

    def allreduce_max(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return t


class LoopbackHub:
    """Meeting point of the ranks of one process (threads)."""

    def __init__(self, ranks: int, timeout: float = 900.0):
        self.ranks = ranks
        self.barrier = threading.Barrier(ranks, timeout=timeout)
        self.box = {}


class LoopbackComm:
    """The exchanges of ``TorchComm`` between threads of one process.  Each rank's tensors are
    complete (its stream synchronised) before the others read them; all-reduce adds in rank
    order."""

    def __init__(self, hub: LoopbackHub, rank: int):
        self.hub = hub
        self.rank = rank
        self.size = hub.ranks

    @staticmethod
    def _settle(t):
        if t.is_cuda:
            import torch
            torch.cuda.current_stream(t.device).synchronize()

    def exchange(self, sends: dict, recvs: dict) -> dict:
        if self.size == 1:
            return recvs
        box, me = self.hub.box, self.rank
        for q, t in sends.items():
            self._settle(t)
            box[("x", me, q)] = t
        self.hub.barrier.wait()
        for q, buf in recvs.items():
            buf.copy_(box[("x", q, me)])
            self._settle(buf)
        self.hub.barrier.wait()
        for q in sends:
            del box[("x", me, q)]
        return recvs

    def counts(self, send_counts: list, device=None) -> list:
        if self.size == 1:
            return [0]
        box, me = self.hub.box, self.rank
        box[("c", me)] = list(send_counts)
        self.hub.barrier.wait()
        out = [box[("c", q)][me] for q in range(self.size)]
        self.hub.barrier.wait()
        return out

    def share(self, obj) -> list:
        if self.size == 1:
            return [obj]
        box, me = self.hub.box, self.rank
        box[("s", me)] = obj
        self.hub.barrier.wait()
        out = [box[("s", q)] for q in range(self.size)]
        self.hub.barrier.wait()
        return out

    def fence(self, device=None):
        if self.size == 1:
            return
        import torch
        if device is not None and device.type == "cuda":
            torch.cuda.current_stream(device).synchronize()
        self.hub.barrier.wait()

    def allreduce_max(self, t):
        if self.size == 1:
            return t
        box, me = self.hub.box, self.rank
        mine = t.clone()
        self._settle(mine)
        box[("m", me)] = mine
        self.hub.barrier.wait()
        total = box[("m", 0)].clone()
        for q in range(1, self.size):
            total = self._max(total, box[("m", q)])
        t.copy_(total)
        self._settle(t)
        self.hub.barrier.wait()
        return t

    @staticmethod
    def _max(a, b):
        import torch
        return torch.maximum(a, b)

    def allreduce_sum(self, t):
        if self.size == 1:   # nothing to add: no barrier, no stream synchronisation
            return t
        box, me = self.hub.box, self.rank
        mine = t.clone()
        self._settle(mine)
        box[("a", me)] = mine
        self.hub.barrier.wait()
        total = box[("a", 0)].clone()
        for q in range(1, self.size):
            total += box[("a", q)]
        t.copy_(total)
        self._settle(t)
        self.hub.barrier.wait()
        return t


# ----------------------------------------------------------------------------- library stages

class LibraryStages:
    """One rank's DFSPH or PBF stages on the sm_100a library; state in CUDA tensors (FP32)."""

    def __init__(self, config: dict, fluid_pos0: np.ndarray, bnd_pos: np.ndarray, bnd_gid: np.ndarray,
                 boundary_first: bool, capacity: int, n_objects: int):
        import torch
        from ._lib import check, lib
        self.torch = torch
        self.check = check
        self.L = lib()
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = torch.float32
        self.nobj = int(n_objects)
        self.pbf = "PBF" in config
        fp = np.ascontiguousarray(fluid_pos0, np.float32)
        bp = np.ascontiguousarray(bnd_pos, np.float32)
        bg = np.ascontiguousarray(bnd_gid, np.uint32)
        h = C.c_void_p()
        check(self.L.vtp_domain_create(json.dumps(config).encode(), fp.ctypes.data, fp.shape[0], bp.ctypes.data,
                                       bg.ctypes.data, bp.shape[0], int(boundary_first), int(capacity), self.nobj,
                                       C.byref(h)), "vtp_domain_create")
        self.h = h
        self.capacity = int(capacity)
        # The worker's kernels go to torch's current stream, in order with the exchanges; torch's
        # default stream is CUDA's legacy default stream (handle 0, which the library reads as
        # "its own stream"), passed as cudaStreamLegacy (0x1).
        handle = torch.cuda.current_stream().cuda_stream or 1
        check(self.L.vtp_domain_set_stream(h, C.c_void_p(handle)), "vtp_domain_set_stream")
        self.n_own = 0
        self.launches = 0   # library kernels launched by the stage calls so far

    def close(self):
        if self.h:
            self.L.vtp_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def empty(self, field: int, count: int):
        shape = {FIELD_KAPPA: (count,), FIELD_LAMBDA: (count,), FIELD_POSVEL: (count, 8)}.get(field, (count, 4))
        return self.torch.empty(shape, dtype=self.torch.float32, device=self.device)

    def load(self, n_own, pos, vel, gid, obj):
        t = self.torch
        n = pos.shape[0]
        if n > self.capacity:
            raise RuntimeError(f"domain rows {n} exceed the worker capacity {self.capacity}: "
                               "raise capacity_factor")
        self._pos = pos.to(t.float32).contiguous()
        self._vel = vel.to(t.float32).contiguous()
        self._gid = gid.to(t.int32).contiguous()
        self._obj = obj.to(t.int32).contiguous()
        self.n_own = int(n_own)
        self.check(self.L.vtp_domain_load(self.h, self.n_own, n - self.n_own, self._pos.data_ptr(),
                                          self._vel.data_ptr(), self._gid.data_ptr(), self._obj.data_ptr()),
                   "vtp_domain_load")
        self.launches += 1

    def vmax2(self) -> float:
        """Largest |v|^2 of the loaded owned rows (the adaptive step's own arithmetic)."""
        out = C.c_float()
        self.check(self.L.vtp_domain_owned_vmax2(self.h, C.byref(out)), "vtp_domain_owned_vmax2")
        self.launches += 1
        return float(out.value)

    def set_dt(self, dt: float):
        self.check(self.L.vtp_domain_set_dt(self.h, float(dt)), "vtp_domain_set_dt")

    def prepare(self):
        self.check(self.L.vtp_domain_prepare(self.h), "vtp_domain_prepare")
        # hash, 3 scan kernels, scatter, rank/reorder, lists, slot map (+ DFSPH: tiles, ratio/alpha)
        self.launches += 8 if self.pbf else 10

    # --- peer-store halos (DFSPH)
    def export_ipc(self) -> bytes:
        """CUDA IPC handles of the buffers peers store ghost values into, for another process."""
        buf = (C.c_ubyte * (8 * 64 + 12))()
        self.check(self.L.vtp_domain_export_ipc(self.h, C.cast(buf, C.c_void_p)), "vtp_domain_export_ipc")
        return bytes(buf)

    def link_local(self, peer: int, other: "LibraryStages"):
        self.check(self.L.vtp_domain_link_peer(self.h, int(peer), other.h), "vtp_domain_link_peer")

    def link_ipc(self, peer: int, handles: bytes):
        buf = (C.c_ubyte * len(handles)).from_buffer_copy(handles)
        self.check(self.L.vtp_domain_link_peer_ipc(self.h, int(peer), C.cast(buf, C.c_void_p)),
                   "vtp_domain_link_peer_ipc")

    def set_halo(self, on: bool):
        self.check(self.L.vtp_domain_set_halo(self.h, int(bool(on))), "vtp_domain_set_halo")

    def parity(self) -> tuple:
        out = (C.c_int32 * 3)()
        self.check(self.L.vtp_domain_buffer_parity(self.h, out), "vtp_domain_buffer_parity")
        return int(out[0]), int(out[1]), int(out[2])

    def rows(self, first: int, count: int):
        out = self.torch.empty(count, dtype=self.torch.int32, device=self.device)
        self.check(self.L.vtp_domain_rows(self.h, int(first), int(count), out.data_ptr()), "vtp_domain_rows")
        self.launches += 1
        return out

    def halo_targets(self, peer: int, slots, dst_rows, peer_capacity: int):
        s = slots.to(self.torch.int32).contiguous()
        d = dst_rows.to(self.torch.int32).contiguous()
        self.check(self.L.vtp_domain_halo_targets(self.h, int(peer), s.data_ptr(), d.data_ptr(), s.numel(),
                                                   int(peer_capacity)), "vtp_domain_halo_targets")
        self.launches += 1

    def pbf_lambda(self):
        self.check(self.L.vtp_domain_pbf_lambda(self.h), "vtp_domain_pbf_lambda")
        self.launches += 1

    def pbf_dx(self):
        self.check(self.L.vtp_domain_pbf_dx(self.h), "vtp_domain_pbf_dx")
        self.launches += 1

    def pbf_xsph(self):
        self.check(self.L.vtp_domain_pbf_xsph(self.h), "vtp_domain_pbf_xsph")
        self.launches += 1

    def solve_begin(self, which: int):
        self.check(self.L.vtp_domain_solve_begin(self.h, int(which)), "vtp_domain_solve_begin")
        self.launches += 2

    def solve_a(self):
        sums = self.torch.empty(self.nobj, dtype=self.torch.float64, device=self.device)
        self.check(self.L.vtp_domain_solve_a(self.h, sums.data_ptr()), "vtp_domain_solve_a")
        self.launches += 3
        return sums

    def solve_b(self):
        self.check(self.L.vtp_domain_solve_b(self.h), "vtp_domain_solve_b")
        self.launches += 1

    def forces(self):
        self.check(self.L.vtp_domain_forces(self.h), "vtp_domain_forces")
        self.launches += 2

    def tension(self):
        self.check(self.L.vtp_domain_tension(self.h), "vtp_domain_tension")
        self.launches += 1

    def finalize(self):
        self.check(self.L.vtp_domain_finalize(self.h), "vtp_domain_finalize")
        self.launches += 1

    def pack(self, field: int, slots):
        s = slots.to(self.torch.int32).contiguous()
        out = self.empty(field, s.numel())
        self.check(self.L.vtp_domain_pack(self.h, field, s.data_ptr(), s.numel(), out.data_ptr()),
                   "vtp_domain_pack")
        self.launches += 1
        return out

    def unpack(self, field: int, first: int, values):
        v = values.contiguous()
        self.check(self.L.vtp_domain_unpack(self.h, field, int(first), v.shape[0], v.data_ptr()),
                   "vtp_domain_unpack")
        self.launches += 1

    def read(self):
        t = self.torch
        pos = t.empty((self.n_own, 3), dtype=t.float32, device=self.device)
        vel = t.empty((self.n_own, 3), dtype=t.float32, device=self.device)
        self.check(self.L.vtp_domain_read(self.h, pos.data_ptr(), vel.data_ptr()), "vtp_domain_read")
        self.launches += 1
        return pos, vel


# ----------------------------------------------------------------------------- one rank

class DomainRank:
    """One rank of a decomposed DFSPH or PBF scene: owns its slab's fluid particles and drives its
    worker's stages with the exchanges of the module docstring."""

    def __init__(self, arrays: SceneArrays, plan: SlabPlan, comm, make_stages=LibraryStages,
                 capacity_factor: float = 2.0, speculate: bool = True, halo: str = "auto"):
        import torch
        self.torch = torch
        self.speculate = speculate
        self.a = arrays
        self.kind = arrays.solver
        self.plan = plan
        self.comm = comm
        self.rank = comm.rank
        if plan.ranks != comm.size:
            raise ValueError(f"plan has {plan.ranks} slabs for {comm.size} ranks")
        req = arrays.config[self.kind]["Required"]
        opt = arrays.config[self.kind].get("Optional", {})
        ext = arrays.config.get("B200", {})
        self.dt = float(np.float32(req["timeStep"]))
        if self.kind == "DFSPH":
            # the adaptive step ("cfl"): one max all-reduce of the owned rows' |v|^2 per substep
            self.cfl = float(np.float32(ext.get("cfl", 0.0)))
            self.diameter = np.float32(np.float32(2) * np.float32(req["particleRadius"]))
            self.dts = []
            self.thr = (float(np.float32(req["divFreeThreshold"])), float(np.float32(req["incompThreshold"])))
            self.force = (int(ext.get("forceDivIterations", 0)), int(ext.get("forceIncompIterations", 0)))
            self.force_seq = [tuple(int(v) for v in p) for p in ext.get("forceIterationsPerTick", [])]
            self.gamma = float(np.float32(req["surfaceTensionCoefficient"]))
            reach = 0.0
        else:
            # PBF builds its lists on the positions after the external force, x + dt (v + g dt):
            # ghosts are chosen on the loaded positions with twice the largest such move added
            # (`_reach`), within a fixed half-h allowance the boundary band is widened by.
            self.iterations = int(req["iterationNum"])
            g = opt.get("gravity", [0.0, -9.8, 0.0]) if opt.get("enable", False) else [0.0, -9.8, 0.0]
            self.g_norm = float(np.linalg.norm(np.asarray(g, np.float64)))
            reach = 0.5 * arrays.h
        self.reach_limit = reach
        self.inv_count = [1.0 / float(c) for c in arrays.obj_count]
        self.max_iters = 101
        ax, w = plan.axis, plan.ghost
        lo, hi = plan.slab(self.rank)
        fx = arrays.fluid_pos[:, ax]
        own = plan.owner(fx) == self.rank
        near = (fx >= lo - w - 2 * reach) & (fx < hi + w + 2 * reach)
        bx = arrays.bnd_pos[:, ax]
        band = (bx >= lo - 2 * w - reach) & (bx < hi + 2 * w + reach)
        n0 = int(near.sum())
        cap = min(max(int(capacity_factor * n0), n0 + 4096), 1 << 24)
        self.stages = make_stages(arrays.config, arrays.fluid_pos[near], arrays.bnd_pos[band], arrays.bnd_gid[band],
                                  arrays.boundary_first, cap, len(arrays.obj_count))
        dev, dt = self.stages.device, self.stages.dtype
        self.pos = torch.as_tensor(arrays.fluid_pos[own], device=dev).to(dt)
        self.vel = torch.as_tensor(arrays.fluid_vel[own], device=dev).to(dt)
        self.gid = torch.as_tensor(arrays.fluid_gid[own], device=dev)
        self.obj = torch.as_tensor(arrays.fluid_obj[own], device=dev)
        self.substeps = 0
        self.iters = []            # (divergence, density) iterations per substep (PBF: (iterations, 0))
        self.residuals = []
        self.crashed = False
        # Halo transport: "peer" (library stages, at most 8 ranks): the owners' stage kernels
        # store ghost values straight into the peers' ghost rows and a fence orders the peers'
        # next stage; "exchange": pack, send / receive, unpack.
        if halo == "auto":
            halo = "peer" if (hasattr(self.stages, "link_local") and 1 < comm.size <= 8
                              and (isinstance(comm, LoopbackComm) or self._nccl())) else "exchange"
        if halo not in ("peer", "exchange"):
            raise ValueError("halo must be 'auto', 'peer' or 'exchange'")
        self.peer_mode = halo == "peer" and comm.size > 1
        if self.peer_mode:
            self._link_peers()

    def _adaptive_step(self):
        """dt = min(timeStep, cfl 2r / max |v|) over all ranks' fluid, at least timeStep 1e-4,
        in FP32 with the operations of the solver's adaptive step (k_cfl_step); timeStep when
        the fluid is at rest."""
        t = self.torch
        v2 = t.tensor([self.stages.vmax2()], dtype=t.float32, device=self.pos.device)
        v2 = np.float32(self.comm.allreduce_max(v2).cpu().numpy()[0])
        f32 = np.float32
        dt_max = f32(self.dt)
        vmax = np.sqrt(v2)
        dt = dt_max
        if vmax > 0:
            dt = max(min(dt_max, f32(f32(self.cfl) * self.diameter) / vmax), f32(dt_max * f32(1e-4)))
        self.stages.set_dt(float(dt))
        self.dts.append(float(dt))

    def _nccl(self) -> bool:
        try:
            return self.comm.dist.get_backend() == "nccl"
        except Exception:
            return False

    def _link_peers(self):
        """Map every peer worker's ghost-target buffers: directly within one process, through
        CUDA IPC handles across processes."""
        st = self.stages
        if isinstance(self.comm, LoopbackComm):
            workers = self.comm.share(st)
            for q in self._peers():
                st.link_local(q, workers[q])
            self.peer_cap = [w.capacity for w in workers]
        else:
            shared = self.comm.share((st.export_ipc(), st.capacity))
            for q in self._peers():
                st.link_ipc(q, shared[q][0])
            self.peer_cap = [c for _, c in shared]
        st.set_halo(True)

    def _halo_targets(self):
        """Peer mode, after prepare: the rows this rank holds each peer's ghosts at go to that
        peer; the rows each peer holds this rank's sends at come back and become targets."""
        t = self.torch
        dev = self.pos.device
        sends = {q: self.stages.rows(self.ghost_first[q], self.recv_count[q]) for q in self.ghost_first}
        recvs = {q: t.empty(idx.numel(), dtype=t.int32, device=dev) for q, idx in self.send_slots.items()
                 if idx.numel()}
        self.comm.exchange(sends, recvs)
        for q, rows in recvs.items():
            self.stages.halo_targets(q, self.send_slots[q], rows, self.peer_cap[q])
        if self.substeps == 0:
            par = self.comm.share(self.stages.parity())
            if any(p != par[0] for p in par):
                raise RuntimeError(f"workers' buffer parities differ: {par}")

    # --- exchanges
    def _peers(self):
        return [q for q in range(self.comm.size) if q != self.rank]

    def _send_rows(self, index_of: dict, arrays: list) -> list:
        """Send rows index_of[q] of each array to q; returns, per array, the received blocks in
        rank order."""
        t = self.torch
        counts = [0] * self.comm.size
        for q, idx in index_of.items():
            counts[q] = int(idx.numel())
        got = self.comm.counts(counts, self.pos.device)
        out = []
        for arr in arrays:
            sends = {q: arr[idx] for q, idx in index_of.items() if idx.numel()}
            recvs = {q: t.empty((got[q],) + tuple(arr.shape[1:]), dtype=arr.dtype, device=arr.device)
                     for q in self._peers() if got[q]}
            self.comm.exchange(sends, recvs)
            out.append([recvs[q] for q in sorted(recvs)])
        return out, got

    def _migrate(self):
        if self.comm.size == 1:
            return
        t = self.torch
        dest = self.plan.owner(self.pos[:, self.plan.axis])
        index_of = {q: t.nonzero(dest == q).flatten() for q in self._peers()}
        (pos_in, vel_in, gid_in, obj_in), _ = self._send_rows(index_of, [self.pos, self.vel, self.gid, self.obj])
        keep = dest == self.rank
        self.pos = t.cat([self.pos[keep]] + pos_in)
        self.vel = t.cat([self.vel[keep]] + vel_in)
        self.gid = t.cat([self.gid[keep]] + gid_in)
        self.obj = t.cat([self.obj[keep]] + obj_in)

    def _reach(self) -> float:
        """PBF: the largest distance a particle moves under the external force this substep,
        dt (max |v| + |g| dt) over all ranks (one max all-reduce), with a margin."""
        t = self.torch
        v = self.vel.norm(dim=1).max() if self.vel.shape[0] else t.zeros((), dtype=self.vel.dtype,
                                                                           device=self.vel.device)
        vmax = float(self.comm.allreduce_max(v.reshape(1).to(t.float64)).cpu().numpy()[0])
        d = 1.01 * self.dt * (vmax + self.g_norm * self.dt) + 1e-6 * self.a.h
        if d > self.reach_limit:
            raise RuntimeError(f"a particle moves {d:.3g} under the external force in one substep, more than the "
                               f"decomposition's allowance {self.reach_limit:.3g} (h / 2)")
        return d

    def _ghosts(self, reach: float = 0.0):
        t = self.torch
        if self.comm.size == 1:
            self.send_slots, self.recv_count, self.ghost_first = {}, [0], {}
            return self.pos, self.vel, self.gid, self.obj
        x = self.pos[:, self.plan.axis]
        w = self.plan.ghost + 2 * reach
        self.send_slots = {}
        for q in self._peers():
            lo, hi = self.plan.slab(q)
            self.send_slots[q] = t.nonzero((x >= lo - w) & (x < hi + w)).flatten()
        (gpos, gvel, ggid), got = self._send_rows(self.send_slots, [self.pos, self.vel, self.gid])
        self.recv_count = got
        self.ghost_first = {}
        first = self.pos.shape[0]
        for q in self._peers():
            if got[q]:
                self.ghost_first[q] = first
                first += got[q]
        n_ghost = first - self.pos.shape[0]
        zeros = t.zeros(n_ghost, dtype=self.obj.dtype, device=self.obj.device)
        return t.cat([self.pos] + gpos), t.cat([self.vel] + gvel), t.cat([self.gid] + ggid), t.cat([self.obj, zeros])

    def _exchange(self, field: int):
        if self.peer_mode:
            # the stage stored the ghost values into the peers itself; order the peers' next
            # stage after the stores (after solve_b the residual all-reduce does it)
            if field != FIELD_VADV:
                self.comm.fence(self.pos.device)
            return
        sends = {q: self.stages.pack(field, idx) for q, idx in self.send_slots.items() if idx.numel()}
        recvs = {q: self.stages.empty(field, self.recv_count[q]) for q in self.ghost_first}
        self.comm.exchange(sends, recvs)
        for q, buf in recvs.items():
            self.stages.unpack(field, self.ghost_first[q], buf)

    def _fetch(self, t):
        """Start copying `t` to the host; returns a function that waits for the copy (and only
        for it) and gives the values as a numpy array."""
        if not t.is_cuda:
            a = t.numpy().copy()
            return lambda: a
        torch = self.torch
        if getattr(self, "_host", None) is None or self._host.numel() < t.numel():
            self._host = torch.empty(max(t.numel(), 16), dtype=t.dtype, pin_memory=True)
        h = self._host[: t.numel()]
        h.copy_(t, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()

        def wait():
            ev.synchronize()
            return h.numpy().copy()
        return wait

    def _solve(self, which: int):
        """One pressure solve: the loop of vfsph_div / vfsph_incomp (DFSPHSolver.cpp:355-391) with
        the residual summed over ranks; every rank takes the same decision from the same sum.

        With `speculate` the next iteration's solve_a (and its kappa exchange) is queued before
        the host waits for the summed residual, so the GPU keeps working through the host round
        trip; when the test stops the solve, that pass is dropped: solve_a writes only delta,
        kappa and the packed {x, kappa} rows, which the next stage rewrites before reading."""
        st = self.stages
        st.solve_begin(which)
        force = self.force[which]
        if self.substeps < len(self.force_seq):
            force = self.force_seq[self.substeps][which]
        it = 0
        sums = st.solve_a()
        self._exchange(FIELD_KAPPA)
        while True:
            it += 1
            st.solve_b()
            self._exchange(FIELD_VADV)
            result = self._fetch(self.comm.allreduce_sum(sums))
            if self.speculate:
                sums = st.solve_a()
                self._exchange(FIELD_KAPPA)
            tot = result()
            acc = 0.0
            for o, v in enumerate(tot):
                acc += float(v) * self.inv_count[o]
            residual = acc / len(tot)
            if force > 0:
                stop = it >= force
            else:
                stop = residual < self.thr[which] or it > self.max_iters - 1
            if not math.isfinite(residual):
                raise FloatingPointError(f"non-finite pressure-solve residual at substep {self.substeps}")
            if stop:
                if force == 0 and it > self.max_iters - 1:
                    self.crashed = True
                return it, residual
            if not self.speculate:
                sums = st.solve_a()
                self._exchange(FIELD_KAPPA)

    # --- the substep
    def step(self, n: int = 1):
        for _ in range(n):
            self.substep()

    def substep(self):
        if self.kind == "PBF":
            return self._pbf_substep()
        if self.crashed:
            raise RuntimeError("DFSPHSolver is crashed.")
        st = self.stages
        if self.substeps > 0:
            self._migrate()
        pos, vel, gid, obj = self._ghosts()
        st.load(self.pos.shape[0], pos, vel, gid, obj)
        if self.cfl > 0:
            self._adaptive_step()
        st.prepare()
        if self.peer_mode:
            self._halo_targets()
        div = self._solve(0)
        st.forces()
        if self.gamma != 0.0:
            self._exchange(FIELD_NORMAL)
            st.tension()
        self._exchange(FIELD_VEL)
        inc = self._solve(1)
        st.finalize()
        self.pos, self.vel = st.read()
        self.iters.append((div[0], inc[0]))
        self.residuals.append((div[1], inc[1]))
        self.substeps += 1

    def _pbf_substep(self):
        """PBFSolver::tick (PBFSolver.cpp:326-376) over the rank's rows: the external force in
        the sort, `iterationNum` constraint iterations (lambda to the ghosts after each lambda
        pass, positions and velocities after each correction pass), XSPH."""
        st = self.stages
        if self.substeps > 0:
            self._migrate()
        reach = self._reach() if self.comm.size > 1 else 0.0
        pos, vel, gid, obj = self._ghosts(reach)
        st.load(self.pos.shape[0], pos, vel, gid, obj)
        st.prepare()
        if self.peer_mode:
            self._halo_targets()
        for _ in range(self.iterations):
            st.pbf_lambda()
            self._exchange(FIELD_LAMBDA)
            st.pbf_dx()
            self._exchange(FIELD_POSVEL)
        st.pbf_xsph()
        self.pos, self.vel = st.read()
        self.iters.append((self.iterations, 0))
        self.residuals.append((0.0, 0.0))
        self.substeps += 1

    def timed_steps(self, n: int) -> float:
        """n substeps; milliseconds between CUDA events recorded on this rank's stream before and
        after them (host time with CPU stages)."""
        t = self.torch
        if not self.pos.is_cuda:
            import time
            t0 = time.perf_counter()
            self.step(n)
            return 1e3 * (time.perf_counter() - t0)
        a, b = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        t.cuda.current_stream().synchronize()
        a.record()
        self.step(n)
        b.record()
        b.synchronize()
        return a.elapsed_time(b)

    def state(self) -> dict:
        """Owned particles: scene-wide ids, positions, velocities (host numpy)."""
        return {"gid": self.gid.cpu().numpy(), "pos": self.pos.cpu().numpy(), "vel": self.vel.cpu().numpy(),
                "iters": list(self.iters), "residuals": list(self.residuals)}

    def close(self):
        close = getattr(self.stages, "close", None)
        if close:
            close()


def merge_states(arrays: SceneArrays, states: list) -> dict:
    """Every rank's owned rows in the scene's fluid order (ascending id); each particle exactly
    once."""
    gid = np.concatenate([s["gid"] for s in states])
    order = np.argsort(gid, kind="stable")
    if not np.array_equal(gid[order], arrays.fluid_gid):
        raise RuntimeError("fluid particles lost or duplicated across domains")
    return {"pos": np.concatenate([s["pos"] for s in states])[order],
            "vel": np.concatenate([s["vel"] for s in states])[order],
            "owned": [len(s["gid"]) for s in states],
            "iters": states[0]["iters"], "residuals": states[0]["residuals"]}


def local_ranks(arrays: SceneArrays, plan: SlabPlan, body, make_stages=LibraryStages,
                capacity_factor: float = 2.0, speculate: bool = True, halo: str = "auto") -> list:
    """Run ``body(rank)`` for every domain of `plan` inside this process, one thread (and, with
    the library's stages, one CUDA stream) per domain, exchanging through ``LoopbackComm``;
    returns the bodies' results in rank order.  A failure on one domain releases the others
    and is raised here."""
    import torch
    hub = LoopbackHub(plan.ranks)
    results = [None] * plan.ranks
    errors = []
    use_cuda = make_stages is LibraryStages

    ranks = [None] * plan.ranks

    def work(k):
        try:
            ctx = torch.cuda.stream(torch.cuda.Stream()) if use_cuda else _null()
            with ctx:
                ranks[k] = DomainRank(arrays, plan, LoopbackComm(hub, k), make_stages, capacity_factor, speculate,
                                      halo)
                results[k] = body(ranks[k])
        except BaseException as e:   # wake the other domains, report the first failure
            errors.append(e)
            hub.barrier.abort()

    threads = [threading.Thread(target=work, args=(k,), daemon=True) for k in range(plan.ranks)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    # Workers are released only once every domain has stopped: with peer-store halos a
    # domain's kernels write into the others' buffers.
    if use_cuda:
        torch.cuda.synchronize()
    for r in ranks:
        if r is not None:
            r.close()
    if errors:
        real = [e for e in errors if not isinstance(e, threading.BrokenBarrierError)]
        raise (real or errors)[0]
    return results


def run_local(scene, ranks: int, steps: int, make_stages=LibraryStages, axis: int | None = None,
              capacity_factor: float = 2.0, extra: dict | None = None, speculate: bool = True,
              plan: SlabPlan | None = None, halo: str = "auto") -> dict:
    """Run `scene` decomposed into `ranks` slabs inside this process (``local_ranks``) for
    `steps` substeps and merge the ranks' owned particles into the scene's fluid order.
    `plan` replaces the quantile slabs of ``plan_slabs``."""
    arrays = scene_arrays(scene)
    if extra:
        arrays.config = json.loads(json.dumps(arrays.config))
        arrays.config["B200"] = dict(extra)
    plan = plan or plan_slabs(arrays, ranks, axis)

    def body(rank):
        rank.step(steps)
        return rank.state()

    out = merge_states(arrays, local_ranks(arrays, plan, body, make_stages, capacity_factor, speculate, halo))
    out["plan"] = plan
    return out


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False
