"""Host-side mirror of the reference's solver plugin interface over the C ABI.

Method names, argument meaning and boolean returns follow the reference's
``VT_Physics::Solver`` (Simulator/Runtime/Include/Framework/Solver.hpp:27-62),
``SolverManager::createSolver`` (Simulator/Runtime/Source/Manager/SolverManager.cpp:19-40)
and the ``Object`` API (Simulator/Runtime/Include/Framework/Object.hpp:15-48) the
examples use (Examples/*/Usage-1.cpp).  Failures return False and keep the
message in ``last_error`` as the reference logs it; ``strict=True`` raises.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Iterable

import numpy as np

from . import scenes
from ._lib import FIELDS, SOLVER_TYPES, VtpConservation, VtpError, VtpKernelTime, VtpStats, check, lib

PBF, DFSPH, IMM, IMMCT = 0, 1, 2, 3
EPM_FLUID, EPM_BOUNDARY = 0, 1

Particle_Common, Particle_Sphere, Particle_Cube, Particle_Cylinder, Particle_Plane, Particle_Box = range(6)


class Object:
    """Particle object: geometry config + solver-specific component config (Object.hpp:15-48)."""

    _next_id = 0

    def __init__(self, obj_type: int = Particle_Common, name: str | None = None):
        Object._next_id += 1
        self._id = Object._next_id
        self._name = name or f"obj_{self._id}"
        self._type = obj_type
        self._cfg: dict = {"epmMaterial": 255, "particleRadius": 0.05}
        self._solver_cfg: dict = {}
        self.pos = np.zeros((0, 3), np.float32)
        self.velocity: np.ndarray | None = None

    def getID(self):
        return self._id

    def getName(self):
        return self._name

    def rename(self, name):
        self._name = name

    def getObjectComponentConfig(self) -> dict:
        return self._cfg

    def attachSpecificSolverObjectComponentConfig(self, cfg: dict):
        self._solver_cfg = dict(cfg)

    def getSolverObjectComponentConfig(self) -> dict:
        return self._solver_cfg

    def update(self) -> bool:
        """Generate the particles of a Cube / Box object (ModelHandler.cpp:43-67, 124-154)."""
        c = self._cfg
        if self._type == Particle_Cube:
            self.pos = scenes.cube(c["particleRadius"], c["lb"], c["size"])
        elif self._type == Particle_Box:
            self.pos = scenes.box(c["particleRadius"], c["lb"], c["size"], int(c["layerNum"]))
        elif self._type == Particle_Common:
            pass  # positions are set directly (ParticleGeometryComponent::pos)
        else:
            raise NotImplementedError("only Particle_Common / Particle_Cube / Particle_Box are generated here")
        return True

    def getElements(self) -> np.ndarray:
        return np.ascontiguousarray(self.pos, dtype=np.float32).reshape(-1)


class ObjectManager:
    def createObject(self, obj_type: int) -> Object:
        return Object(obj_type)


class Solver:
    """Base of the drop-in solvers; owns one C-ABI handle."""

    solver_type = -1
    key = ""

    def __init__(self, strict: bool = False):
        self.strict = strict
        self.last_error = ""
        self._h = C.c_void_p()
        check(lib().vtp_solver_create(self.solver_type, C.byref(self._h)), "vtp_solver_create")
        self._n = None

    # -- error handling ---------------------------------------------------
    def _call(self, code: int, where: str) -> bool:
        if code == 0:
            return True
        self.last_error = lib().vtp_last_error().decode()
        if self.strict:
            raise VtpError(code, where, self.last_error)
        self._last_code = code
        return False

    # -- reference interface ---------------------------------------------
    def getSolverConfigTemplate(self) -> dict:
        need = C.c_size_t()
        check(lib().vtp_solver_get_config(self._h, None, 0, C.byref(need)), "get_config")
        buf = C.create_string_buffer(need.value)
        check(lib().vtp_solver_get_config(self._h, buf, need.value, None), "get_config")
        return json.loads(buf.value.decode())

    def setConfig(self, config: dict) -> bool:
        return self._call(lib().vtp_solver_set_config(self._h, json.dumps(config).encode()), "setConfig")

    def setConfigByFile(self, path: str) -> bool:
        with open(path) as f:
            return self.setConfig(json.load(f))

    def getSolverObjectComponentConfigTemplate(self) -> dict:
        return {"solverType": self.solver_type, "exportFlag": False, "velocityStart": [0, 0, 0],
                "colorStart": [0, 1, 0]}

    def addScene(self, config: dict) -> int:
        """Add an independent scene (same shared parameters, own domain and gravity); returns its index."""
        idx = C.c_uint32()
        check(lib().vtp_solver_add_scene(self._h, json.dumps(config).encode(), C.byref(idx)), "addScene")
        return idx.value

    def attachObject(self, obj: Object, scene: int = 0) -> bool:
        pos = np.ascontiguousarray(obj.pos, dtype=np.float32).reshape(-1, 3)
        vel = None
        if obj.velocity is not None:
            vel = np.ascontiguousarray(obj.velocity, dtype=np.float32).reshape(-1, 3)
            assert vel.shape == pos.shape
        meta = {"name": obj.getName(), "ObjectComponentConfig": obj.getObjectComponentConfig(),
                "SolverObjectComponentConfig": obj.getSolverObjectComponentConfig()}
        if scene:
            meta["scene"] = int(scene)
        code = lib().vtp_solver_attach_object(self._h, pos.ctypes.data, pos.shape[0],
                                              None if vel is None else vel.ctypes.data,
                                              json.dumps(meta).encode())
        return self._call(code, "attachObject")

    def attachObjects(self, objs: Iterable[Object]) -> bool:
        return all(self.attachObject(o) for o in objs)

    def initialize(self) -> bool:
        return self._call(lib().vtp_solver_initialize(self._h), "initialize")

    def run(self) -> bool:
        return self._call(lib().vtp_solver_run(self._h), "run")

    def tickNsteps(self, n: int) -> bool:
        return self._call(lib().vtp_solver_tick_n_steps(self._h, int(n)), "tickNsteps")

    def reset(self) -> bool:
        return self._call(lib().vtp_solver_reset(self._h), "reset")

    def destroy(self):
        if self._h:
            lib().vtp_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- extensions used by tests and benchmarks ---------------------------
    def counts(self) -> dict:
        a, b, c, d = (C.c_uint32() for _ in range(4))
        check(lib().vtp_solver_particle_counts(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)), "counts")
        return {"total": a.value, "fluid": b.value, "boundary": c.value, "phases": d.value}

    def get_field(self, name: str) -> np.ndarray:
        fid, width = FIELDS[name]
        cnt = self.counts()
        if width < 0:
            width = -width * cnt["phases"]
        dtype = np.int32 if name == "mat" else np.float32
        out = np.empty((cnt["total"], width), dtype=dtype)
        check(lib().vtp_solver_get_field(self._h, fid, out.ctypes.data, out.nbytes), f"get_field({name})")
        return out if width > 1 else out[:, 0]

    def set_field(self, name: str, arr: np.ndarray):
        fid, width = FIELDS[name]
        a = np.ascontiguousarray(arr, dtype=np.float32)
        check(lib().vtp_solver_set_field(self._h, fid, a.ctypes.data, a.nbytes), f"set_field({name})")

    def set_field_ptr(self, name: str, ptr: int, nbytes: int):
        """Upload from a raw host pointer (e.g. pinned memory)."""
        fid, _ = FIELDS[name]
        check(lib().vtp_solver_set_field(self._h, fid, ptr, nbytes), f"set_field({name})")

    def get_field_ptr(self, name: str, ptr: int, nbytes: int):
        fid, _ = FIELDS[name]
        check(lib().vtp_solver_get_field(self._h, fid, ptr, nbytes), f"get_field({name})")

    def set_field_range_ptr(self, name: str, first: int, count: int, ptr: int, nbytes: int):
        """Upload particles [first, first + count) (attach order) from a raw host pointer."""
        fid, _ = FIELDS[name]
        check(lib().vtp_solver_set_field_range(self._h, fid, int(first), int(count), ptr, nbytes),
              f"set_field_range({name})")

    def get_field_range_ptr(self, name: str, first: int, count: int, ptr: int, nbytes: int):
        fid, _ = FIELDS[name]
        check(lib().vtp_solver_get_field_range(self._h, fid, int(first), int(count), ptr, nbytes),
              f"get_field_range({name})")

    def set_state_range_ptr(self, first: int, count: int, pos_ptr: int, vel_ptr: int):
        """Upload positions and velocities of particles [first, first + count) from raw host pointers."""
        check(lib().vtp_solver_set_state_range(self._h, int(first), int(count), pos_ptr, vel_ptr), "set_state_range")

    def get_state_range_ptr(self, first: int, count: int, pos_ptr: int, vel_ptr: int):
        check(lib().vtp_solver_get_state_range(self._h, int(first), int(count), pos_ptr, vel_ptr), "get_state_range")

    def step_state_range_ptr(self, first: int, count: int, pos_in: int, vel_in: int, n: int, pos_out: int,
                             vel_out: int) -> bool:
        """One host-driven frame in one call: upload the positions and velocities of particles
        [first, first + count), advance n substeps, read them back (raw host pointers; in and out
        may be the same buffers).  False, with last_error, when the substeps fail as tickNsteps
        does."""
        return self._call(lib().vtp_solver_step_state_range(self._h, int(first), int(count), pos_in, vel_in, int(n),
                                                            pos_out, vel_out), "step_state_range")

    def step_state_ranges_ptr(self, ranges, pos_in: int, vel_in: int, n: int, pos_out: int, vel_out: int) -> bool:
        """step_state_range_ptr for several attach-order ranges [(first, count), ...], ascending and
        disjoint, whose particles the host buffers hold back to back."""
        firsts = (C.c_uint32 * max(len(ranges), 1))(*[int(f) for f, _ in ranges])
        counts = (C.c_uint32 * max(len(ranges), 1))(*[int(c) for _, c in ranges])
        return self._call(lib().vtp_solver_step_state_ranges(self._h, len(ranges), C.cast(firsts, C.c_void_p),
                                                             C.cast(counts, C.c_void_p), pos_in, vel_in, int(n),
                                                             pos_out, vel_out), "step_state_ranges")

    def get_field_range(self, name: str, first: int, count: int) -> np.ndarray:
        fid, width = FIELDS[name]
        w = width if isinstance(width, int) and width > 0 else 1
        out = np.empty((count, w) if w > 1 else count, np.float32)
        self.get_field_range_ptr(name, first, count, out.ctypes.data, out.nbytes)
        return out

    def get_neighbors(self, max_nbr: int):
        n = self.counts()["total"]
        cnt = np.empty(n, np.uint32)
        nb = np.empty((n, max_nbr), np.uint32)
        check(lib().vtp_solver_get_neighbors(self._h, cnt.ctypes.data, nb.ctypes.data, max_nbr), "get_neighbors")
        return cnt, nb

    def get_sorted_order(self):
        n = self.counts()["total"]
        ids = np.empty(n, np.uint32)
        keys = np.empty(n, np.uint32)
        check(lib().vtp_solver_get_sorted_order(self._h, ids.ctypes.data, keys.ctypes.data), "get_sorted_order")
        return ids, keys

    def stats(self) -> dict:
        s = VtpStats()
        check(lib().vtp_solver_get_stats(self._h, C.byref(s)), "get_stats")
        return s.as_dict()

    def conservation(self, scene: int = -1) -> dict:
        """FP64 device sums of the fluid: mass, momentum, kinetic energy, mean density
        error and (IMM / IMM-CT) per-phase mass, of one scene or (-1) all."""
        c = VtpConservation()
        check(lib().vtp_solver_get_conservation(self._h, int(scene), C.byref(c)), "get_conservation")
        return c.as_dict()

    def scene_stats(self, scene: int) -> dict:
        s = VtpStats()
        check(lib().vtp_solver_get_scene_stats(self._h, int(scene), C.byref(s)), "get_scene_stats")
        return s.as_dict()

    def stage_times(self):
        a = (C.c_float * 3)()
        check(lib().vtp_solver_get_stage_times(self._h, a), "stage_times")
        return list(a)

    def profile_kernels(self, n: int) -> dict:
        """Run n substeps with per-kernel CUDA events; {name: (total_ms, launches)}."""
        cap = 64
        arr = (VtpKernelTime * cap)()
        cnt = C.c_uint32()
        check(lib().vtp_solver_profile_kernels(self._h, int(n), arr, cap, C.byref(cnt)), "profile_kernels")
        return {arr[k].name.decode(): (arr[k].total_ms, arr[k].launches) for k in range(cnt.value)}

    def launch_count(self) -> int:
        v = C.c_uint64()
        check(lib().vtp_solver_get_launch_count(self._h, C.byref(v)), "launch_count")
        return v.value


class HostBuffer:
    """Page-locked host array from vtp_host_alloc (float32, shape (n, 3) by default)."""

    def __init__(self, shape, dtype=np.float32):
        self.shape = tuple(shape)
        self.dtype = np.dtype(dtype)
        nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = C.c_void_p()
        check(lib().vtp_host_alloc(nbytes, C.byref(p)), "host_alloc")
        self._p = p
        self.nbytes = nbytes
        buf = (C.c_char * nbytes).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype).reshape(self.shape)

    @property
    def ptr(self) -> int:
        return self._p.value

    def free(self):
        if self._p is not None and self._p.value:
            self.array = None
            lib().vtp_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PBFSolver(Solver):
    solver_type = PBF
    key = "PBF"


class DFSPHSolver(Solver):
    solver_type = DFSPH
    key = "DFSPH"


class IMMSolver(Solver):
    solver_type = IMM
    key = "IMM"


class IMMCTSolver(Solver):
    solver_type = IMMCT
    key = "IMMCT"


_CLASSES = {PBF: PBFSolver, DFSPH: DFSPHSolver, IMM: IMMSolver, IMMCT: IMMCTSolver}


class SolverManager:
    """SolverManager::createSolver (SolverManager.cpp:19-40)."""

    def createSolver(self, solver_type: int, strict: bool = False) -> Solver:
        return _CLASSES[solver_type](strict=strict)


def tick_together(solvers, n: int) -> bool:
    """Advance every solver `n` substeps with their CUDA streams running at the same time.

    Each solver runs on its own stream and its tick call holds the calling thread until its
    substeps finish, so one host thread per solver submits them (the library's calls release
    the interpreter lock) and independent solvers - the PBF and DFSPH batches of a mixed set
    of scenes, say - overlap on the GPU.  Returns whether every solver advanced; the first
    exception a strict solver raises is raised here after all threads have finished."""
    import threading
    done = [False] * len(solvers)
    errors = []

    def run(k):
        try:
            done[k] = bool(solvers[k].tickNsteps(n))
        except BaseException as e:
            errors.append(e)

    threads = [threading.Thread(target=run, args=(k,)) for k in range(len(solvers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return all(done)


def _attach_scene_objects(s: Solver, scene: "scenes.Scene", index: int = 0):
    for o in scene.objects:
        obj = Object(Particle_Common, o.name)
        obj.getObjectComponentConfig()["epmMaterial"] = o.material
        sc = {"solverType": s.solver_type, "exportFlag": o.export_flag, "velocityStart": list(o.velocity_start),
              "colorStart": list(o.color_start)}
        if o.phase_fraction is not None:
            sc["phaseFraction"] = list(o.phase_fraction)
        obj.attachSpecificSolverObjectComponentConfig(sc)
        obj.pos = o.pos
        obj.velocity = o.velocity
        s.attachObject(obj, scene=index)


def solver_from_scene(scene: "scenes.Scene", extra: dict | None = None, strict: bool = True) -> Solver:
    """Create, configure and attach a scene (convenience for tests and benchmarks)."""
    s = _CLASSES[SOLVER_TYPES[scene.solver]](strict=strict)
    cfg = json.loads(json.dumps(scene.config))
    if extra:
        cfg["B200"] = dict(extra)
    s.setConfig(cfg)
    _attach_scene_objects(s, scene)
    return s


def solver_from_scenes(scene_list, extra: dict | None = None, strict: bool = True):
    """One solver advancing several scenes of the same solver type together.

    Returns (solver, ranges) where ranges[k] = (start, end) is scene k's slice of the
    attach order (objects are attached scene by scene).
    """
    kinds = {sc.solver for sc in scene_list}
    if len(kinds) != 1:
        raise ValueError("a batched solver holds scenes of one solver type")
    s = _CLASSES[SOLVER_TYPES[scene_list[0].solver]](strict=strict)
    ranges = []
    start = 0
    for k, sc in enumerate(scene_list):
        cfg = json.loads(json.dumps(sc.config))
        if extra:
            cfg["B200"] = dict(extra)
        if k == 0:
            s.setConfig(cfg)
        else:
            s.addScene(cfg)
        _attach_scene_objects(s, sc, k)
        ranges.append((start, start + sc.n_total))
        start += sc.n_total
    return s, ranges
