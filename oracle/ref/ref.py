"""ctypes front end of the reference harness ``oracle/_ref/libvtref.so`` (test infrastructure).

The reference keeps function-local statics in its neighbour search and
solvers (UGNSCudaImpl.cu:100-102, DFSPHSolver.cpp:340-346), so one process
may drive ONE reference solver; callers run each scene in its own process.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent.parent / "_ref" / "libvtref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        P = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_char_p]
        L.ref_attach.argtypes = [C.c_int, P, C.c_uint32, P, C.c_char_p]
        L.ref_initialize.argtypes = [C.c_int]
        L.ref_tick.argtypes = [C.c_int, C.c_uint32]
        L.ref_tick_timed.argtypes = [C.c_int, C.c_uint32]
        L.ref_tick_timed.restype = C.c_float
        L.ref_get.argtypes = [C.c_int, C.c_char_p, P, C.c_size_t]
        L.ref_set.argtypes = [C.c_int, C.c_char_p, P, C.c_size_t]
        L.ref_take_means.argtypes = [P, C.c_uint32]
        L.ref_take_means.restype = C.c_uint32
        L.ref_destroy.argtypes = [C.c_int]
        L.ref_generate.argtypes = [C.c_char_p, P, C.c_int64]
        L.ref_generate.restype = C.c_int64
        L.ref_export_ply.argtypes = [C.c_char_p, C.c_char_p, P, C.c_int64, P, P, C.c_int]
        _lib = L
    return _lib


class RefSolver:
    """The reference solver for one scene (attach order = scene object order)."""

    def __init__(self, scene):
        self.scene = scene
        self.kind = scene.solver
        tid = {"PBF": 0, "DFSPH": 1, "IMM": 2, "IMMCT": 3}[self.kind]
        cfg = json.loads(json.dumps(scene.config))
        cfg.pop("B200", None)
        self.h = lib().ref_create(tid, json.dumps(cfg).encode())
        if self.h < 0:
            raise RuntimeError(f"ref_create failed ({self.h})")
        self.n = 0
        for o in scene.objects:
            pos = np.ascontiguousarray(o.pos, np.float32)
            vel = None if o.velocity is None else np.ascontiguousarray(o.velocity, np.float32)
            sc = {"solverType": tid, "exportFlag": o.export_flag, "velocityStart": list(o.velocity_start),
                  "colorStart": list(o.color_start)}
            if o.phase_fraction is not None:
                sc["phaseFraction"] = list(o.phase_fraction)
            meta = {"name": o.name, "ObjectComponentConfig": {"epmMaterial": o.material},
                    "SolverObjectComponentConfig": sc}
            rc = lib().ref_attach(self.h, pos.ctypes.data, pos.shape[0], None if vel is None else vel.ctypes.data,
                                  json.dumps(meta).encode())
            if rc != 0:
                raise RuntimeError(f"ref_attach failed ({rc})")
            self.n += pos.shape[0]
        self.maxnbr = int(scene.config[self.kind]["Required"]["maxNeighborNum"])

    def initialize(self):
        rc = lib().ref_initialize(self.h)
        if rc != 0:
            raise RuntimeError(f"ref_initialize failed ({rc})")

    def tick(self, n: int = 1) -> bool:
        rc = lib().ref_tick(self.h, int(n))
        if rc == -4:
            raise RuntimeError("CUDA error in the reference")
        return rc == 0

    def tick_timed(self, n: int) -> float:
        ms = lib().ref_tick_timed(self.h, int(n))
        if ms < 0:
            raise RuntimeError(f"reference tick failed ({ms})")
        return ms

    def get(self, field: str, width: int = 1, dtype=np.float32) -> np.ndarray:
        shape = (self.n, width) if width > 1 else (self.n,)
        out = np.empty(shape, dtype)
        rc = lib().ref_get(self.h, field.encode(), out.ctypes.data, out.nbytes)
        if rc != 0:
            raise RuntimeError(f"ref_get({field}) failed ({rc})")
        return out

    def get_prefix(self, field: str, count: int) -> np.ndarray:
        """pos / vel of the first `count` particles (attach order)."""
        out = np.empty((count, 3), np.float32)
        rc = lib().ref_get(self.h, field.encode(), out.ctypes.data, out.nbytes)
        if rc != 0:
            raise RuntimeError(f"ref_get({field}) failed ({rc})")
        return out

    def set(self, field: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, np.float32)
        rc = lib().ref_set(self.h, field.encode(), a.ctypes.data, a.nbytes)
        if rc != 0:
            raise RuntimeError(f"ref_set({field}) failed ({rc})")

    def neighbors(self):
        cnt = self.get("neighborNum", 1, np.uint32)
        nb = self.get("neighbors", self.maxnbr, np.uint32)
        return cnt, nb

    def take_means(self) -> np.ndarray:
        buf = np.empty(1 << 16, np.float32)
        k = lib().ref_take_means(buf.ctypes.data, buf.size)
        return buf[:min(k, buf.size)].copy()

    def destroy(self):
        lib().ref_destroy(self.h)


def split_iterations(means: np.ndarray, n_fluid_objects: int, div_thr: float, inc_thr: float):
    """Rebuild (div_iters, incomp_iters) of one tick from the recorded cal_mean values.

    The loops of vfsph_div / vfsph_incomp (DFSPHCudaImpl.cu:449-503, 556-611)
    stop after the iteration whose averaged object mean is below the
    threshold, or after iteration 101.
    """
    k = n_fluid_objects
    vals = [float(np.float32(np.sum(means[i:i + k], dtype=np.float32) / np.float32(k)))
            for i in range(0, len(means), k)]
    iters = []
    pos = 0
    for thr in (div_thr, inc_thr):
        it = 0
        while pos < len(vals):
            it += 1
            v = vals[pos]
            pos += 1
            if v < thr or it > 100:
                break
        iters.append(it)
    return iters[0], iters[1], pos == len(vals)


def split_ticks(means: np.ndarray, n_fluid_objects: int, div_thr: float, inc_thr: float):
    """(div_iters, incomp_iters) of every tick in a run of consecutive ticks, from the
    cal_mean values recorded over them (each tick runs both loops at least once, so the
    sequence splits unambiguously; the same stop rule as split_iterations)."""
    k = n_fluid_objects
    vals = [float(np.float32(np.sum(means[i:i + k], dtype=np.float32) / np.float32(k)))
            for i in range(0, len(means), k)]
    out, pos = [], 0
    while pos < len(vals):
        tick = []
        for thr in (div_thr, inc_thr):
            it = 0
            while pos < len(vals):
                it += 1
                v = vals[pos]
                pos += 1
                if v < thr or it > 100:
                    break
            tick.append(it)
        out.append(tuple(tick))
    return out


def generate(config: dict) -> np.ndarray:
    """ModelHandler::generateObjectElements of the reference build (host code) -> (n, 3) float32."""
    cfg = json.dumps(config).encode()
    n = lib().ref_generate(cfg, None, 0)
    if n < 0:
        raise RuntimeError("ref_generate: bad config")
    out = np.empty((n, 3), np.float32)
    if n:
        lib().ref_generate(cfg, out.ctypes.data, n)
    return out


def export_ply(directory: str, name: str, pos, color=None, phase=None):
    """ExportUtil::exportData of the reference build; returns the path it wrote
    (the reference joins directory and name with a backslash)."""
    p = np.ascontiguousarray(pos, np.float32)
    c = None if color is None else np.ascontiguousarray(color, np.float32)
    ph = None if phase is None else np.ascontiguousarray(phase, np.float32)
    nph = 0 if ph is None else ph.shape[1]
    rc = lib().ref_export_ply(str(directory).encode(), name.encode(), p.ctypes.data, p.shape[0],
                              None if c is None else c.ctypes.data, None if ph is None else ph.ctypes.data, nph)
    if rc != 0:
        raise RuntimeError("ref_export_ply failed")
    return f"{directory}\\{name}.ply"
