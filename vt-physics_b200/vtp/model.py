"""Particle geometry on the host through the C ABI: the reference's particle
generators (ModelHandler::generateObjectElements, ModelHandler.cpp:13-175),
the PLY particle loader (load_PLY_ParticleElements, :207-228) and the PLY
writer of the exports (ExportUtil::exportAsPly, ExportUtil.cpp:28-88)."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np

from ._lib import check, lib


def generate(config: dict) -> np.ndarray:
    """Particles of a generator config ("genType" 1 sphere, 2 cube, 3 cylinder, 4 plane,
    5 box, with the keys the reference's object components set) -> (n, 3) float32."""
    cfg = json.dumps(config).encode()
    n = C.c_uint64()
    check(lib().vtp_generate_particles(cfg, None, 0, C.byref(n)), "generate_particles")
    out = np.empty((n.value, 3), np.float32)
    if n.value:
        check(lib().vtp_generate_particles(cfg, out.ctypes.data, n.value, C.byref(n)), "generate_particles")
    return out


def read_ply(path) -> np.ndarray:
    """Every vertex of a PLY file as one particle -> (n, 3) float32."""
    p = str(path).encode()
    n = C.c_uint64()
    check(lib().vtp_read_ply(p, None, 0, C.byref(n)), "read_ply")
    out = np.empty((n.value, 3), np.float32)
    if n.value:
        check(lib().vtp_read_ply(p, out.ctypes.data, n.value, C.byref(n)), "read_ply")
    return out


def write_ply(directory, name: str, pos, color=None, phase=None) -> Path:
    """ASCII PLY of the exports at directory/name.ply; returns the path."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    c = None if color is None else np.ascontiguousarray(color, np.float32).reshape(-1, 3)
    ph = None if phase is None else np.ascontiguousarray(phase, np.float32).reshape(p.shape[0], -1)
    check(lib().vtp_write_ply(str(directory).encode(), name.encode(), p.ctypes.data, p.shape[0],
                              None if c is None else c.ctypes.data, None if ph is None else ph.ctypes.data,
                              0 if ph is None else ph.shape[1]), "write_ply")
    return Path(directory) / f"{name}.ply"
