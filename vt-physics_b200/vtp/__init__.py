"""B200 particle-fluid hot path: uniform-grid neighbour search + PBF / DFSPH / IMM-CT.

The compute path is the sm_100a library ``libvtp.so`` behind the C ABI in
``include/vtp.h``; this package is its Python host mirror.
"""
from . import model, scenes
from ._lib import FIELDS, LIB_PATH, VtpError, lib, status_string
from .solver import (DFSPH, EPM_BOUNDARY, EPM_FLUID, IMM, IMMCT, PBF, DFSPHSolver, HostBuffer, IMMCTSolver,
                     IMMSolver, Object,
                     ObjectManager, PBFSolver, Solver, SolverManager, Particle_Box, Particle_Common, Particle_Cube,
                     solver_from_scene, solver_from_scenes, tick_together)

__all__ = ["scenes", "FIELDS", "LIB_PATH", "VtpError", "lib", "status_string", "DFSPH", "EPM_BOUNDARY", "EPM_FLUID",
           "IMM", "IMMCT", "PBF", "DFSPHSolver", "IMMCTSolver", "IMMSolver", "Object", "ObjectManager", "PBFSolver",
           "Solver", "SolverManager", "Particle_Box", "Particle_Common", "Particle_Cube", "solver_from_scene",
           "solver_from_scenes", "tick_together", "HostBuffer"]
