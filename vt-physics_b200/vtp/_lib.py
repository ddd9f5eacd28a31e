"""ctypes binding of ``libvtp.so`` (the C ABI declared in include/vtp.h)."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# VTP_LIBRARY=checked selects the checked build (device-side bounds checks, build.py --checked);
# any other value is a path to the library.
_choice = os.environ.get("VTP_LIBRARY", "")
LIB_PATH = (Path(__file__).resolve().parent / "libvtp_checked.so" if _choice == "checked" else
            Path(_choice) if _choice else Path(__file__).resolve().parent / "libvtp.so")

VTP_OK = 0
VTP_ERR_CONFIG = 1
VTP_ERR_CUDA = 2
VTP_NOT_CONVERGED = 3
VTP_ERR_NAN = 4
VTP_ERR_TIMEOUT = 5
VTP_ERR_BOUNDS = 6
VTP_ERR_STATE = 7
VTP_ERR_ARG = 8
VTP_ERR_NOMEM = 9

SOLVER_TYPES = {"PBF": 0, "DFSPH": 1, "IMM": 2, "IMMCT": 3}

FIELDS = {
    "pos": (0, 3), "vel": (1, 3), "color": (2, 3), "mat": (3, 1), "mass": (4, 1), "volume": (5, 1),
    "density": (6, 1), "lambda": (7, 1), "alpha": (8, 1), "kappa": (9, 1), "rest_density": (10, 1),
    "vol_frac": (11, -1), "phase_vel": (12, -3), "conformation": (13, 9), "vel_grad": (14, 9),
    "stress": (15, 9), "cd": (16, 1), "delta": (17, 1),
}

# Every symbol include/vtp.h declares, with (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "vtp_status_string": (C.c_char_p, [C.c_int]),
    "vtp_version": (C.c_char_p, []),
    "vtp_last_error": (C.c_char_p, []),
    "vtp_solver_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "vtp_solver_set_config": (C.c_int, [_P, C.c_char_p]),
    "vtp_solver_attach_object": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_char_p]),
    "vtp_solver_initialize": (C.c_int, [_P]),
    "vtp_solver_add_scene": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_uint32)]),
    "vtp_solver_get_scene_stats": (C.c_int, [_P, C.c_uint32, _P]),
    "vtp_solver_tick_n_steps": (C.c_int, [_P, C.c_uint32]),
    "vtp_solver_run": (C.c_int, [_P]),
    "vtp_solver_reset": (C.c_int, [_P]),
    "vtp_solver_destroy": (None, [_P]),
    "vtp_solver_get_config": (C.c_int, [_P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "vtp_solver_get_stats": (C.c_int, [_P, _P]),
    "vtp_solver_particle_counts": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "vtp_solver_get_field": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "vtp_solver_set_field": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "vtp_solver_get_field_range": (C.c_int, [_P, C.c_int, C.c_uint32, C.c_uint32, _P, C.c_size_t]),
    "vtp_solver_set_field_range": (C.c_int, [_P, C.c_int, C.c_uint32, C.c_uint32, _P, C.c_size_t]),
    "vtp_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(_P)]),
    "vtp_host_free": (None, [_P]),
    "vtp_selftest_cube": (C.c_int, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "vtp_solver_get_conservation": (C.c_int, [_P, C.c_int, _P]),
    "vtp_generate_cube": (C.c_int, [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_double, C.c_double,
                                    C.c_uint64, _P, C.c_uint32, C.POINTER(C.c_uint32), _P]),
    "vtp_generate_box": (C.c_int, [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32, _P,
                                   C.c_uint32, C.POINTER(C.c_uint32), _P]),
    "vtp_generate_particles": (C.c_int, [C.c_char_p, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "vtp_read_ply": (C.c_int, [C.c_char_p, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "vtp_write_ply": (C.c_int, [C.c_char_p, C.c_char_p, _P, C.c_uint64, _P, _P, C.c_int32]),
    "vtp_solver_get_state_range": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P]),
    "vtp_solver_set_state_range": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P]),
    "vtp_solver_step_state_range": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, C.c_uint32, _P, _P]),
    "vtp_solver_step_state_ranges": (C.c_int, [_P, C.c_uint32, _P, _P, _P, _P, C.c_uint32, _P, _P]),
    "vtp_solver_get_neighbors": (C.c_int, [_P, _P, _P, C.c_uint32]),
    "vtp_solver_get_sorted_order": (C.c_int, [_P, _P, _P]),
    "vtp_solver_get_stage_times": (C.c_int, [_P, _P]),
    "vtp_solver_get_launch_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "vtp_solver_profile_kernels": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "vtp_solver_diff_forward": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int]),
    "vtp_solver_diff_backward": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(C.c_double)]),
    "vtp_solver_diff_lists": (C.c_int, [_P, C.c_uint32, _P, _P, C.c_uint32]),
    "vtp_solver_diff_iterations": (C.c_int, [_P, C.c_uint32, _P, _P]),
    "vtp_solver_dfsph_solve_forward": (C.c_int, [_P, C.c_int, _P, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "vtp_solver_dfsph_solve_backward": (C.c_int, [_P, _P, _P]),
    "vtp_ugns_neighbors_noalloc": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                             C.c_uint32, _P, _P, _P]),
    "vtp_domain_create": (C.c_int, [C.c_char_p, _P, C.c_uint32, _P, _P, C.c_uint32, C.c_int, C.c_uint32, C.c_uint32,
                                    C.POINTER(_P)]),
    "vtp_domain_destroy": (None, [_P]),
    "vtp_domain_set_stream": (C.c_int, [_P, _P]),
    "vtp_domain_capacity": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "vtp_domain_load": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P, _P]),
    "vtp_domain_prepare": (C.c_int, [_P]),
    "vtp_domain_owned_vmax2": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "vtp_domain_set_dt": (C.c_int, [_P, C.c_float]),
    "vtp_domain_solve_begin": (C.c_int, [_P, C.c_int]),
    "vtp_domain_solve_a": (C.c_int, [_P, _P]),
    "vtp_domain_solve_b": (C.c_int, [_P]),
    "vtp_domain_forces": (C.c_int, [_P]),
    "vtp_domain_tension": (C.c_int, [_P]),
    "vtp_domain_finalize": (C.c_int, [_P]),
    "vtp_domain_pbf_lambda": (C.c_int, [_P]),
    "vtp_domain_pbf_dx": (C.c_int, [_P]),
    "vtp_domain_pbf_xsph": (C.c_int, [_P]),
    "vtp_domain_pack": (C.c_int, [_P, C.c_int, _P, C.c_uint32, _P]),
    "vtp_domain_unpack": (C.c_int, [_P, C.c_int, C.c_uint32, C.c_uint32, _P]),
    "vtp_domain_read": (C.c_int, [_P, _P, _P]),
    "vtp_domain_export_ipc": (C.c_int, [_P, _P]),
    "vtp_domain_link_peer": (C.c_int, [_P, C.c_int, _P]),
    "vtp_domain_link_peer_ipc": (C.c_int, [_P, C.c_int, _P]),
    "vtp_domain_set_halo": (C.c_int, [_P, C.c_int]),
    "vtp_domain_buffer_parity": (C.c_int, [_P, _P]),
    "vtp_domain_rows": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P]),
    "vtp_domain_halo_targets": (C.c_int, [_P, C.c_int, _P, _P, C.c_uint32, C.c_uint32]),
}


class VtpKernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("total_ms", C.c_float), ("launches", C.c_uint32)]


class VtpStats(C.Structure):
    _fields_ = [("steps_done", C.c_uint64), ("sim_time", C.c_float), ("last_div_iters", C.c_uint32),
                ("last_incomp_iters", C.c_uint32), ("total_div_iters", C.c_uint64),
                ("total_incomp_iters", C.c_uint64), ("last_div_residual", C.c_double),
                ("last_incomp_residual", C.c_double), ("neighbor_overflow", C.c_uint32),
                ("dead_particles", C.c_uint32), ("phase_retries", C.c_uint32), ("status_bits", C.c_uint32),
                ("last_dt", C.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class VtpConservation(C.Structure):
    _fields_ = [("fluid_mass", C.c_double), ("momentum", C.c_double * 3), ("kinetic_energy", C.c_double),
                ("mean_density_error", C.c_double), ("fluid_particles", C.c_uint32), ("phases", C.c_uint32),
                ("phase_mass", C.c_double * 8)]

    def as_dict(self) -> dict:
        return {"fluid_mass": self.fluid_mass, "momentum": list(self.momentum),
                "kinetic_energy": self.kinetic_energy, "mean_density_error": self.mean_density_error,
                "fluid_particles": self.fluid_particles, "phase_mass": list(self.phase_mass[: self.phases])}


class VtpError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str):
        super().__init__(f"{where}: {status_string(code)} ({code}): {detail}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load libvtp.so; raises if the CUDA library has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python vt-physics_b200/build.py`")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(code: int) -> str:
    try:
        return lib().vtp_status_string(code).decode()
    except Exception:
        return str(code)


def check(code: int, where: str) -> int:
    if code != VTP_OK:
        raise VtpError(code, where, lib().vtp_last_error().decode())
    return code
