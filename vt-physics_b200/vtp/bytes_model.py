"""Algorithmic bytes per kernel launch (state arrays touched once; FP32, float4 = 16 B).

N = all rows (fluid + boundary), Nf = fluid rows, K = number of grid key
buckets, k = mean neighbours per fluid row (self excluded), P = phases.  "state" bytes
follow the per-pass accounting of the project's bytes model; "list" adds the
neighbour-list indices (4 B per stored neighbour), which the list-based
design reads on top.
"""
from __future__ import annotations


UGNS_KERNELS = ("ugns_clear_hash", "ugns_cell_scan", "ugns_scatter", "ugns_rank_reorder", "ugns_lists")


def neighbor_pass_bytes(kind: str, Nf: int, K: int) -> float:
    """Algorithmic bytes of one neighbour pass (re-bin the fluid rows; the static boundary is
    binned once): Nf (12 key-in + 4 key + 4 key re-read + 4 permutation + 2 S) + 16 K, where S
    is the reordered per-particle state (28 B: position, velocity, material for PBF / DFSPH;
    84 B for IMM-CT: position, velocity, two phase velocities, two fractions, symmetric Q,
    material).  The neighbour-list writes are not in this model."""
    S = 84 if kind in ("IMM", "IMMCT") else 28
    return Nf * (12 + 4 + 4 + 4 + 2 * S) + 16.0 * K


def kernel_bytes(kind: str, name: str, N: int, Nf: int, K: int, k: float, P: int = 2) -> dict:
    lst = 4.0 * k * Nf
    if name == "ugns_clear_hash":
        state = 4 * (K + 1) + 16 * Nf + 8 * Nf + (16 * Nf if kind == "PBF" else 0)
        lst = 0
    elif name == "ugns_cell_scan":
        state, lst = 12 * (K + 1), 0
    elif name == "ugns_scatter":
        state, lst = 28 * Nf, 0
    elif name == "ugns_rank_reorder":
        fields = 2 if kind == "PBF" else 3
        state, lst = 12 * Nf + 2 * 16 * fields * Nf + 8 * Nf, 0
    elif name == "ugns_lists":
        state = 16 * N + 16 * K + 4 * Nf
    elif name == "pbf_lambda":
        state = 16 * N + 8 * Nf
    elif name == "pbf_dx":
        state = 16 * N + 4 * N + 16 * Nf + 32 * Nf
    elif name == "pbf_xsph":
        state = 16 * N + 16 * N + 4 * N + 32 * Nf
    elif name == "dfsph_ratio_alpha":
        state = 16 * N + 8 * Nf
    elif name == "dfsph_solve_a":
        state = 32 * N + 16 * Nf
    elif name == "dfsph_solve_b":
        state = 20 * N + 32 * Nf
    elif name in ("dfsph_viscosity", "dfsph_vis_normal"):
        state = 48 * N + 32 * Nf
    elif name == "dfsph_tension":
        state = 48 * N + 48 * Nf
    elif name == "dfsph_finalize":
        state, lst = 96 * Nf, 0
    elif name == "dfsph_solve_end":
        state, lst = 8 * ((Nf + 127) // 128), 0
    elif name == "imm_precompute":          # pos, rest density, fraction of phase 1 gathered; 3 outputs
        state = 16 * N + 8 * Nf + 12 * Nf
    elif name in ("imm_vis", "imm_vis_normal"):
        state = 32 * N + (16 * P + 8) * Nf + 16 * P * Nf + 32 * Nf
    elif name == "imm_tension":
        state = 36 * N + 16 * P * Nf + 32 * Nf
    elif name == "immct_ct":                # pos, vel, rest density gathered; symmetric Q read + write (6
        # floats each), symmetric tau written, the 48-byte packed stress row written
        state = 36 * N + 16 * Nf + 48 * Nf + 24 * Nf + 48 * Nf
    elif name == "immct_pct":               # packed {x, V, tau / rho^2} rows (48 B) gathered, own tau read,
        # phase velocities updated
        state = 48 * N + 24 * Nf + 32 * P * Nf + 32 * Nf
    elif name == "imm_drift_diffuse":       # pos, vel, flag, fractions, phase velocities gathered
        state = (36 + 20 * P) * N + 8 * P * Nf
    elif name == "imm_apply_pressure":
        state = 32 * P * Nf + 4 * P * Nf + 72 * Nf
    elif name == "imm_phase_finish":
        state = 12 * P * Nf + 32 * P * Nf + 48 * Nf
    else:
        state, lst = 0, 0
    return {"state": float(state), "list": float(lst), "total": float(state + lst)}


# FP32 operations per neighbour pair, counted from the kernel sources (an FMA counts 2,
# sqrt / rsqrt / division 1): W evaluation ~16 and gradient factor ~22 as in the
# project's work model, plus each pass's own combination terms.
FLOPS_PER_PAIR = {
    "dfsph_ratio_alpha": 16 + 22 + 19,   # W, g, ratio fma, gradient sums, alpha_2 term
    "dfsph_solve_a": 22 + 11,            # g, r.(v_i - v_j) scaled, fma into delta
    "dfsph_solve_b": 22 + 10,            # g, (k_i + k_j) c_i V_j g, three fma
    "dfsph_viscosity": 22 + 27,          # g, pressure-applied v_j, r.v_ij / (d2 + eps), three fma
    "dfsph_vis_normal": 22 + 33,
    "dfsph_tension": 30 + 24,
    "pbf_lambda": 16 + 22 + 16,
    "pbf_dx": 22 + 8,
    "pbf_xsph": 16 + 13,
}


def kernel_flops(name: str, Nf: int, k: float) -> float:
    """Algorithmic FP32 flops of one launch (0 for passes without neighbour arithmetic)."""
    return float(FLOPS_PER_PAIR.get(name, 0)) * k * Nf
