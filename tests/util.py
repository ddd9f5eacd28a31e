"""Shared comparison helpers for the parity tests."""
import numpy as np


def rel_err(a, b, floor: float = 0.0) -> float:
    """max_i |a_i - b_i| / max(max_i |b_i|, floor) over all components."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = max(float(np.max(np.abs(b))) if b.size else 0.0, floor)
    if den == 0.0:
        return float(np.max(np.abs(a - b))) if a.size else 0.0
    return float(np.max(np.abs(a - b))) / den


def fluid_mask(scene):
    return np.concatenate([np.full(o.n, o.material == 0) for o in scene.objects])
