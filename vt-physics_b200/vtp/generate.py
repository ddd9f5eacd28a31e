"""Scene generation on the device (``vtp_generate_cube`` / ``vtp_generate_box``).

The same particles as the host generators in ``vtp.scenes`` (``cube``, ``box``,
``jitter``), bit for bit, written into a CUDA tensor instead of built on the
host and copied: for million-particle scenes generation then takes a fraction
of a millisecond on the GPU instead of a host loop and a transfer.
"""
from __future__ import annotations

import ctypes as C

from ._lib import check, lib


def _vec3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def _generate(fn, args, torch, device):
    cnt = C.c_uint32()
    rc = fn(*args(None, 0, C.byref(cnt)))
    if rc not in (0,) and cnt.value == 0:
        check(rc, "generate")
    out = torch.empty((cnt.value, 3), dtype=torch.float32, device=device)
    if cnt.value:
        stream = torch.cuda.current_stream(device).cuda_stream
        check(fn(*args(C.c_void_p(out.data_ptr()), cnt.value, C.byref(cnt), C.c_void_p(stream))), "generate")
    return out


def cube(r: float, lb, size, jitter_amp: float = 0.0, jitter_spacing: float | None = None, seed: int = 0,
         device: str = "cuda"):
    """Lattice cube as ``scenes.jitter(scenes.cube(r, lb, size), jitter_amp, jitter_spacing, seed)``
    (``jitter_spacing`` defaults to 2 r), as an (n, 3) float32 CUDA tensor."""
    import torch
    sp = 2.0 * r if jitter_spacing is None else jitter_spacing
    L = lib()

    def args(ptr, cap, cnt, stream=None):
        return (C.c_float(r), _vec3(lb), _vec3(size), C.c_double(jitter_amp), C.c_double(sp),
                C.c_uint64(seed), ptr, cap, cnt, stream)
    return _generate(L.vtp_generate_cube, args, torch, device)


def box(r: float, lb, size, layer_num: int, device: str = "cuda"):
    """Hollow box as ``scenes.box(r, lb, size, layer_num)``, as an (n, 3) float32 CUDA tensor."""
    import torch
    L = lib()

    def args(ptr, cap, cnt, stream=None):
        return (C.c_float(r), _vec3(lb), _vec3(size), C.c_int32(layer_num), ptr, cap, cnt, stream)
    return _generate(L.vtp_generate_box, args, torch, device)
