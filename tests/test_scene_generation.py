"""Scene generation on the device (vtp_generate_cube / vtp_generate_box): the
same particles as the host generators of vtp.scenes, bit for bit."""
import ctypes as C
import time

import numpy as np
import pytest

from vtp import scenes

pytestmark = pytest.mark.gpu

CUBES = [  # (radius, lb, size, jitter amplitude, seed): the test and bench scenes' fluid blocks
    (0.01, (0.04, 0.04, 0.04), (0.4, 0.8, 0.4), 0.1, 1001),     # PBF dam break
    (0.005, (0.03, 0.03, 0.03), (1.0, 1.0, 1.0), 0.05, 2002),   # DFSPH 1M
    (0.01, (0.2, 0.2, 0.2), (0.8, 0.8, 0.8), 0.0, 0),           # differentiable PBF
    (0.005, (0.04, 0.04, 0.04), (0.13, 0.05, 0.07), 0.05, 7),   # a small odd-sized block
]
BOXES = [  # (radius, lb, size, layers)
    (0.01, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2),
    (0.005, (0.0, 0.0, 0.0), (2.0, 1.5, 1.06), 3),
    (0.01, (0.0, 0.0, 0.0), (1.2, 1.2, 1.2), 2),
    (0.005, (0.0, 0.0, 0.0), (0.1, 0.07, 0.05), 4),            # layers meeting in the middle
]


@pytest.mark.parametrize("case", CUBES)
def test_device_cube_matches_host_generator(vtp_gpu, case):
    import torch
    from vtp import generate
    r, lb, size, amp, seed = case
    t0 = time.perf_counter()
    host = scenes.cube(r, lb, size)
    if amp:
        host = scenes.jitter(host, amp, 2 * r, seed)
    th = time.perf_counter() - t0
    t0 = time.perf_counter()
    dev = generate.cube(r, lb, size, amp, 2 * r, seed)
    torch.cuda.synchronize()
    td = time.perf_counter() - t0
    print(f"cube r={r} n={host.shape[0]}: host {th * 1e3:.1f} ms, device {td * 1e3:.2f} ms")
    assert dev.shape == host.shape
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))


@pytest.mark.parametrize("case", BOXES)
def test_device_box_matches_host_generator(vtp_gpu, case):
    from vtp import generate
    r, lb, size, layers = case
    host = scenes.box(r, lb, size, layers)
    dev = generate.box(r, lb, size, layers)
    assert dev.shape == host.shape
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))


def test_generator_reports_the_count_when_the_buffer_is_short(vtp_gpu):
    lib = vtp_gpu.lib()
    lb, size = (C.c_float * 3)(0.0, 0.0, 0.0), (C.c_float * 3)(0.1, 0.1, 0.1)
    cnt = C.c_uint32()
    rc = lib.vtp_generate_cube(C.c_float(0.01), lb, size, 0.0, 0.0, 0, None, 0, C.byref(cnt), None)
    assert rc != 0 and cnt.value == 125
    rc = lib.vtp_generate_box(C.c_float(0.01), lb, size, 1, None, 10, C.byref(cnt), None)
    assert rc != 0 and cnt.value == scenes.box(0.01, (0, 0, 0), (0.1, 0.1, 0.1), 1).shape[0]
