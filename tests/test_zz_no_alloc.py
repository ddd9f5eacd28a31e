"""The allocation-free neighbour search against the solver's own neighbour search.

vtp_ugns_neighbors_noalloc serves callers that cannot allocate device memory
when they need neighbour lists: hosts that run this library under a fixed
memory budget managed by their own allocator, and real-time loops that forbid
allocation after start-up.  They pass device buffers for positions and lists,
and the library works in a fixed scratch array of its own.  These tests hand
it device buffers (allocated here, by the test) and check that two calls in a
row give exactly the lists the solver API returns (vtp_solver_get_neighbors)
for the same positions; neighbour lists are integer data, so the comparison is
bit-exact.  A second test runs in a fresh process without torch: it checks
that a call after the first one leaves the device's free memory unchanged, and
that a call after cudaDeviceReset (which reloads the library's device code and
can move the scratch array) still gives the same lists.  The file is named to
be collected last.
"""
import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _noalloc(vtp, torch, pos_np, req):
    n = pos_np.shape[0]
    maxnbr = int(req["maxNeighborNum"])
    h = np.float32(np.float32(req["particleRadius"]) * np.float32(4))
    lb = (C.c_float * 3)(*[float(np.float32(v)) for v in req["simSpaceLB"]])
    size = (C.c_float * 3)(*[float(np.float32(v)) for v in req["simSpaceSize"]])
    d_pos = torch.from_numpy(np.ascontiguousarray(pos_np, np.float32)).cuda()
    d_cnt = torch.empty(n, dtype=torch.int32, device="cuda")
    d_nbr = torch.empty(n * maxnbr, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = vtp.lib().vtp_ugns_neighbors_noalloc(d_pos.data_ptr(), n, lb, size, float(h), maxnbr, d_cnt.data_ptr(),
                                             d_nbr.data_ptr(), stream)
    assert rc == 0, vtp.lib().vtp_last_error().decode()
    torch.cuda.synchronize()
    cnt = d_cnt.cpu().numpy().view(np.uint32)
    nbr = d_nbr.cpu().numpy().view(np.uint32).reshape(n, maxnbr)
    return cnt, nbr


@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_noalloc_neighbors_match_solver_api_twice(vtp_gpu, kind):
    import torch
    vtp = vtp_gpu
    torch.cuda.set_device(0)
    sc = vtp.scenes.pbf_dam_break() if kind == "PBF" else vtp.scenes.dam_break("DFSPH", 20000, seed=41)
    req = sc.config[kind]["Required"]
    s = vtp.solver_from_scene(sc)
    assert s.initialize()
    assert s.tickNsteps(3)
    pos = s.get_field("pos")
    ref_cnt, ref_nbr = s.get_neighbors(int(req["maxNeighborNum"]))
    s.destroy()
    for _ in range(2):  # the scratch array keeps the previous call's contents
        cnt, nbr = _noalloc(vtp, torch, pos, req)
        assert np.array_equal(cnt, ref_cnt)
        assert np.array_equal(nbr, ref_nbr)


def test_noalloc_upper_face_and_outside_particles_match_the_oracle(vtp_gpu, oracle_lib):
    """Particles in the grid's inclusive upper cell layer (cell index == cells per axis, which
    the reference's cellIsAvailable accepts and which shares its bucket numbering with the
    next row of cells), exactly on the upper face, and outside the grid on either side: the
    lists equal the FP32 restatement of the reference's search (no list, count 0, outside)."""
    import torch
    vtp = vtp_gpu
    torch.cuda.set_device(0)
    # h = 1/8 and size 1 give exactly 8 cells per axis; [1, 1.125) is the inclusive layer
    req = {"particleRadius": 0.03125, "simSpaceLB": [0.0, 0.0, 0.0], "simSpaceSize": [1.0, 1.0, 1.0],
           "maxNeighborNum": 60}
    ax = np.arange(0.78, 1.2, 0.045, dtype=np.float32)
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    lattice = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    face = np.array([[1.0, 0.9, 0.95], [1.0, 1.0, 1.0], [0.95, 1.0, 1.05], [1.12, 1.124, 0.9],
                     [1.125, 0.9, 0.9], [-0.01, 0.5, 0.5], [0.5, -1e-7, 0.5], [0.0, 0.0, 0.0],
                     # cells (0, y + 1, z) share their buckets with the inclusive-layer cells (8, y, z)
                     [0.01, 1.01, 0.9], [0.05, 1.06, 0.95], [0.03, 1.0, 1.0]], np.float32)
    pos = np.ascontiguousarray(np.concatenate([lattice, face]), np.float32)
    ref_cnt, ref_nbr, _, _ = oracle_lib.neighbors(pos, oracle_lib.make_grid(req))
    assert (ref_cnt == 0).sum() > 0 and (ref_cnt > 1).sum() > 100
    for _ in range(2):
        cnt, nbr = _noalloc(vtp, torch, pos, req)
        assert np.array_equal(cnt, ref_cnt)
        for i in np.nonzero(ref_cnt)[0]:
            assert np.array_equal(nbr[i, : ref_cnt[i]], ref_nbr[i, : ref_cnt[i]])


def test_noalloc_rejects_oversized_input(vtp_gpu):
    import torch
    vtp = vtp_gpu
    lib = vtp.lib()
    lb = (C.c_float * 3)(0.0, 0.0, 0.0)
    size = (C.c_float * 3)(1.0, 1.0, 1.0)
    d = torch.empty(16, dtype=torch.int32, device="cuda")
    too_many = 1048576 + 1
    rc = lib.vtp_ugns_neighbors_noalloc(d.data_ptr(), too_many, lb, size, 0.04, 60, d.data_ptr(), d.data_ptr(), None)
    assert rc == 6 and b"scratch limit" in lib.vtp_last_error()
    fine = (C.c_float * 3)(100.0, 100.0, 100.0)   # 2500^3 cells
    rc = lib.vtp_ugns_neighbors_noalloc(d.data_ptr(), 4, lb, fine, 0.04, 60, d.data_ptr(), d.data_ptr(), None)
    assert rc == 6 and b"scratch limit" in lib.vtp_last_error()
    tiny = (C.c_float * 3)(1.0, 1.0, 1.0)          # 1 / 1e-30 cells per axis: rejected before any integer cast
    rc = lib.vtp_ugns_neighbors_noalloc(d.data_ptr(), 4, lb, tiny, 1e-30, 60, d.data_ptr(), d.data_ptr(), None)
    assert rc == 6 and b"scratch limit" in lib.vtp_last_error()
    bad = (C.c_float * 3)(float("nan"), 1.0, 1.0)
    rc = lib.vtp_ugns_neighbors_noalloc(d.data_ptr(), 4, bad, size, 0.04, 60, d.data_ptr(), d.data_ptr(), None)
    assert rc == 8 and b"finite" in lib.vtp_last_error()


# Runs in a fresh process that never initialises torch's CUDA state, so that
# cudaDeviceReset ends no allocation but the test's own.  The CUDA runtime is
# the one libvtp.so links (same soname, same loaded instance).
_RESET_SCRIPT = r"""
import ctypes as C, sys
import numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/vt-physics_b200"]
import vtp
lib = vtp.lib()
rt = C.CDLL("libcudart.so.12")
sc = vtp.scenes.dam_break("DFSPH", 20000, seed=43)
req = sc.config["DFSPH"]["Required"]
pos = np.ascontiguousarray(np.concatenate([o.pos for o in sc.objects]), np.float32)
n, M = pos.shape[0], int(req["maxNeighborNum"])
h = float(np.float32(np.float32(req["particleRadius"]) * np.float32(4)))
lb = (C.c_float * 3)(*[float(np.float32(v)) for v in req["simSpaceLB"]])
size = (C.c_float * 3)(*[float(np.float32(v)) for v in req["simSpaceSize"]])

def check(rc):
    assert rc == 0, rt.cudaGetErrorString(rc)

def run():
    bufs = []
    for nbytes in (pos.nbytes, 4 * n, 4 * n * M):
        p = C.c_void_p()
        check(rt.cudaMalloc(C.byref(p), C.c_size_t(nbytes)))
        bufs.append(p)
    check(rt.cudaMemcpy(bufs[0], pos.ctypes.data_as(C.c_void_p), C.c_size_t(pos.nbytes), 1))
    out = []
    free = []
    for _ in range(2):
        f, t = C.c_size_t(), C.c_size_t()
        check(rt.cudaDeviceSynchronize())
        check(rt.cudaMemGetInfo(C.byref(f), C.byref(t)))
        rc = lib.vtp_ugns_neighbors_noalloc(bufs[0], n, lb, size, C.c_float(h), M, bufs[1], bufs[2], None)
        assert rc == 0, lib.vtp_last_error()
        check(rt.cudaDeviceSynchronize())
        f2 = C.c_size_t()
        check(rt.cudaMemGetInfo(C.byref(f2), C.byref(t)))
        free.append((f.value, f2.value))
        cnt = np.empty(n, np.uint32)
        nbr = np.empty(n * M, np.uint32)
        check(rt.cudaMemcpy(cnt.ctypes.data_as(C.c_void_p), bufs[1], C.c_size_t(cnt.nbytes), 2))
        check(rt.cudaMemcpy(nbr.ctypes.data_as(C.c_void_p), bufs[2], C.c_size_t(nbr.nbytes), 2))
        out.append((cnt, nbr))
    for b in bufs:
        check(rt.cudaFree(b))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    return out[0], free[1]

(c1, l1), free1 = run()
# The second call of a run found the library's device code loaded: it allocated nothing.
assert free1[0] == free1[1], free1
check(rt.cudaDeviceReset())
(c2, l2), free2 = run()
assert free2[0] == free2[1], free2
assert np.array_equal(c1, c2) and np.array_equal(l1, l2)
assert int(c1.sum()) > 20 * n   # non-trivial lists
print("noalloc reset ok", int(c1.sum()))
"""


def test_noalloc_allocates_nothing_and_survives_device_reset(vtp_gpu):
    env = dict(os.environ)
    r = subprocess.run([sys.executable, "-c", _RESET_SCRIPT, str(ROOT)], capture_output=True, text=True,
                       timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "noalloc reset ok" in r.stdout
