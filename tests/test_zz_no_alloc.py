"""The allocation-free neighbour search against the solver's own neighbour search.

vtp_ugns_neighbors_noalloc serves callers that cannot allocate device memory
when they need neighbour lists (while recording a CUDA graph by stream
capture, or under a host-managed fixed memory budget): they pass device
buffers for positions and lists, and the library works in a fixed scratch
array of its own.  This test hands it device buffers (allocated here, by the
test) and checks that two calls in a row give exactly the lists the solver
API returns (vtp_solver_get_neighbors) for the same positions; neighbour
lists are integer data, so the comparison is bit-exact.  The file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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
