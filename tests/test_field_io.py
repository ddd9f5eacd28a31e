"""Field I/O by attach-order particle range (vtp_solver_get/set_field_range)."""
import numpy as np
import pytest

import vtp
from vtp import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_range_io_matches_full_io(vtp_gpu, kind):
    sc = scenes.dam_break(kind, 3000, seed=31)
    s = vtp.solver_from_scene(sc)
    assert s.initialize() and s.tickNsteps(3)
    n, nf = sc.n_total, sc.objects[0].n
    for name in ("pos", "vel", "volume"):
        full = s.get_field(name)
        assert np.array_equal(s.get_field_range(name, 0, nf), full[:nf])
        assert np.array_equal(s.get_field_range(name, nf, n - nf), full[nf:])
        assert np.array_equal(s.get_field_range(name, 100, 7), full[100:107])
    # set a sub-range of fluid velocities: only those particles change
    v = s.get_field("vel")
    new = (v[10:20] + 0.5).astype(np.float32)
    s.set_field_range_ptr("vel", 10, 10, np.ascontiguousarray(new).ctypes.data, new.nbytes)
    v2 = s.get_field("vel")
    assert np.array_equal(v2[10:20], new)
    assert np.array_equal(np.delete(v2, np.s_[10:20], axis=0), np.delete(v, np.s_[10:20], axis=0))
    with pytest.raises(vtp.VtpError):
        s.get_field_range("pos", n - 5, 10)
    s.destroy()


def test_state_range_io_matches_field_io(vtp_gpu):
    import ctypes as C
    sc = scenes.dam_break("DFSPH", 3000, seed=32)
    s = vtp.solver_from_scene(sc)
    assert s.initialize() and s.tickNsteps(2)
    nf = sc.objects[0].n
    p = np.empty((nf, 3), np.float32)
    v = np.empty((nf, 3), np.float32)
    s.get_state_range_ptr(0, nf, p.ctypes.data, v.ctypes.data)
    assert np.array_equal(p, s.get_field_range("pos", 0, nf))
    assert np.array_equal(v, s.get_field_range("vel", 0, nf))
    p2, v2 = (p + 0.001).astype(np.float32), (v * 0.5).astype(np.float32)
    s.set_state_range_ptr(0, nf, p2.ctypes.data, v2.ctypes.data)
    assert np.array_equal(s.get_field("pos")[:nf], p2)
    assert np.array_equal(s.get_field("vel")[:nf], v2)
    # the next substep starts from the new state: same as setting pos / vel one by one
    t = vtp.solver_from_scene(sc)
    assert t.initialize() and t.tickNsteps(2)
    t.set_field_range_ptr("pos", 0, nf, p2.ctypes.data, p2.nbytes)
    t.set_field_range_ptr("vel", 0, nf, v2.ctypes.data, v2.nbytes)
    assert s.tickNsteps(1) and t.tickNsteps(1)
    assert np.array_equal(s.get_field("pos"), t.get_field("pos"))
    s.destroy()
    t.destroy()


def test_host_buffers_round_trip_state(vtp_gpu):
    sc = scenes.dam_break("PBF", 2000, seed=33)
    s = vtp.solver_from_scene(sc)
    assert s.initialize() and s.tickNsteps(2)
    nf = sc.objects[0].n
    p, v = vtp.HostBuffer((nf, 3)), vtp.HostBuffer((nf, 3))
    s.get_state_range_ptr(0, nf, p.ptr, v.ptr)
    assert np.array_equal(p.array, s.get_field("pos")[:nf])
    assert np.array_equal(v.array, s.get_field("vel")[:nf])
    p.array[:] += 0.01
    s.set_state_range_ptr(0, nf, p.ptr, v.ptr)
    assert np.array_equal(s.get_field("pos")[:nf], p.array)
    p.free()
    v.free()
    s.destroy()


@pytest.mark.parametrize("kind,extra,steps", [("PBF", None, 1), ("PBF", None, 3), ("DFSPH", {"cfl": 0.4}, 1),
                                              ("DFSPH", {"useGraphs": False}, 2)])
def test_one_call_frame_equals_set_tick_get(vtp_gpu, kind, extra, steps):
    """vtp_solver_step_state_range (upload, n substeps, read back, one synchronisation) gives
    what set_state_range, tickNsteps and get_state_range give one after another, frame after
    frame, with the output buffers also serving as the next frame's input."""
    sc = scenes.dam_break(kind, 3000, seed=34)
    nf = sc.objects[0].n
    a, b = vtp.solver_from_scene(sc, extra=extra), vtp.solver_from_scene(sc, extra=extra)
    assert a.initialize() and b.initialize() and a.tickNsteps(2) and b.tickNsteps(2)
    pa, va = vtp.HostBuffer((nf, 3)), vtp.HostBuffer((nf, 3))
    pb, vb = vtp.HostBuffer((nf, 3)), vtp.HostBuffer((nf, 3))
    a.get_state_range_ptr(0, nf, pa.ptr, va.ptr)
    b.get_state_range_ptr(0, nf, pb.ptr, vb.ptr)
    for frame in range(3):
        va.array[:5] *= 0.5     # the host edits the state between frames
        vb.array[:5] *= 0.5
        assert a.step_state_range_ptr(0, nf, pa.ptr, va.ptr, steps, pa.ptr, va.ptr), a.last_error
        b.set_state_range_ptr(0, nf, pb.ptr, vb.ptr)
        assert b.tickNsteps(steps), b.last_error
        b.get_state_range_ptr(0, nf, pb.ptr, vb.ptr)
        assert np.array_equal(pa.array, pb.array) and np.array_equal(va.array, vb.array), frame
        assert a.stats() == b.stats()
    assert a.step_state_range_ptr(0, 0, 0, 0, 1, 0, 0) and b.tickNsteps(1)   # count 0 only ticks
    assert np.array_equal(a.get_field("pos"), b.get_field("pos"))
    # no substeps: the state goes in and comes back unchanged
    a.get_state_range_ptr(0, nf, pa.ptr, va.ptr)
    pin, vin = pa.array.copy(), va.array.copy()
    pb.array[:] = 0.0
    vb.array[:] = 0.0
    assert a.step_state_range_ptr(0, nf, pa.ptr, va.ptr, 0, pb.ptr, vb.ptr), a.last_error
    assert np.array_equal(pb.array, pin) and np.array_equal(vb.array, vin)
    assert a.stats()["steps_done"] == b.stats()["steps_done"]
    with pytest.raises(vtp.VtpError):
        a.strict = True
        a.step_state_range_ptr(nf, sc.n_total, pa.ptr, va.ptr, 1, pa.ptr, va.ptr)
    for buf in (pa, va, pb, vb):
        buf.free()
    a.destroy()
    b.destroy()
