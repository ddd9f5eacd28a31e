"""A pressure solve that runs past 100 iterations stops the solver the way the
reference's does (vfsph_div / vfsph_incomp flag a crash, DFSPHCudaImpl.cu:449-503,
and DFSPHSolver::tick stops ticking, DFSPHSolver.cpp:339-406): tickNsteps fails
after that substep, later ticks fail at once, and with "stopOnNonConvergence": false
the run goes on to the requested substeps and reports the status at the end."""
import pytest

import vtp
from vtp import scenes

pytestmark = pytest.mark.gpu


def _unreachable(kind="DFSPH"):
    sc = scenes.dam_break(kind, 3000, seed=35)
    sc.config[kind]["Required"]["divFreeThreshold"] = 1e-12   # the residual never gets there
    return sc


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("n", [1, 3])
def test_solve_past_100_iterations_stops_the_solver(vtp_gpu, graphs, n):
    s = vtp.solver_from_scene(_unreachable(), extra={"useGraphs": graphs})
    s.strict = False    # the reference's API: tickNsteps returns false and logs the error
    assert s.initialize()
    assert not s.tickNsteps(n)
    assert "exceeded 100 iterations" in s.last_error
    assert s.stats()["steps_done"] == 1          # stopped after the first substep
    assert not s.tickNsteps(1) and "crashed" in s.last_error
    s.destroy()


def test_without_stop_the_run_reports_at_the_end(vtp_gpu):
    s = vtp.solver_from_scene(_unreachable(), extra={"stopOnNonConvergence": False})
    s.strict = False
    assert s.initialize()
    assert not s.tickNsteps(3)
    assert "solver status after tick" in s.last_error
    assert s.stats()["status_bits"] & (1 << 3)    # ST_NOT_CONVERGED
    s.destroy()


def test_one_call_frame_reports_the_stop(vtp_gpu):
    sc = _unreachable()
    s = vtp.solver_from_scene(sc)
    s.strict = False
    assert s.initialize()
    nf = sc.objects[0].n
    p, v = vtp.HostBuffer((nf, 3)), vtp.HostBuffer((nf, 3))
    s.get_state_range_ptr(0, nf, p.ptr, v.ptr)
    assert not s.step_state_range_ptr(0, nf, p.ptr, v.ptr, 2, p.ptr, v.ptr)
    assert "exceeded 100 iterations" in s.last_error and s.stats()["steps_done"] == 1
    p.free()
    v.free()
    s.destroy()
