"""bench.py's host-side plumbing on the CPU: default configurations, workload scenes and
the self-launch of ranks (the command it builds; nothing is run)."""
import importlib
import sys

import pytest


@pytest.fixture(scope="module")
def bench():
    return importlib.import_module("bench")


def test_default_extra_merges_tuned_and_fixed_keys(bench):
    e = bench.default_extra("dfsph_1m")
    assert e["cfl"] == 0.4                       # the benchmark's adaptive step, always on
    assert set(e) - {"cfl"} <= {"blockSize", "unroll", "rowLanes", "listLanes", "cellOrder", "stagedSolve"}
    assert "cfl" not in bench.default_extra("pbf")


def test_workload_scenes(bench):
    assert bench.make_scene("pbf_m1").config["PBF"]["Required"]["particleRadius"] == 0.05
    assert bench.make_scene("pbf").config["PBF"]["Required"]["particleRadius"] == 0.01
    a, b = bench.batched_mix("batched"), bench.batched_mix("batched_m1")
    assert len(a) == len(b) == 64
    assert [s.n_fluid for s in a[48:]] == [s.n_fluid for s in b[48:]]     # the DFSPH half is shared
    assert all(s.config["PBF"]["Required"]["particleRadius"] == 0.05 for s in b[:48])


def test_gpus_flag_starts_its_own_ranks(bench, monkeypatch):
    calls = []
    monkeypatch.setattr(bench.subprocess, "call", lambda cmd: calls.append(cmd) or 0)
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "4", "--steps", "5", "--warmup", "3"])
    assert bench.main() == 0
    cmd = calls[0]
    assert "torch.distributed.run" in cmd and "--nproc-per-node=4" in cmd
    assert "--master-addr" in cmd and cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-6:] == ["--gpus", "4", "--steps", "5", "--warmup", "3"]
    assert cmd[:3] == ["timeout", "-k", "60"]


def test_tick_together_runs_every_solver_at_once_and_reports_failures():
    """tick_together submits each solver's substeps from its own thread: all run at the same
    time (a barrier only the whole group passes), results are combined, errors re-raised."""
    import threading
    from vtp.solver import tick_together

    gate = threading.Barrier(3, timeout=10)

    class Fake:
        def __init__(self, ok=True, boom=False):
            self.ok, self.boom, self.n = ok, boom, 0

        def tickNsteps(self, n):
            gate.wait()          # returns only when all three are inside their call
            if self.boom:
                raise RuntimeError("tick failed")
            self.n += n
            return self.ok

    a, b, c = Fake(), Fake(), Fake()
    assert tick_together([a, b, c], 7) and a.n == b.n == c.n == 7
    assert not tick_together([Fake(), Fake(ok=False), Fake()], 1)
    with pytest.raises(RuntimeError, match="tick failed"):
        tick_together([Fake(), Fake(boom=True), Fake()], 1)
