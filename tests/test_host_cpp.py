"""The C++ host interface (vt-physics_b200/host: the reference's Solver / Object /
SolverManager classes over the C ABI), driven by a C++ program written the way the
reference's examples are."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "vt-physics_b200"


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    sys.path.insert(0, str(PKG))
    import build
    build.build()
    out = tmp_path_factory.mktemp("host") / "dam_break"
    return build.build_host_program(PKG / "host" / "examples" / "dam_break.cpp", out)


def run(exe, *args):
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_cpp_generators_match_the_python_generators(example, tmp_path):
    from vtp import scenes
    dump = tmp_path / "pos.bin"
    out = run(example, "PBF", "0", "--dry", "--dump", str(dump))
    assert (out["fluid"], out["boundary"]) == (16000, 35315)
    got = np.fromfile(dump, np.float32).reshape(-1, 3)
    want = np.concatenate([scenes.cube(0.01, (0.04, 0.04, 0.04), (0.4, 0.8, 0.4)),
                           scenes.box(0.01, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2)])
    assert np.array_equal(got, want)


def test_cpp_config_errors_are_reported(example, tmp_path):
    r = subprocess.run([str(example), "PBF", "0", "--dry"], capture_output=True, text=True)
    assert r.returncode == 0 and "[vtp]" not in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_cpp_program_matches_python_api(vtp_gpu, example, kind):
    from vtp import scenes
    out = run(example, kind, "8")
    r = 0.01 if kind == "PBF" else 0.005
    cfg = (scenes.pbf_config(dt=1.0 / 240.0, r=r, lb=(-0.1,) * 3, size=(1.2,) * 3) if kind == "PBF" else
           scenes.dfsph_config(dt=1e-3, r=r, lb=(-0.1,) * 3, size=(1.2,) * 3))
    fluid = scenes.cube(r, (0.04, 0.04, 0.04), (0.4, 0.8, 0.4))
    wall = scenes.box(r, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2 if kind == "PBF" else 3)
    sc = scenes.Scene(kind, cfg, [scenes.SceneObject("fluid", fluid, 0, export_flag=True),
                                  scenes.SceneObject("box", wall, 1)])
    s = vtp_gpu.solver_from_scene(sc)
    assert s.initialize() and s.tickNsteps(8)
    mean = s.get_field("pos")[: fluid.shape[0]].astype(np.float64).mean(0)
    s.destroy()
    assert (out["fluid"], out["boundary"]) == (fluid.shape[0], wall.shape[0])
    assert np.allclose(out["mean"], mean, rtol=1e-8, atol=0)
