"""PLY export (EXPORT block of the solver config): the reference's file layout,
frame trigger and ASCII format (ExportUtil.cpp:28-88, PBFSolver.cpp:248-368)."""
import json

import numpy as np
import pytest

import vtp
from vtp import scenes

pytestmark = pytest.mark.gpu


def read_ply(path):
    lines = path.read_text().splitlines()
    assert lines[0] == "ply" and lines[1] == "format ascii 1.0"
    n = int(lines[2].split()[-1])
    props = [ln.split()[-1] for ln in lines[3:lines.index("end_header")]]
    body = lines[lines.index("end_header") + 1:]
    assert len(body) == n
    data = np.array([[float(x) for x in ln.split()] for ln in body]) if n else np.zeros((0, len(props)))
    return props, data


def _solver(sc, policy, out, fps):
    cfg = json.loads(json.dumps(sc.config))
    cfg["EXPORT"] = {"Common": {"exportTargetDir": str(out), "exportFilePrefix": "frame_", "exportFileType": "PLY"},
                     "SolverRequired": {"enable": True, "exportFps": fps, "exportGroupPolicy": policy}}
    sc2 = scenes.Scene(sc.solver, cfg, sc.objects)
    return vtp.solver_from_scene(sc2)


@pytest.mark.parametrize("policy", ["MERGE", "SPLIT"])
def test_pbf_export_files(vtp_gpu, tmp_path, policy):
    sc = scenes.dam_break("PBF", 2000, seed=21)
    dt = sc.config["PBF"]["Required"]["timeStep"]
    # frames advance when simTime >= frame / fps; with 1/fps = 2.4 dt the frames fall on
    # substeps 1, 3 and 5 whatever the FP32 rounding of the accumulated time
    s = _solver(sc, policy, tmp_path, fps=1.0 / (2.4 * dt))
    assert s.initialize() and s.tickNsteps(5)
    pos = s.get_field("pos")
    color = s.get_field("color")
    nf = sc.objects[0].n
    if policy == "MERGE":
        files = sorted((tmp_path / "Fluid").glob("*.ply"), key=lambda p: int(p.stem))
        assert [p.stem for p in files] == ["1", "2", "3"]
        props, d = read_ply(files[-1])
        assert props == ["x", "y", "z"]
        assert np.allclose(d, pos[:nf], rtol=1e-5, atol=1e-6)
        assert not (tmp_path / "Boundary").exists()        # the box has exportFlag false
    else:
        files = sorted((tmp_path / "fluid").glob("*.ply"))
        assert [p.name for p in files] == ["frame_1.ply", "frame_2.ply", "frame_3.ply"]
        props, d = read_ply(files[-1])
        assert props == ["x", "y", "z", "red", "green", "blue"]
        assert np.allclose(d[:, :3], pos[:nf], rtol=1e-5, atol=1e-6)
        assert np.allclose(d[:, 3:], color[:nf])
    s.destroy()


def test_mixture_merge_exports_phase_fractions(vtp_gpu, tmp_path):
    sc = scenes.layered_mixture("IMMCT", 10, seed=2)
    key = sc.solver
    dt = sc.config[key]["Required"]["timeStep"]
    s = _solver(sc, "MERGE", tmp_path, fps=1.0 / dt)
    assert s.initialize() and s.tickNsteps(2)
    files = sorted((tmp_path / "Fluid").glob("*.ply"), key=lambda p: int(p.stem))
    assert len(files) == 2
    props, d = read_ply(files[-1])
    P = len(sc.config[key]["Required"]["phaseRestDensity"])
    assert props == ["x", "y", "z", "red", "green", "blue"] + [f"p{k + 1}" for k in range(P)]
    fluid = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    frac = s.get_field("vol_frac")
    assert np.allclose(d[:, 6:], frac[fluid], rtol=1e-5, atol=1e-6)
    s.destroy()
