"""C ABI on the CPU: the library loads, exports every declared entry point, and
validates configs / objects the way the reference's setConfig / attachObject do.
No call here touches a GPU."""
import ctypes as C
import json
import re
from pathlib import Path

import pytest

import vtp
from vtp import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "vtp.h"


def declared_symbols():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"VTP_API\s+[^;(]*?\b(vtp_\w+)\s*\(", txt)))


def test_header_declarations_are_all_exported():
    lib = vtp.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} missing from the ctypes binding"


def test_checked_build_exports_the_same_entry_points():
    """The checked build (device-side bounds checks, VTP_LIBRARY=checked) is a drop-in copy."""
    path = Path(_lib.__file__).resolve().parent / "libvtp_checked.so"
    if not path.exists():
        pytest.skip("libvtp_checked.so not built")
    lib = C.CDLL(str(path), mode=C.RTLD_LOCAL)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_status_strings_and_version():
    lib = vtp.lib()
    assert lib.vtp_version().startswith(b"vtp")
    assert lib.vtp_status_string(0) == b"ok"
    assert b"100 iterations" in lib.vtp_status_string(3)


def _cfg(kind):
    return vtp.solver.Solver.__new__(vtp.solver._CLASSES[kind]).__class__


@pytest.mark.parametrize("kind", [vtp.PBF, vtp.DFSPH, vtp.IMM, vtp.IMMCT])
def test_templates_round_trip_through_set_config(kind):
    s = vtp.SolverManager().createSolver(kind)
    tpl = s.getSolverConfigTemplate()
    assert s.setConfig(tpl), s.last_error
    s.destroy()


def test_missing_required_key_is_rejected_like_the_reference():
    s = vtp.PBFSolver()
    cfg = vtp.scenes.pbf_dam_break().config
    del cfg["PBF"]["Required"]["XSPH_k"]
    assert not s.setConfig(cfg)
    assert "missing Required key: XSPH_k" in s.last_error
    cfg2 = vtp.scenes.pbf_dam_break().config
    del cfg2["PBF"]["Optional"]["gravity"]
    assert not s.setConfig(cfg2)
    assert not s.setConfig({})
    s.destroy()


def test_object_checks_follow_attach_object():
    s = vtp.DFSPHSolver()
    assert s.setConfig(vtp.scenes.dfsph_config(dt=1e-3, r=0.005, lb=(0, 0, 0), size=(1, 1, 1)))
    o = vtp.Object(vtp.Particle_Common)
    o.pos = vtp.scenes.cube(0.005, (0.1, 0.1, 0.1), (0.05, 0.05, 0.05))
    o.getObjectComponentConfig()["epmMaterial"] = 0
    o.attachSpecificSolverObjectComponentConfig({"solverType": 0, "exportFlag": False,
                                                 "velocityStart": [0, 0, 0], "colorStart": [0, 0, 0]})
    assert not s.attachObject(o)                     # solverType of another solver
    o.attachSpecificSolverObjectComponentConfig({"solverType": 1, "exportFlag": False,
                                                 "velocityStart": [0, 0, 0]})
    assert not s.attachObject(o)                     # colorStart missing
    o.attachSpecificSolverObjectComponentConfig({"solverType": 1, "exportFlag": False,
                                                 "velocityStart": [0, 0, 0], "colorStart": [0, 0, 0]})
    o.getObjectComponentConfig()["epmMaterial"] = 7
    assert not s.attachObject(o)                     # unsupported material
    o.getObjectComponentConfig()["epmMaterial"] = 0
    assert s.attachObject(o), s.last_error
    assert s.counts() == {"total": o.pos.shape[0], "fluid": o.pos.shape[0], "boundary": 0, "phases": 0}
    s.destroy()


def test_mixture_objects_need_matching_phase_fractions():
    sc = vtp.scenes.layered_mixture("IMMCT", 8, seed=1)
    s = vtp.IMMCTSolver()
    assert s.setConfig(sc.config), s.last_error
    o = vtp.Object(vtp.Particle_Common)
    o.pos = sc.objects[0].pos
    o.getObjectComponentConfig()["epmMaterial"] = 0
    o.attachSpecificSolverObjectComponentConfig({"solverType": 3, "exportFlag": False,
                                                 "velocityStart": [0, 0, 0], "phaseFraction": [1, 0, 0]})
    assert not s.attachObject(o) and "phaseFraction" in s.last_error
    o.attachSpecificSolverObjectComponentConfig({"solverType": 3, "exportFlag": False,
                                                 "velocityStart": [0, 0, 0], "phaseFraction": [1, 0]})
    assert s.attachObject(o), s.last_error
    assert s.counts()["phases"] == 2
    s.destroy()


def test_bad_extension_values_are_rejected():
    s = vtp.PBFSolver()
    cfg = vtp.scenes.pbf_dam_break().config
    cfg["B200"] = {"unroll": 3}
    assert not s.setConfig(cfg) and "unroll" in s.last_error
    cfg["B200"] = {"blockSize": 100}
    assert not s.setConfig(cfg)
    cfg["B200"] = {"cubicCube": "cubed"}
    assert not s.setConfig(cfg) and "cubicCube" in s.last_error
    cfg["B200"] = {"cubicCube": "powf"}
    assert s.setConfig(cfg), s.last_error
    cfg["B200"] = {"listLanes": 4}
    assert not s.setConfig(cfg) and "listLanes" in s.last_error
    cfg["B200"] = {"rowLanes": 2}
    assert not s.setConfig(cfg) and "rowLanes" in s.last_error
    cfg["B200"] = {"adjointLanes": 3}
    assert not s.setConfig(cfg) and "adjointLanes" in s.last_error
    cfg["B200"] = {"adjointLanes": 4}
    assert s.setConfig(cfg), s.last_error
    cfg["B200"] = {"phaseRetry": "some"}
    assert not s.setConfig(cfg) and "phaseRetry" in s.last_error
    cfg["B200"] = {"cellOrder": "hilbert"}
    assert not s.setConfig(cfg) and "cellOrder" in s.last_error
    cfg["B200"] = {"cfl": 0.4}   # a PBF solver: the adaptive step is a DFSPH extension
    assert not s.setConfig(cfg) and "DFSPH" in s.last_error
    d = vtp.DFSPHSolver()
    dcfg = vtp.scenes.dam_break("DFSPH", 500, seed=1).config
    dcfg["B200"] = {"cfl": 1.5}
    assert not d.setConfig(dcfg) and "cfl" in d.last_error
    dcfg["B200"] = {"cfl": 0.4}
    assert d.setConfig(dcfg), d.last_error
    d.destroy()
    s.destroy()


def test_field_calls_before_initialize_fail_cleanly():
    s = vtp.PBFSolver()
    buf = (C.c_float * 3)()
    rc = vtp.lib().vtp_solver_get_field(s._h, 0, buf, 12)
    assert rc == _lib.VTP_ERR_STATE
    s.destroy()


def test_range_io_before_initialize_fails_cleanly():
    s = vtp.PBFSolver()
    assert s.setConfig(vtp.scenes.pbf_dam_break().config)
    buf = (C.c_float * 30)()
    assert vtp.lib().vtp_solver_get_field_range(s._h, 0, 0, 10, buf, 120) == _lib.VTP_ERR_STATE
    assert vtp.lib().vtp_solver_set_field_range(s._h, 0, 0, 10, buf, 120) == _lib.VTP_ERR_STATE
    s.destroy()


def test_export_config_is_validated():
    cfg = vtp.scenes.pbf_dam_break().config
    cfg["EXPORT"]["SolverRequired"]["enable"] = True
    cfg["EXPORT"]["SolverRequired"]["exportFps"] = 0
    s = vtp.PBFSolver()
    assert not s.setConfig(cfg) and "exportFps" in s.last_error
    cfg["EXPORT"]["SolverRequired"]["exportFps"] = 30
    del cfg["EXPORT"]["Common"]["exportTargetDir"]
    assert not s.setConfig(cfg) and "exportTargetDir" in s.last_error
    s.destroy()


def test_product_path_fails_loudly_without_the_library(tmp_path):
    """With no built library the solver API raises; nothing falls back to a CPU path."""
    import os
    import subprocess
    import sys
    root = Path(__file__).resolve().parents[1]
    code = ("import sys; sys.path.insert(0, 'vt-physics_b200')\n"
            "import vtp\n"
            "try:\n"
            "    s = vtp.DFSPHSolver()\n"
            "except RuntimeError as e:\n"
            "    print('raised:', e)\n"
            "    sys.exit(0)\n"
            "sys.exit(3)\n")
    env = dict(os.environ, VTP_LIBRARY=str(tmp_path / "absent" / "libvtp.so"))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "is missing" in r.stdout
