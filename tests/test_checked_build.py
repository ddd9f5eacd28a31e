"""The checked build (VTP_LIBRARY=checked: every neighbour-list entry and
cell-segment slot bounds-checked on the device, an offence reported as
VTP_ERR_BOUNDS instead of an out-of-range access) gives the same trajectories
as the default build, with no check firing, on PBF, DFSPH (global-memory and
staged pressure solves) and IMM-CT scenes."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent

_RUN = r"""
import sys
import numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/vt-physics_b200"]
import vtp
out = {}
for name, sc, extra, steps in [
        ("pbf", vtp.scenes.pbf_dam_break(), None, 5),
        ("dfsph", vtp.scenes.dam_break("DFSPH", 20000, seed=9), None, 6),
        ("dfsph_staged", vtp.scenes.dam_break("DFSPH", 20000, seed=9), {"stagedSolve": True}, 6),
        ("immct", vtp.scenes.layered_mixture("IMMCT", 16, seed=3), None, 4)]:
    s = vtp.solver_from_scene(sc, extra=extra)
    ok = s.tickNsteps(steps)
    out[name + "_ok"] = np.array(ok)
    out[name + "_status"] = np.array(s.stats()["status_bits"])
    out[name + "_pos"] = s.get_field("pos")
    s.destroy()
np.savez(sys.argv[2], **out)
print("ran", vtp._lib.LIB_PATH.name)
"""


def _run(tmp_path, library):
    env = dict(os.environ)
    env.pop("VTP_LIBRARY", None)
    if library:
        env["VTP_LIBRARY"] = library
    out = tmp_path / f"{library or 'default'}.npz"
    r = subprocess.run([sys.executable, "-c", _RUN, str(ROOT), str(out)], capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout, np.load(out)


def test_checked_build_matches_default_build(vtp_gpu, tmp_path):
    if not (ROOT / "vt-physics_b200" / "vtp" / "libvtp_checked.so").exists():
        pytest.fail("libvtp_checked.so is missing: python vt-physics_b200/build.py builds it")
    msg_c, checked = _run(tmp_path, "checked")
    assert "libvtp_checked.so" in msg_c
    _, default = _run(tmp_path, None)
    for name in ("pbf", "dfsph", "dfsph_staged", "immct"):
        assert bool(checked[name + "_ok"]) and bool(default[name + "_ok"])
        assert int(checked[name + "_status"]) == 0
        assert np.array_equal(checked[name + "_pos"], default[name + "_pos"]), name
