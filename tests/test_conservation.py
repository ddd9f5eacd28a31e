"""FP64 conservation and density-error sums on the device (vtp_solver_get_conservation)
against the same sums formed on the host from the exported fields."""
import numpy as np
import pytest

from vtp import scenes

pytestmark = pytest.mark.gpu


def _host_sums(s, sc, mask):
    f64 = np.float64
    vel = s.get_field("vel")[mask].astype(f64)
    if sc.solver == "PBF":
        m = s.get_field("mass")[mask].astype(f64)
        derr = s.get_field("density")[mask].astype(f64) * f64(np.float32(1.0 / 1000.0)) - 1.0
    elif sc.solver == "DFSPH":
        m = s.get_field("mass")[mask].astype(f64)
        derr = s.get_field("density")[mask].astype(f64) - 1.0
    else:   # mixture: mass = rest density * volume, formed in FP64 like the device sums
        m = s.get_field("rest_density")[mask].astype(f64) * s.get_field("volume")[mask].astype(f64)
        derr = s.get_field("density")[mask].astype(f64) - 1.0
    out = {"mass": m.sum(), "mom": (m[:, None] * vel).sum(0), "ke": 0.5 * (m * (vel ** 2).sum(1)).sum(),
           "derr": derr.mean()}
    if sc.solver in ("IMM", "IMMCT"):
        vol = s.get_field("volume")[mask].astype(f64)
        frac = s.get_field("vol_frac")[mask].astype(f64)
        rho = np.array(sc.config[sc.solver]["Required"]["phaseRestDensity"], np.float32).astype(f64)
        out["phase"] = (vol[:, None] * frac * rho[None, :]).sum(0)
    return out


@pytest.mark.parametrize("kind", ["PBF", "DFSPH", "IMMCT"])
def test_device_sums_match_host_sums(vtp_gpu, kind):
    vtp = vtp_gpu
    sc = {"PBF": lambda: scenes.pbf_dam_break(),
          "DFSPH": lambda: scenes.dam_break("DFSPH", 8000, seed=51),
          "IMMCT": lambda: scenes.layered_mixture("IMMCT", 16, seed=52)}[kind]()
    s = vtp.solver_from_scene(sc)
    assert s.tickNsteps(5), s.last_error
    mask = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    d = s.conservation()
    h = _host_sums(s, sc, mask)
    rel = lambda a, b: abs(a - b) / max(abs(b), 1e-300)
    assert d["fluid_particles"] == int(mask.sum())
    assert rel(d["fluid_mass"], h["mass"]) < 1e-12
    assert rel(d["kinetic_energy"], h["ke"]) < 1e-12
    scale = np.abs(h["mom"]).max()
    assert np.max(np.abs(np.array(d["momentum"]) - h["mom"])) <= 1e-12 * scale
    assert abs(d["mean_density_error"] - h["derr"]) <= 1e-6 * max(abs(h["derr"]), 1e-9) + 1e-12
    if kind == "IMMCT":
        assert len(d["phase_mass"]) == 2
        assert np.allclose(d["phase_mass"], h["phase"], rtol=1e-12, atol=0)
    # a fixed summation order: the same state gives the same bits
    assert s.conservation() == d
    s.destroy()


def test_per_scene_sums_add_up(vtp_gpu):
    vtp = vtp_gpu
    mix = [scenes.dam_break("DFSPH", 3000, seed=53), scenes.dam_break("DFSPH", 5000, seed=54)]
    b, _ = vtp.solver_from_scenes(mix)
    assert b.initialize() and b.tickNsteps(3)
    a, c, both = b.conservation(0), b.conservation(1), b.conservation()
    assert a["fluid_particles"] + c["fluid_particles"] == both["fluid_particles"]
    assert abs(a["fluid_mass"] + c["fluid_mass"] - both["fluid_mass"]) <= 1e-12 * both["fluid_mass"]
    b.destroy()
