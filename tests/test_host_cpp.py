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


_GEOMETRY_PROGRAM = r"""
#include <cstdio>
#include <fstream>
#include <string>
#include "Framework/Object.hpp"
using namespace VT_Physics;
int main(int argc, char **argv) {
    // argv[1]: output file; argv[2]: a PLY file for the particle-file object
    std::ofstream out(argv[1], std::ios::binary);
    auto dump = [&](Object &o) {
        if (!o.update()) { std::fprintf(stderr, "update failed\n"); std::exit(1); }
        auto e = o.getObjectComponent()->getElements();
        uint64_t n = e.size() / 3;
        out.write((const char *)&n, 8);
        out.write((const char *)e.data(), e.size() * 4);
    };
    Object sphere(Particle_Sphere);
    sphere.getObjectComponentConfig() = {{"particleRadius", 0.01}, {"volumeCenter", {0.5, 0.5, 0.5}}, {"volumeRadius", 0.2}};
    dump(sphere);
    Object cyl(Particle_Cylinder);
    cyl.getObjectComponentConfig() = {{"particleRadius", 0.01}, {"center", {0.5, 0.5, 0.5}},
                                      {"bottomAreaRadius", 0.2}, {"height", 0.3}};
    dump(cyl);
    Object plane(Particle_Plane);
    plane.getObjectComponentConfig() = {{"particleRadius", 0.01}, {"lb", {0, 0, 0}}, {"size", {1, 0.1, 1}}, {"layerNum", 2}};
    dump(plane);
    Object file(Particle_Common);
    file.getObjectComponentConfig() = {{"particleRadius", 0.01}, {"particleGeometryPath", std::string(argv[2])}};
    dump(file);
    return 0;
}
"""


def test_cpp_objects_generate_every_particle_type(tmp_path):
    """Sphere, cylinder and plane objects and a Particle_Common object loaded from a PLY file
    (the reference's ObjectComponents update paths) through the C++ host interface."""
    sys.path.insert(0, str(PKG))
    import build
    from vtp import model
    build.build()
    src = tmp_path / "geometry.cpp"
    src.write_text(_GEOMETRY_PROGRAM)
    exe = build.build_host_program(src, tmp_path / "geometry")
    pts = np.random.default_rng(3).uniform(-1, 1, (50, 3)).astype(np.float32)
    ply = model.write_ply(tmp_path, "cloud", pts)
    dump = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(dump), str(ply)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    raw = dump.read_bytes()
    got, off = [], 0
    while off < len(raw):
        n = int(np.frombuffer(raw[off:off + 8], np.uint64)[0])
        got.append(np.frombuffer(raw[off + 8:off + 8 + 12 * n], np.float32).reshape(n, 3))
        off += 8 + 12 * n
    want = [model.generate({"genType": 1, "particleRadius": 0.01, "volumeCenter": [0.5, 0.5, 0.5], "volumeRadius": 0.2}),
            model.generate({"genType": 3, "particleRadius": 0.01, "center": [0.5, 0.5, 0.5],
                            "bottomAreaRadius": 0.2, "height": 0.3}),
            model.generate({"genType": 4, "particleRadius": 0.01, "lb": [0, 0, 0], "size": [1, 0.1, 1], "layerNum": 2}),
            model.read_ply(ply)]
    assert len(got) == 4
    for a, b in zip(got, want):
        assert a.shape == b.shape and a.shape[0] > 0 and np.array_equal(a, b)
