"""Particle geometry against the reference's own build (CPU: host code only).

oracle/_ref/libvtref.so is the reference compiled from its sources; its
ModelHandler generators and ExportUtil run on the host, so these tests need
no GPU.  They pin:
  * vtp_generate_particles (all five particle generators) to
    ModelHandler::generateObjectElements bit for bit, and the project's
    Python scene builders (vtp.scenes.cube / box, which make every benchmark
    scene) to the same generators;
  * vtp_write_ply to ExportUtil::exportAsPly byte for byte (same arrays in,
    same text out; only the file path differs: the reference joins the
    directory and the name with a backslash);
  * vtp_read_ply: reading the files either writer produced gives back the
    positions they hold (ASCII, 6 significant digits), binary PLY exactly.
"""
import struct

import numpy as np
import pytest

from vtp import model, scenes

pytestmark = []

GENERATORS = [
    {"genType": 2, "particleRadius": 0.01, "lb": [0.04, 0.04, 0.04], "size": [0.4, 0.8, 0.4]},
    {"genType": 2, "particleRadius": 0.005, "lb": [0.03, 0.03, 0.03], "size": [1.0, 0.25, 1.0]},
    {"genType": 2, "particleRadius": 0.05, "lb": [-1.3, 0.7, -0.11], "size": [0.9, 0.77, 0.5]},
    {"genType": 5, "particleRadius": 0.01, "lb": [0, 0, 0], "size": [1, 1, 1], "layerNum": 2},
    {"genType": 5, "particleRadius": 0.005, "lb": [0, 0, 0], "size": [2.0, 1.5, 1.06], "layerNum": 3},
    {"genType": 5, "particleRadius": 0.05, "lb": [-2.0, -0.5, -1.0], "size": [4.0, 3.0, 2.0], "layerNum": 1},
    {"genType": 1, "particleRadius": 0.01, "volumeCenter": [0.5, 0.5, 0.5], "volumeRadius": 0.2},
    {"genType": 1, "particleRadius": 0.025, "volumeCenter": [-0.3, 1.1, 0.07], "volumeRadius": 0.51},
    {"genType": 3, "particleRadius": 0.01, "center": [0.5, 0.5, 0.5], "bottomAreaRadius": 0.2, "height": 0.3},
    {"genType": 3, "particleRadius": 0.02, "center": [-0.2, 0.9, 1.3], "bottomAreaRadius": 0.37, "height": 0.81},
    {"genType": 4, "particleRadius": 0.01, "lb": [0, 0, 0], "size": [1, 0.1, 1], "layerNum": 2},
    {"genType": 4, "particleRadius": 0.015, "lb": [-0.4, 0.2, 0.33], "size": [0.7, 0.3, 1.1], "layerNum": 3},
]


@pytest.fixture(scope="module")
def ref():
    from oracle.ref import ref as R
    if not R.available():
        pytest.skip("the reference build oracle/_ref/libvtref.so is not present")
    return R


@pytest.mark.parametrize("cfg", GENERATORS, ids=lambda c: f"gen{c['genType']}-r{c['particleRadius']}")
def test_generators_match_reference_bit_exact(ref, cfg):
    ours = model.generate(cfg)
    theirs = ref.generate(cfg)
    assert ours.shape == theirs.shape and ours.shape[0] > 0
    assert np.array_equal(ours.view(np.uint32), theirs.view(np.uint32))


@pytest.mark.parametrize("cfg", [c for c in GENERATORS if c["genType"] in (2, 5)],
                         ids=lambda c: f"gen{c['genType']}-r{c['particleRadius']}")
def test_scene_builders_match_reference_generators(ref, cfg):
    """vtp.scenes restates the cube and box generators in numpy; every benchmark scene is built
    with them."""
    r = np.float32(cfg["particleRadius"])
    if cfg["genType"] == 2:
        ours = scenes.cube(float(r), tuple(cfg["lb"]), tuple(cfg["size"]))
    else:
        ours = scenes.box(float(r), tuple(cfg["lb"]), tuple(cfg["size"]), cfg["layerNum"])
    theirs = ref.generate(cfg)
    assert np.array_equal(np.asarray(ours, np.float32).view(np.uint32), theirs.view(np.uint32))


def _arrays(n, P, seed):
    rng = np.random.default_rng(seed)
    pos = (rng.normal(size=(n, 3)) * np.array([1.0, 1e-3, 300.0])).astype(np.float32)
    pos[0] = (0.0, -0.0, 1e-7)
    color = rng.uniform(size=(n, 3)).astype(np.float32)
    frac = rng.dirichlet(np.ones(P), size=n).astype(np.float32) if P else None
    return pos, color, frac


@pytest.mark.parametrize("kind", ["pos", "pos+color", "pos+color+phases"])
def test_ply_writer_matches_reference_text(ref, tmp_path, kind):
    pos, color, frac = _arrays(257, 3, 7)
    c = color if kind != "pos" else None
    ph = frac if kind == "pos+color+phases" else None
    ours = model.write_ply(tmp_path / "ours", "frame_7", pos, c, ph)
    theirs = ref.export_ply(str(tmp_path / "theirs"), "frame_7", pos, c, ph)
    assert ours.read_bytes() == open(theirs, "rb").read()


def test_ply_reader_reads_both_writers(ref, tmp_path):
    pos, color, frac = _arrays(300, 2, 9)
    a = model.read_ply(model.write_ply(tmp_path, "a", pos, color, frac))
    b = model.read_ply(ref.export_ply(str(tmp_path / "r"), "b", pos, color, frac))
    assert np.array_equal(a, b)
    # ASCII with the default 6 significant digits
    assert np.allclose(a, pos, rtol=1e-5, atol=0)


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian"])
def test_ply_reader_binary_is_exact(tmp_path, fmt):
    pos, _, _ = _arrays(100, 0, 11)
    e = "<" if fmt == "binary_little_endian" else ">"
    head = (f"ply\nformat {fmt} 1.0\ncomment made by a test\nelement vertex {len(pos)}\n"
            "property float x\nproperty float y\nproperty float z\nproperty uchar red\nproperty double w\n"
            "element face 1\nproperty list uchar int vertex_indices\nend_header\n").encode()
    body = b"".join(struct.pack(e + "fffBd", *p, 7, 0.5) for p in pos) + struct.pack(e + "Biii", 3, 0, 1, 2)
    path = tmp_path / "bin.ply"
    path.write_bytes(head + body)
    got = model.read_ply(path)
    assert np.array_equal(got, pos)


def test_ply_reader_rejects_bad_files(tmp_path):
    from vtp import VtpError
    p = tmp_path / "bad.ply"
    p.write_text("ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\nproperty float y\nend_header\n1 2\n3 4\n")
    with pytest.raises(VtpError):
        model.read_ply(p)
    with pytest.raises(VtpError):
        model.read_ply(tmp_path / "missing.ply")
