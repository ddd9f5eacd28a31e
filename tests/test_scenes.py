"""Scene generators: counts and coordinates follow the reference generators' arithmetic."""
import numpy as np

from vtp import scenes


def test_pbf_dam_break_counts():
    sc = scenes.pbf_dam_break()
    assert [o.n for o in sc.objects] == [16000, 35315]
    wall = sc.objects[1].pos
    # 2 layers low (0.01, 0.03) and 3 high (0.97, 0.99, 1.01) per axis
    assert np.isclose(wall[:, 0].min(), 0.01) and np.isclose(wall[:, 0].max(), 1.01)


def test_dfsph_1m_counts_and_clearance():
    sc = scenes.dfsph_1m()
    f, b = sc.objects
    assert f.n == 1_000_000 and b.n == 453_957
    # the far z wall starts one spacing beyond the fluid
    assert f.pos[:, 2].max() < 1.035 - 0.005


def test_immct_500k_counts():
    sc = scenes.immct_500k()
    assert [o.n for o in sc.objects] == [250_000, 250_000, 187_369]
    assert sc.objects[0].phase_fraction == (0.0, 1.0) and sc.objects[1].phase_fraction == (1.0, 0.0)


def test_cube_float32_running_sum():
    # x += diameter in FP32 from lb + r while x < lb + size (ModelHandler.cpp:50-64)
    p = scenes.cube(0.01, (0.04, 0.04, 0.04), (0.4, 0.8, 0.4))
    xs = np.unique(p[:, 0])
    assert xs.size == 20 and xs.dtype == np.float32
    ref = [np.float32(0.04) + np.float32(0.01)]
    for _ in range(19):
        ref.append(np.float32(ref[-1] + np.float32(0.02)))
    assert np.array_equal(xs, np.array(ref, np.float32))


def test_jitter_is_seeded_and_bounded():
    base = scenes.cube(0.005, (0, 0, 0), (0.1, 0.1, 0.1))
    a = scenes.jitter(base, 0.05, 0.01, 7)
    b = scenes.jitter(base, 0.05, 0.01, 7)
    c = scenes.jitter(base, 0.05, 0.01, 8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.max(np.abs(a.astype(np.float64) - base)) <= 0.05 * 0.01 + 1e-7


def test_splitmix64_known_values():
    # SplitMix64 from seed 0: first outputs 0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4
    u = scenes.splitmix64_uniform(0, 2)
    expect = np.array([0xE220A8397B1DCDAF >> 11, 0x6E789E6AA1B965F4 >> 11], np.float64) / 2.0 ** 53
    assert np.array_equal(u, expect)
