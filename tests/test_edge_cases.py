"""Edge cases of the neighbour search and the solvers, library against the oracle:
truncated lists, particles outside the grid, coincident particles, the three
fluid/boundary attach orders, fluid-only / boundary-only / one-particle scenes."""
import numpy as np
import pytest

from vtp import scenes

pytestmark = pytest.mark.gpu


def _scene(kind, objs, r=0.125, lb=(-1.0,) * 3, size=(5.0,) * 3, max_nbr=60):
    if kind == "PBF":
        cfg = scenes.pbf_config(dt=1e-3, r=r, lb=lb, size=size)
    else:
        cfg = scenes.dfsph_config(dt=1e-3, r=r, lb=lb, size=size)
    cfg[kind]["Required"]["maxNeighborNum"] = max_nbr
    return scenes.Scene(kind, cfg, [scenes.SceneObject(n, np.asarray(p, np.float32), m) for n, p, m in objs])


def _lattice(n, step=0.25, origin=0.0):
    g = np.arange(n, dtype=np.float32) * np.float32(step) + np.float32(origin)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1).astype(np.float32)


def _compare(vtp, oracle_lib, sc, ticks=0, lanes=0):
    s = vtp.solver_from_scene(sc, extra={"listLanes": lanes})
    assert s.initialize(), s.last_error
    if ticks:
        assert s.tickNsteps(ticks), s.last_error
    grid = oracle_lib.make_grid(sc.config[sc.solver]["Required"])
    pos = s.get_field("pos")
    oc, on, oi, ok = oracle_lib.neighbors(pos, grid)
    cnt, nb = s.get_neighbors(grid.maxnbr)
    assert np.array_equal(cnt, oc)
    assert np.array_equal(nb, on)
    ids, keys = s.get_sorted_order()
    inside = keys != 0xFFFFFFFF
    assert np.array_equal(ids[: inside.sum()], oi) and np.array_equal(keys[: inside.sum()], ok)
    return s


@pytest.mark.parametrize("lanes", [1, 8])
@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_truncated_lists_match_oracle(vtp_gpu, oracle_lib, kind, lanes):
    # 33 neighbours per interior particle (spacing h/2, exact binary fractions) against a cap of 10
    fluid = _lattice(9)
    sc = _scene(kind, [("fluid", fluid, 0)], max_nbr=10)
    s = _compare(vtp_gpu, oracle_lib, sc, lanes=lanes)
    cnt, _ = s.get_neighbors(10)
    assert cnt.max() == 10
    assert s.tickNsteps(1)
    assert s.stats()["neighbor_overflow"] > 0
    s.destroy()


def test_particles_outside_the_grid(vtp_gpu, oracle_lib):
    fluid = np.concatenate([_lattice(4, origin=0.5), np.array([[9.0, 9.0, 9.0], [-3.0, 0.5, 0.5]], np.float32)])
    sc = _scene("PBF", [("fluid", fluid, 0)])
    s = _compare(vtp_gpu, oracle_lib, sc)
    cnt, _ = s.get_neighbors(60)
    assert cnt[-1] == 0 and cnt[-2] == 0
    s.destroy()


def test_coincident_particles_are_not_neighbours(vtp_gpu, oracle_lib):
    fluid = np.concatenate([_lattice(3, origin=0.5), np.array([[0.5, 0.5, 0.5], [0.75, 0.5, 0.5]], np.float32)])
    sc = _scene("PBF", [("fluid", fluid, 0)])
    s = _compare(vtp_gpu, oracle_lib, sc)
    s.destroy()


@pytest.mark.parametrize("lanes", [1, 8])
@pytest.mark.parametrize("order", ["fluid_first", "boundary_first", "interleaved"])
def test_attach_orders_match_oracle(vtp_gpu, oracle_lib, order, lanes):
    sc0 = scenes.dam_break("DFSPH", 2000, seed=40)
    f, b = sc0.objects
    half = f.n // 2
    if order == "fluid_first":
        objs = [("f", f.pos, 0), ("b", b.pos, 1)]
    elif order == "boundary_first":
        objs = [("b", b.pos, 1), ("f", f.pos, 0)]
    else:
        objs = [("f1", f.pos[:half], 0), ("b", b.pos, 1), ("f2", f.pos[half:], 0)]
    req = sc0.config["DFSPH"]["Required"]
    sc = _scene("DFSPH", objs, r=req["particleRadius"], lb=req["simSpaceLB"], size=req["simSpaceSize"])
    s = _compare(vtp_gpu, oracle_lib, sc, ticks=2, lanes=lanes)
    s.destroy()


@pytest.mark.parametrize("kind", ["PBF", "DFSPH"])
def test_fluid_only_boundary_only_and_single_particle(vtp_gpu, oracle_lib, kind):
    for objs in ([("fluid", _lattice(5, origin=0.5), 0)],
                 [("box", _lattice(5, origin=0.5), 1)],
                 [("one", np.array([[0.5, 0.5, 0.5]], np.float32), 0)]):
        sc = _scene(kind, objs)
        s = _compare(vtp_gpu, oracle_lib, sc)
        assert s.tickNsteps(3), s.last_error
        p = s.get_field("pos")
        assert np.all(np.isfinite(p))
        if objs[0][2] == 1:
            assert np.array_equal(p, objs[0][1])   # boundary particles never move
        s.destroy()
