"""The autotuner's search and cache, with a fake measurement (no GPU)."""
import math

import pytest

from vtp import autotune as A


def fake(costs):
    """measure(config) from a per-dimension cost table (sum of the chosen values' costs)."""
    calls = []

    def measure(cfg):
        calls.append(dict(cfg))
        tile = "staged" if cfg["stagedSolve"] else cfg["cellOrder"]
        if tile == "linear" and cfg.get("unroll") == 8:
            raise RuntimeError("rejected configuration")
        return (costs["blockSize"][cfg["blockSize"]] + costs["unroll"][cfg["unroll"]] + costs["cellTile"][tile]
                + costs.get("listLanes", {}).get(cfg.get("listLanes"), 0.0))
    return measure, calls


COSTS = {"blockSize": {64: 3.0, 128: 2.0, 256: 1.5}, "unroll": {1: 4.0, 2: 3.0, 4: 2.5, 8: 2.6},
         "cellTile": {"brick": 1.0, "linear": 2.0, "staged": 0.5}, "listLanes": {0: 0.2, 1: 0.2, 8: 0.1}}


def test_coordinate_descent_finds_the_separable_optimum_and_measures_each_point_once():
    measure, calls = fake(COSTS)
    res = A.tune(measure, "DFSPH")
    assert res["best"] == {"blockSize": 256, "unroll": 4, "cellTile": "staged", "listLanes": 8}
    assert res["config"] == {"blockSize": 256, "unroll": 4, "listLanes": 8, "cellOrder": "brick", "stagedSolve": True}
    assert math.isclose(res["ms_per_step"], 1.5 + 2.5 + 0.5 + 0.1)
    keys = [tuple(sorted(c.items())) for c in calls]
    assert len(keys) == len(set(keys))          # no configuration measured twice
    assert len(calls) < 3 * 4 * 3 * 3           # fewer than the full product


def test_failing_configurations_are_skipped():
    costs = dict(COSTS)
    costs["cellTile"] = {"brick": 1.0, "linear": 0.1, "staged": 5.0}
    costs["unroll"] = {1: 4.0, 2: 3.0, 4: 2.5, 8: 0.1}   # unroll 8 is best but "linear" rejects it
    measure, _ = fake(costs)
    res = A.tune(measure, "DFSPH")
    assert math.isfinite(res["ms_per_step"])
    assert not (res["best"]["cellTile"] == "linear" and res["best"]["unroll"] == 8)
    assert any(math.isinf(t["ms_per_step"]) for t in res["trials"])


def test_pbf_has_no_staged_tile_and_arithmetic_keys_are_optional():
    assert "staged" not in A.candidates("cellTile", "PBF")
    assert "staged" in A.candidates("cellTile", "DFSPH")
    assert "rowLanes" in A.dims_for("PBF") and "rowLanes" not in A.dims_for("PBF", allow_arithmetic=False)
    assert "rowLanes" not in A.dims_for("DFSPH")


def test_cache_round_trip_and_b200_fallback(tmp_path):
    path = tmp_path / "tuned.json"
    measure, _ = fake(COSTS)
    res = A.tune(measure, "DFSPH")
    A.store("dfsph_1m", res, gpu="NVIDIA B200", path=path)
    assert A.tuned_extra("dfsph_1m", gpu="NVIDIA B200", path=path) == res["config"]
    # another B200 name (driver or SKU string) finds the B200 entry; other GPUs get nothing
    assert A.tuned_extra("dfsph_1m", gpu="NVIDIA B200 SXM", path=path) == res["config"]
    assert A.tuned_extra("dfsph_1m", gpu="Some Other GPU", path=path) == {}
    assert A.tuned_extra("pbf", gpu="NVIDIA B200", path=path) == {}


def test_workload_keys():
    assert A.workload_key("PBF", 16000) == "PBF:2^14"
    assert A.workload_key("DFSPH", 1_000_000) == "DFSPH:2^20"
    assert A.workload_key("DFSPH", 5, name="dfsph_1m") == "dfsph_1m"


def test_committed_cache_is_well_formed():
    cache = A.load_cache()
    for gpu, table in cache.items():
        for key, entry in table.items():
            cfg = entry["B200"]
            assert set(cfg) <= {"blockSize", "unroll", "rowLanes", "listLanes", "cellOrder", "stagedSolve",
                                "adjointLanes"}
            assert cfg.get("cellOrder", "brick") in ("brick", "linear")


def test_adjoint_lanes_are_tuned_on_their_own_measurement_and_keep_the_tuned_tile():
    """The differentiable workload's second search: only "adjointLanes", whose config carries
    no cell-tile keys, so merging it into the forward's tuned block keeps that block's tile."""
    calls = []

    def measure(cfg):
        calls.append(dict(cfg))
        assert set(cfg) == {"adjointLanes"}
        return {1: 2.3, 2: 2.2, 4: 2.0, 8: 2.1}[cfg["adjointLanes"]]

    res = A.tune(measure, "PBF", ("adjointLanes",))
    assert res["best"] == {"adjointLanes": 4} and res["config"] == {"adjointLanes": 4}
    assert len(calls) == 4
    forward = {"blockSize": 256, "unroll": 4, "cellOrder": "linear", "stagedSolve": False}
    forward.update(res["config"])
    assert forward["cellOrder"] == "linear" and forward["adjointLanes"] == 4
    assert A.DIMENSIONS["adjointLanes"] == (1, 2, 4, 8) and A.DEFAULTS["adjointLanes"] == 1
