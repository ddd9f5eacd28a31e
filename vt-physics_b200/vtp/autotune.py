"""Launch-configuration autotuner for the neighbour passes, and its cache.

Tuned dimensions (keys of the solver config's "B200" block):
  * blockSize  - threads per block = fluid rows per scene-offset tile of the
                 pressure solve (32..256);
  * unroll     - neighbour-list entries whose gathers a thread keeps in
                 flight (1, 2, 4, 8);
  * cell tile  - how rows are grouped into cells and cell tiles: "linear"
                 (the reference's cell order), "brick" (4 x 4 x 4-cell
                 bricks, Morton order inside) or, for DFSPH, "staged" (bricks
                 whose neighbourhoods the pressure solve copies into shared
                 memory; "cellOrder" / "stagedSolve" / "stageRows");
  * rowLanes   - threads per row of the PBF neighbour passes (1, 4, 8);
  * listLanes  - threads per row of the list builder (0: by row count, 1, 8);
  * adjointLanes - threads per row of the PBF adjoint's neighbour passes (1, 2,
                 4, 8), tuned for the differentiable workload only, after the
                 forward's keys, on the backward's wall-clock time.
Every candidate is timed with the library's per-kernel CUDA-event profiler
(the substep's kernel time; the adjoint's keys: a recorded rollout's backward),
by coordinate descent from the current best:
each dimension in turn is swept with the others fixed, until a full pass
changes nothing.  `tune` takes the measurement as a function, so the search
itself runs without a GPU (tests/test_autotune.py).

Results are cached in vtp/tuned.json, keyed by the GPU's name and a workload
key (solver type and fluid-particle count rounded to a power of two, or a
named workload); `tuned_extra` returns the cached "B200" block, which
bench.py and batched runs apply by default.  Keys that change FP32 arithmetic
(rowLanes) are tuned only when the caller allows it: a batched run and the
per-scene runs it is compared with must share them.
"""
from __future__ import annotations

import json
import math
import time
from pathlib import Path

CACHE = Path(__file__).resolve().parent / "tuned.json"

DIMENSIONS = {
    "blockSize": (64, 128, 256),
    "unroll": (1, 2, 4, 8),
    "cellTile": ("brick", "linear", "staged"),
    "rowLanes": (1, 4, 8),
    "listLanes": (0, 1, 8),
    "adjointLanes": (1, 2, 4, 8),
}
DEFAULTS = {"blockSize": 128, "unroll": 4, "cellTile": "brick", "rowLanes": 1, "listLanes": 0, "adjointLanes": 1}
# Dimensions each solver type has (the others leave its kernels unchanged).
SOLVER_DIMS = {
    "PBF": ("blockSize", "unroll", "cellTile", "rowLanes", "listLanes"),
    "DFSPH": ("blockSize", "unroll", "cellTile", "listLanes"),
    "IMM": ("blockSize", "unroll", "cellTile", "listLanes"),
    "IMMCT": ("blockSize", "unroll", "cellTile", "listLanes"),
}


def to_config(point: dict) -> dict:
    """The "B200" config keys of a search point (the cell tile's keys only when the point has
    one, so a search over other keys leaves a tuned tile in place)."""
    out = {k: point[k] for k in ("blockSize", "unroll", "rowLanes", "listLanes", "adjointLanes") if k in point}
    if "cellTile" in point:
        tile = point["cellTile"]
        out["cellOrder"] = "linear" if tile == "linear" else "brick"
        out["stagedSolve"] = tile == "staged"
    return out


def dims_for(solver: str, allow_arithmetic: bool = True) -> tuple:
    """Tuned dimensions of a solver type; without `allow_arithmetic`, only those that leave the
    FP32 results unchanged."""
    d = SOLVER_DIMS[solver]
    if not allow_arithmetic:
        d = tuple(x for x in d if x != "rowLanes")
    return d


def candidates(dim: str, solver: str) -> tuple:
    vals = DIMENSIONS[dim]
    if dim == "cellTile" and solver != "DFSPH":
        vals = tuple(v for v in vals if v != "staged")
    return vals


def tune(measure, solver: str, dims=None, start: dict | None = None, max_passes: int = 3,
         verbose: bool = False) -> dict:
    """Coordinate descent over `dims`: measure(config) -> milliseconds per substep (inf for a
    configuration that fails).  Returns {"best": point, "ms_per_step", "trials": [...]}; every
    configuration is measured once."""
    dims = tuple(dims or SOLVER_DIMS[solver])
    best = dict(DEFAULTS)
    best.update(start or {})
    best = {k: best[k] for k in dims}
    seen = {}

    def cost(point):
        key = json.dumps(point, sort_keys=True)
        if key not in seen:
            try:
                ms = float(measure(to_config(point)))
            except Exception:   # a configuration the solver rejects
                ms = math.inf
            seen[key] = ms
            if verbose:
                print(json.dumps({"point": point, "ms_per_step": ms}), flush=True)
        return seen[key]

    best_ms = cost(best)
    for _ in range(max_passes):
        changed = False
        for dim in dims:
            for v in candidates(dim, solver):
                if v == best[dim]:
                    continue
                p = dict(best)
                p[dim] = v
                ms = cost(p)
                if ms < best_ms:
                    best, best_ms, changed = p, ms, True
        if not changed:
            break
    trials = [{"point": json.loads(k), "ms_per_step": v} for k, v in seen.items()]
    return {"best": best, "config": to_config(best), "ms_per_step": best_ms, "trials": trials,
            "when": time.strftime("%Y-%m-%dT%H:%M:%S")}


def library_measure(scene, warmup: int = 3, steps: int = 3, base_extra: dict | None = None):
    """measure(config) for `tune`: the substep's kernel time of `scene` (or a list of scenes of
    one solver type, run as one batched solver) with the per-kernel CUDA-event profiler."""
    from .solver import solver_from_scene, solver_from_scenes

    def measure(cfg: dict) -> float:
        extra = dict(base_extra or {})
        extra.update(cfg)
        if isinstance(scene, (list, tuple)):
            s, _ = solver_from_scenes(list(scene), extra=extra)
        else:
            s = solver_from_scene(scene, extra=extra)
        try:
            if not s.initialize():
                return math.inf
            if warmup and not s.tickNsteps(warmup):
                return math.inf
            prof = s.profile_kernels(steps)
            return sum(v[0] for v in prof.values()) / steps
        finally:
            s.destroy()
    return measure


def adjoint_measure(scene, steps: int = 20, checkpoint_every: int = 10, base_extra: dict | None = None):
    """measure(config) for `tune` over the adjoint's keys: milliseconds per substep of the
    backward of a recorded `steps`-substep rollout of the differentiable PBF `scene` (the
    second of two, so that tapes and the backward's segment graphs exist), loss = mean fluid
    position along (1, 1, 1)."""
    import numpy as np

    from . import diff

    def measure(cfg: dict) -> float:
        extra = dict(base_extra or {})
        extra.update(cfg)
        s = diff.pbf_solver(scene, extra=extra)
        try:
            mask = diff.fluid_mask(scene)
            g = np.zeros((mask.size, 3), np.float32)
            g[mask] = 1.0 / mask.sum()
            best = math.inf
            for _ in range(2):
                diff.diff_forward(s, steps, checkpoint_every)
                t0 = time.perf_counter()
                diff.diff_backward(s, g, None)
                best = min(best, 1e3 * (time.perf_counter() - t0) / steps)
            return best
        finally:
            s.destroy()
    return measure


def workload_key(solver: str, n_fluid: int, name: str | None = None) -> str:
    """Cache key of a workload: a named workload, or the solver type and the fluid-particle
    count rounded to the nearest power of two."""
    if name:
        return name
    return f"{solver}:2^{max(0, round(math.log2(max(n_fluid, 1))))}"


def gpu_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:
        pass
    return "unknown"


def load_cache(path: Path = CACHE) -> dict:
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def store(key: str, result: dict, gpu: str | None = None, path: Path = CACHE) -> dict:
    """Record a tuning result (its "B200" config keys and timing) in the cache file."""
    cache = load_cache(path)
    cache.setdefault(gpu or gpu_name(), {})[key] = {"B200": result["config"], "ms_per_step": result["ms_per_step"],
                                                    "when": result.get("when")}
    Path(path).write_text(json.dumps(cache, indent=1, sort_keys=True) + "\n")
    return cache


def tuned_extra(key: str, gpu: str | None = None, path: Path = CACHE) -> dict:
    """The cached "B200" block for a workload key on this GPU ({} when none is cached).  A
    B200 whose name string is not in the cache takes the entry of another B200 name."""
    cache = load_cache(path)
    g = gpu or gpu_name()
    entry = cache.get(g, {}).get(key)
    if entry is None and "B200" in g:
        for name, table in cache.items():
            if "B200" in name and key in table:
                entry = table[key]
                break
    return dict(entry["B200"]) if entry else {}


def main(argv=None):
    """Tune a workload on this GPU; --write records the result in vtp/tuned.json."""
    import argparse
    from . import scenes

    ap = argparse.ArgumentParser(description="tune a workload on this GPU and record it in vtp/tuned.json")
    ap.add_argument("--workload", default="dfsph_1m",
                    choices=["dfsph_1m", "pbf", "pbf_m1", "immct_500k", "batched_pbf", "batched_dfsph", "diff_pbf"])
    ap.add_argument("--write", action="store_true", help="record the result in the cache")
    ap.add_argument("--no-arithmetic", action="store_true",
                    help="leave out keys that change FP32 arithmetic (rowLanes)")
    a = ap.parse_args(argv)
    base = {}
    if a.workload.startswith("batched"):
        kind = "PBF" if a.workload == "batched_pbf" else "DFSPH"
        sc = [m for m in scenes.batched_scenes() if m.solver == kind]
    else:
        sc = {"dfsph_1m": scenes.dfsph_1m, "pbf": scenes.pbf_dam_break, "pbf_m1": scenes.pbf_dam_break_m1,
              "immct_500k": scenes.immct_500k, "diff_pbf": scenes.diff_pbf}[a.workload]()
        kind = sc.solver
        if a.workload == "dfsph_1m":
            base = {"cfl": 0.4}
    res = tune(library_measure(sc, base_extra=base), kind, dims_for(kind, not a.no_arithmetic), verbose=True)
    if a.workload == "diff_pbf":
        # the adjoint's lanes, on the backward, with the forward's tuned keys fixed
        adj = tune(adjoint_measure(sc, base_extra=res["config"]), kind, ("adjointLanes",), verbose=True)
        res["config"].update(adj["config"])
        res["adjoint_ms_per_step"] = adj["ms_per_step"]
    print(json.dumps({k: res[k] for k in ("best", "config", "ms_per_step")}))
    if a.write:
        store(a.workload, res)


if __name__ == "__main__":
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    from vtp.autotune import main as _main   # the package's module, so its relative imports resolve
    _main()
