"""Launch-configuration autotuner for the neighbour passes.

Sweeps threads per block (= rows per scene-offset tile), the neighbour-loop
unroll (neighbours kept in flight per thread), the lanes per row of the PBF
passes and the tile-grid mode of the pressure-solve passes (one block per
tile, or a persistent grid) on a scene
or a batch of scenes, timing each candidate with the per-kernel CUDA-event
profiler of the library, and returns the fastest configuration for the
substep.  Results are plain dicts so callers can cache them
(``"B200": {"blockSize": b, "unroll": u, "persistentTiles": p, "rowLanes": l}``
in the solver config).
"""
from __future__ import annotations

import itertools
import json
import time

from .solver import solver_from_scene, solver_from_scenes

BLOCKS = (64, 128, 256)
UNROLLS = (1, 2, 4, 8)
PERSISTENT = (False,)
ROW_LANES = (1,)


def tune(scene, warmup: int = 3, steps: int = 3, blocks=BLOCKS, unrolls=UNROLLS, persistent=PERSISTENT,
         lanes=ROW_LANES, verbose: bool = False) -> dict:
    """Return {"best": {...}, "trials": [...]} for one scene, or a list of scenes of one
    solver type (tuned as one batched solver)."""
    trials = []
    for b, u, pt, ln in itertools.product(blocks, unrolls, persistent, lanes):
        extra = {"blockSize": b, "unroll": u, "persistentTiles": bool(pt), "rowLanes": ln}
        if isinstance(scene, (list, tuple)):
            s, _ = solver_from_scenes(list(scene), extra=extra)
        else:
            s = solver_from_scene(scene, extra=extra)
        s.initialize()
        if warmup:
            s.tickNsteps(warmup)
        prof = s.profile_kernels(steps)
        s.destroy()
        total = sum(v[0] for v in prof.values())
        rec = {"blockSize": b, "unroll": u, "persistentTiles": bool(pt), "rowLanes": ln, "ms_per_step": total / steps,
               "kernels": {k: v[0] / max(v[1], 1) for k, v in prof.items()}}
        trials.append(rec)
        if verbose:
            print(json.dumps({k: rec[k] for k in ("blockSize", "unroll", "persistentTiles", "rowLanes",
                                                  "ms_per_step")}),
                  flush=True)
    best = min(trials, key=lambda r: r["ms_per_step"])
    return {"best": {"blockSize": best["blockSize"], "unroll": best["unroll"],
                     "persistentTiles": best["persistentTiles"], "rowLanes": best["rowLanes"]}, "trials": trials,
            "when": time.strftime("%Y-%m-%dT%H:%M:%S")}


if __name__ == "__main__":
    import argparse
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    from vtp import scenes

    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="dfsph_1m", choices=["dfsph_1m", "pbf", "batched_pbf", "batched_dfsph"])
    ap.add_argument("--persistent", action="store_true", help="also try the persistent tile grid")
    ap.add_argument("--lanes", action="store_true", help="also try 4 and 8 lanes per row (PBF passes)")
    a = ap.parse_args()
    if a.scene.startswith("batched"):
        mix = scenes.batched_scenes()
        sc = [m for m in mix if m.solver == ("PBF" if a.scene == "batched_pbf" else "DFSPH")]
    else:
        sc = scenes.dfsph_1m() if a.scene == "dfsph_1m" else scenes.pbf_dam_break()
    res = tune(sc, persistent=(False, True) if a.persistent else PERSISTENT,
               lanes=(1, 4, 8) if a.lanes else ROW_LANES, verbose=True)
    print(json.dumps({"best": res["best"], "trials": [{k: t[k] for k in t if k != "kernels"} for t in res["trials"]]}))
    for t in res["trials"]:
        print(t["blockSize"], t["unroll"], t["persistentTiles"], t["rowLanes"],
              json.dumps({k: round(v, 4) for k, v in sorted(t["kernels"].items())}))
