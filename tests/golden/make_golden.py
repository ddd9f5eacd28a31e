"""Generate golden vectors from the reference's own solvers (oracle/_ref/libvtref.so).

Runs on a machine with a CUDA GPU; each case runs in its own process because
the reference keeps function-local statics that tie a process to one solver
(UGNSCudaImpl.cu:100-102).  Inputs are the seeded scenes of vtp.scenes.

    python tests/golden/make_golden.py --all --out <dir>

Each case writes <dir>/<case>.npz.  Large neighbour lists are stored as a
SHA-256 digest of the reference-layout arrays (counts[n] uint32, then
nbrs[n * maxNbr] uint32), small ones in full.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "vt-physics_b200"))

from vtp import scenes  # noqa: E402


def digest(cnt: np.ndarray, nb: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(cnt, np.uint32).tobytes())
    h.update(np.ascontiguousarray(nb, np.uint32).tobytes())
    return h.hexdigest()


def scene_for(case: str):
    if case.startswith("pbf_small"):
        return scenes.dam_break("PBF", 2000, seed=21)
    if case.startswith("pbf_full"):
        return scenes.pbf_dam_break()
    if case == "dfsph_small_tension":
        sc = scenes.dam_break("DFSPH", 8000, seed=23)
        sc.config["DFSPH"]["Required"]["surfaceTensionCoefficient"] = 0.001
        return sc
    if case.startswith("dfsph_small"):
        return scenes.dam_break("DFSPH", 8000, seed=22)
    if case.startswith("dfsph_1m"):
        return scenes.dfsph_1m()
    if case.startswith("immct_500k"):
        return scenes.immct_500k()
    if case == "immct_small":
        return scenes.layered_mixture("IMMCT", 24, seed=31)
    if case == "imm_small":
        return scenes.layered_mixture("IMM", 24, seed=32)
    if case in ("immct_small_notension", "imm_small_notension"):
        kind = "IMMCT" if case.startswith("immct") else "IMM"
        sc = scenes.layered_mixture(kind, 24, seed=33 if kind == "IMMCT" else 34)
        sc.config[kind]["Required"]["surfaceTensionCoefficient"] = 0.0
        return sc
    raise KeyError(case)


CASES = {
    # name: (ticks to record, store full lists?)
    "pbf_small": ([0, 1, 20], True),
    "pbf_full": ([0, 1], False),
    "dfsph_small": ([0, 1, 2, 3, 10], True),
    "dfsph_small_tension": ([0, 1, 2, 3], False),
    "dfsph_1m_ugns": ([0], False),
    "immct_small": ([0, 1, 2, 5], False),
    "imm_small": ([0, 1, 2, 5], False),
    "immct_small_notension": ([0, 1, 2, 5], False),
    "imm_small_notension": ([0, 1, 2, 5], False),
    # the benchmark scenes themselves: per-particle fields on a fixed seeded
    # subsample of fluid rows (SUBSAMPLE rows, in attach order), lists as digests
    "dfsph_1m_steps": ([0, 1, 3], False),
    "immct_500k_step": ([0, 1], False),
}
# Fluid rows kept per tick for the large cases: (count, seed of the choice).
SUBSAMPLE = {"dfsph_1m_steps": (32768, 2025), "immct_500k_step": (32768, 3025)}


def subsample(case: str, n_fluid: int):
    """Sorted fluid-row indices (attach order among fluid rows) stored for a large case."""
    k, seed = SUBSAMPLE[case]
    return np.sort(np.random.default_rng(seed).choice(n_fluid, size=k, replace=False)).astype(np.int64)


def run_case(case: str, out_dir: Path):
    from oracle.ref import ref as R
    sc = scene_for(case)
    ticks, full = CASES[case]
    s = R.RefSolver(sc)
    s.initialize()
    fm = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
    rec = {"case": case, "n": s.n, "n_fluid": int(fm.sum())}
    arrays = {}
    done = 0
    req = sc.config[sc.solver]["Required"]
    nfo = sum(1 for o in sc.objects if o.material == 0)
    iters = []
    sub = subsample(case, int(fm.sum())) if case in SUBSAMPLE else None
    if sub is not None:
        arrays["sub_idx"] = sub.astype(np.int32)

    def fl(a):
        """Fluid rows of a per-particle field (the stored subsample for the large cases)."""
        a = a[fm]
        return a if sub is None else a[sub]
    s.take_means()
    for t in ticks:
        while done < t:
            ok = s.tick(1)
            done += 1
            if sc.solver != "PBF":
                means = s.take_means()
                d, i, _ = R.split_iterations(means, nfo, req["divFreeThreshold"], req["incompThreshold"])
                iters.append((d, i))
                arrays[f"means_{done}"] = means
            if not ok:
                rec["crashed_at"] = done
        cnt, nb = s.neighbors()
        rec[f"nbr_digest_{t}"] = digest(cnt, nb)
        arrays[f"nbr_count_hist_{t}"] = np.bincount(cnt, minlength=s.maxnbr + 1).astype(np.int64)
        if full and t == 0:
            valid = nb != 0xFFFFFFFF
            arrays[f"nbr_count_{t}"] = cnt.astype(np.uint16)
            arrays[f"nbr_flat_{t}"] = nb[valid].astype(np.uint32)
            arrays[f"sorted_ids_{t}"] = s.get("particleIndices", 1, np.uint32)
            arrays[f"cell_ids_{t}"] = s.get("cellIndices", 1, np.uint32)
        big = case == "dfsph_1m_ugns"
        if t > 0 and not big:
            arrays[f"pos_{t}"] = fl(s.get("pos", 3))
            arrays[f"vel_{t}"] = fl(s.get("vel", 3))
        if t == 0:
            vol = s.get("volume")
            if sub is not None:
                vb = vol[~fm].astype(np.float64)
                arrays["volume_0_boundary_stats"] = np.array([vb.sum(), vb.min(), vb.max()])
                arrays["volume_0_fluid"] = fl(vol)
            elif big:
                vb = vol[~fm].astype(np.float64)
                arrays["volume_0_boundary_stats"] = np.array([vb.sum(), vb.min(), vb.max()])
            else:
                arrays["volume_0"] = vol
                if sc.solver == "PBF":
                    arrays["mass_0"] = s.get("mass")
        if sc.solver == "PBF" and t > 0:
            arrays[f"density_{t}"] = fl(s.get("density_sph"))
        if sc.solver != "PBF" and t > 0 and case != "dfsph_1m_ugns":
            arrays[f"ratio_{t}"] = fl(s.get("compression_ratio"))
        if sc.solver in ("IMM", "IMMCT") and t > 0:
            P = len(req["phaseRestDensity"])
            arrays[f"frac_{t}"] = fl(s.get("vol_frac", P))
            if sc.solver == "IMMCT":
                arrays[f"Q_{t}"] = fl(s.get("Q", 9))
                arrays[f"cd_{t}"] = fl(s.get("Cd"))
        if sub is not None and t > 0:
            # whole-scene statistics in FP64: kinetic energy (sum |v|^2) and per-phase volume
            v = s.get("vel", 3)[fm].astype(np.float64)
            arrays[f"sum_v2_{t}"] = np.array([np.sum(v * v)])
            if sc.solver in ("IMM", "IMMCT"):
                arrays[f"phase_sum_{t}"] = s.get("vol_frac", P)[fm].astype(np.float64).sum(0)
    if iters:
        arrays["iters"] = np.array(iters, np.int32)
    rec["ticks"] = ticks
    np.savez_compressed(out_dir / f"{case}.npz", meta=json.dumps(rec), **arrays)
    print(json.dumps({k: v for k, v in rec.items() if not k.startswith("nbr_digest")}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case")
    ap.add_argument("--all", action="store_true")
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    if a.case:
        run_case(a.case, out)
        return
    rc = 0
    for case in CASES:
        r = subprocess.run([sys.executable, __file__, "--case", case, "--out", str(out)])
        print(f"{case}: exit {r.returncode}", flush=True)
        rc |= r.returncode
    sys.exit(rc)


if __name__ == "__main__":
    main()
