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
}


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
            arrays[f"pos_{t}"] = s.get("pos", 3)[fm]
            arrays[f"vel_{t}"] = s.get("vel", 3)[fm]
        if t == 0:
            vol = s.get("volume")
            if big:
                vb = vol[~fm].astype(np.float64)
                arrays["volume_0_boundary_stats"] = np.array([vb.sum(), vb.min(), vb.max()])
            else:
                arrays["volume_0"] = vol
                if sc.solver == "PBF":
                    arrays["mass_0"] = s.get("mass")
        if sc.solver == "PBF" and t > 0:
            arrays[f"density_{t}"] = s.get("density_sph")[fm]
        if sc.solver != "PBF" and t > 0 and case != "dfsph_1m_ugns":
            arrays[f"ratio_{t}"] = s.get("compression_ratio")[fm]
        if sc.solver in ("IMM", "IMMCT") and t > 0:
            P = len(req["phaseRestDensity"])
            arrays[f"frac_{t}"] = s.get("vol_frac", P)[fm]
            if sc.solver == "IMMCT":
                arrays[f"Q_{t}"] = s.get("Q", 9)[fm]
                arrays[f"cd_{t}"] = s.get("Cd")[fm]
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
