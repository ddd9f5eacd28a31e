#!/usr/bin/env python
"""Benchmark of the particle-fluid hot path: one step = one solver substep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dfsph_1m|pbf|pbf_m1|immct_500k|batched|batched_m1|diff_pbf|diff_dfsph|dfsph_1m_dd]

Default workload: DFSPH, 1,000,000 fluid particles (100^3 lattice, spacing 0.01,
jitter +-0.05 spacing, seed 2002) in a 3-layer 2 x 1.5 x 1.06 box of 453,957
boundary particles, dt = 1 ms (CFL 0.4 rule capped there), thresholds 0.1 %,
seeded synthetic input.  Metric: million fluid-particle substeps per second
(whole job, all ranks).  diff_pbf / diff_dfsph time a recorded forward plus
its adjoint over a rollout (64k fluid particles each).

With --gpus N (or under torchrun) one process per GPU: a single scene runs as
replicas (the path has no exchange step), the batched mix is sharded over the
ranks by longest-processing-time assignment, dfsph_1m_dd runs one slab per
rank; timing is the max over ranks.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "vt-physics_b200"))

METRIC = "M particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed substeps (default: 200; 1000 for pbf; 30 for immct_500k, whose scene develops "
                         "outlier speeds after ~45 substeps in the reference and here alike)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["dfsph_1m", "pbf", "pbf_m1", "immct_500k", "batched", "batched_m1",
                                           "diff_pbf", "diff_dfsph", "dfsph_1m_dd"],
                    default="dfsph_1m")
    ap.add_argument("--domains", type=int, default=1,
                    help="dfsph_1m_dd on one process: slabs run as threads on this GPU (under torchrun: one "
                         "slab per rank)")
    ap.add_argument("--checkpoint-every", type=int, default=20)
    ap.add_argument("--fd-steps", type=int, default=20,
                    help="diff_pbf / diff_dfsph: horizon of the finite-difference check")
    ap.add_argument("--fd-directions", type=int, default=4)
    ap.add_argument("--no-loop-baseline", action="store_true",
                    help="batched workload: skip the plain per-scene loop it is compared with")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="substeps of the end-to-end run (0: the same substeps as the timed run)")
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--extra", default="", help='extra "B200" config keys as JSON, e.g. {"unroll": 2}')
    ap.add_argument("--scene-index", type=int, default=-1, help=argparse.SUPPRESS)
    return ap.parse_args()


def make_scene(workload):
    from vtp import scenes
    return {"dfsph_1m": scenes.dfsph_1m, "pbf": scenes.pbf_dam_break, "pbf_m1": scenes.pbf_dam_break_m1,
            "immct_500k": scenes.immct_500k}[workload]()


def batched_mix(workload):
    """The batched mix of a workload: "batched" (PBF scenes at spacing 0.02, whose fluid the
    reference's PBF formulation lets through the floor) or "batched_m1" (PBF particles of
    mass 1, fluid kept in the box)."""
    from vtp import scenes
    return scenes.batched_scenes(pbf_spacing=0.1 if workload == "batched_m1" else None)


class Clocks:
    """nvidia-smi sampler running while the timed region runs (200 ms period)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def fp32_peak_tflops(sm_mhz):
    """FP32 SIMT peak: SMs x 128 lanes x 2 flops (FMA) x SM clock."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return sms * 128 * 2 * float(sm_mhz) * 1e6 / 1e12


def ncu_traffic(workload: str, kernel: str):
    """DRAM bytes per launch measured by ncu for this kernel and workload (profiles/ncu_traffic.json)."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    try:
        return json.loads(p.read_text()).get(workload, {}).get(kernel)
    except (OSError, ValueError):
        return None


def ncu_counter(group: str, workload: str, kernel: str):
    """A per-launch ncu counter of this kernel and workload recorded in profiles/ncu_traffic.json
    under `group` ("warp_instructions", "l1_wavefronts"), if any."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    try:
        return json.loads(p.read_text()).get(group, {}).get(workload, {}).get(kernel)
    except (OSError, ValueError):
        return None


def roofline_of(name, b, flops, per_launch_ms, peak, peak_kind, clocks, workload) -> dict:
    """Roofline of one kernel against the HBM ceiling (no pass is a contraction, so the tensor
    ceiling does not apply): algorithmic state bytes per launch (each state array once, the work
    model of vtp/bytes_model.py) over the CUDA-event launch time, against the measured HBM copy
    bandwidth.  Kept beside it: the list-inclusive bytes, and algorithmic FP32 flops against the
    SIMT peak at the sampled clock (`fp32.ideal_over_hbm` > 1 means the flops, not the bytes, set
    the ideal time)."""
    t = per_launch_ms / 1e3
    hbm = b["state"] / t / 1e9
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    fpk = fp32_peak_tflops(mhz)
    tf = flops / t / 1e12
    t_bytes = b["state"] / (peak * 1e9)
    t_flops = flops / (fpk * 1e12) if fpk else 0.0
    out = {"kernel": name, "ms_per_launch": per_launch_ms,
           "hbm": {"achieved": hbm, "peak": peak, "unit": "GB/s", "frac": hbm / peak, "peak_kind": peak_kind,
                   "bytes_per_launch": b["state"], "bytes_per_launch_with_lists": b["total"],
                   "frac_with_lists": b["total"] / t / 1e9 / peak},
           "fp32": {"achieved": tf, "peak": fpk, "unit": "TFLOP/s", "frac": tf / fpk if fpk else None,
                    "peak_kind": f"computed: SMs x 128 x 2 x {mhz:.0f} MHz", "flops_per_launch": flops}}
    out["fp32"]["ideal_over_hbm"] = t_flops / t_bytes if t_bytes else None
    out.update({"bound": "hbm", "achieved": hbm, "peak": peak, "unit": "GB/s", "frac": hbm / peak})
    out["traffic"] = ncu_traffic(workload, name)
    inst = ncu_counter("warp_instructions", workload, name)
    if inst:
        # An issue-bound kernel (the list builder): its warp instructions from one ncu capture
        # over the live launch time, against 4 issue slots per SM per cycle at the sampled clock.
        sms = 148
        rate = inst / t / 1e9
        cap = 4 * sms * mhz / 1e3
        out["issue"] = {"achieved": rate, "peak": cap, "unit": "G warp-instructions/s", "frac": rate / cap,
                        "instructions_per_launch": inst, "peak_kind": f"computed: 4 x {sms} SMs x {mhz:.0f} MHz",
                        "instructions_from": "profiles/ncu_traffic.json"}
    wf = ncu_counter("l1_wavefronts", workload, name)
    if wf:
        # A gather-bound kernel (the pressure solve): its L1 data-pipe wavefronts (global, local
        # and shared) from one ncu capture over the live launch time, against one wavefront per
        # SM per cycle at the sampled clock.
        sms = 148
        rate = wf / t / 1e9
        cap = sms * mhz / 1e3
        out["l1tex"] = {"achieved": rate, "peak": cap, "unit": "G wavefronts/s", "frac": rate / cap,
                        "wavefronts_per_launch": wf, "peak_kind": f"computed: 1 x {sms} SMs x {mhz:.0f} MHz",
                        "wavefronts_from": "profiles/ncu_traffic.json"}
    return out


def cpu_baseline(scene, seconds: float) -> dict:
    """FP64 OpenMP oracle on the host cores: bounded sample of the same scene."""
    from oracle import oracle as O
    O.lib()
    cores = O.num_threads()
    t0 = time.perf_counter()
    o = O.OracleSolver(scene) if scene.solver in ("PBF", "DFSPH") else O.ImmOracle(scene)
    init_s = time.perf_counter() - t0
    steps = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 1000:
            break
    nf = scene.n_fluid
    return {"value": nf * steps / el / 1e6, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"FP64 OpenMP oracle, first {steps} substeps of the same scene after a {init_s:.1f} s "
                      f"initialization, {el:.1f} s of CPU time"}


def run_reference_batched(args) -> dict:
    """Reference side of the batched mix: each scene in its own process running the reference's
    plain solver (its solvers keep function-local statics, so one solver per process), scenes one
    after another; a time-bounded sample of the 64 scenes, interleaving PBF and DFSPH scenes."""
    from vtp import scenes
    mix = batched_mix(args.workload)
    order = [k for pair in zip(range(48), range(48, 64)) for k in pair] + list(range(16, 48))
    order = list(dict.fromkeys(order))
    steps = max(1, min(args.steps, 50))
    warm = min(args.warmup, 3)
    budget = 150.0
    t_start = time.perf_counter()
    tot_ms, tot_ps, done, e2e = 0.0, 0.0, [], []
    for k in order:
        if time.perf_counter() - t_start > budget:
            break
        cmd = [sys.executable, str(Path(__file__).resolve()), "--impl", "reference", "--workload", args.workload,
               "--scene-index", str(k), "--steps", str(steps), "--warmup", str(warm), "--e2e-steps", "3"]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            continue
        d = json.loads(r.stdout.strip().splitlines()[-1])
        if "ms" not in d:
            continue
        tot_ms += d["ms"]
        tot_ps += mix[k].n_fluid * steps
        e2e.append((mix[k].n_fluid * 3, d["e2e_s"]))
        done.append(k)
    out = {"impl": "reference", "metric": METRIC, "unit": METRIC, "higher_is_better": True}
    if not done:
        out["unavailable"] = "no scene of the batched mix ran in the reference build"
        return out
    value = tot_ps / (tot_ms / 1e3) / 1e6
    out.update({"value": value, "n_gpus": 1, "steps": steps, "warmup": warm, "ms_per_step": tot_ms / steps,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload, "scenes_sampled": done, "scenes": len(mix),
                           "impl": "reference CUDA build (sm_100a, -O3), one process per scene, "
                                   "Solver::tickNsteps per scene one after another"},
                "cpu_baseline": {"value": value, "unit": METRIC, "cores": 0, "kind": "reference",
                                 "sample": f"the reference is GPU code: its own CUDA build on this B200, "
                                           f"{len(done)} of {len(mix)} scenes x {steps} substeps"},
                "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    out["config"]["state_round_trip_value"] = sum(a for a, _ in e2e) / sum(b for _, b in e2e) / 1e6
    return out


def run_reference_scene(args) -> dict:
    """One scene of the batched mix in the reference build (child process of run_reference_batched)."""
    from oracle.ref import ref as R
    from vtp import scenes
    sc = batched_mix(args.workload)[args.scene_index]
    s = R.RefSolver(sc)
    s.initialize()
    if args.warmup:
        s.tick_timed(args.warmup)
    ms = s.tick_timed(args.steps)
    pos, vel = s.get("pos", 3), s.get("vel", 3)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        s.set("pos", pos)
        s.set("vel", vel)
        s.tick(1)
        pos, vel = s.get("pos", 3), s.get("vel", 3)
    return {"ms": ms, "e2e_s": time.perf_counter() - t0}


def run_reference(args) -> dict:
    """The reference's own CUDA build (oracle/_ref/libvtref.so) on this GPU, through its Solver API."""
    import numpy as np
    from oracle.ref import ref as R
    out = {"impl": "reference", "metric": METRIC, "unit": METRIC, "higher_is_better": True}
    if not R.available():
        out["unavailable"] = "oracle/_ref/libvtref.so was not built (the reference sources were not present)"
        return out
    if args.workload in ("batched", "batched_m1"):
        return run_reference_scene(args) if args.scene_index >= 0 else run_reference_batched(args)
    sc = make_scene(args.workload)
    s = R.RefSolver(sc)
    s.initialize()
    if args.warmup:
        s.tick_timed(args.warmup)
    s.take_means()   # residuals recorded so far (initialization, warm-up) are dropped
    clk = Clocks(0)
    clk.start()
    ms = s.tick_timed(args.steps)
    clocks = clk.stop()
    iters = None
    if sc.solver != "PBF":
        # the reference's pressure-solve iterations over the timed substeps, rebuilt from the
        # residuals its cal_mean returned (one per fluid object per iteration)
        req = sc.config[sc.solver]["Required"]
        nfo = sum(1 for o in sc.objects if o.material == 0)
        per_tick = R.split_ticks(s.take_means(), nfo, req["divFreeThreshold"], req["incompThreshold"])
        iters = {"div_iters_total": int(sum(d for d, _ in per_tick)),
                 "incomp_iters_total": int(sum(i for _, i in per_tick)), "substeps_parsed": len(per_tick)}
    nf = sc.n_fluid
    value = nf * args.steps / (ms / 1e3) / 1e6
    # e2e: the fluid state round-trips through host memory every step (positions and
    # velocities of the fluid particles, which the scenes attach first, in; one tick; out),
    # the same bytes as the library's e2e.
    nfl = sum(c for _, c in fluid_ranges(sc))
    assert fluid_ranges(sc) == [(0, nfl)]
    pos = s.get_prefix("pos", nfl)
    vel = s.get_prefix("vel", nfl)
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else min(args.steps, 20)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.set("pos", pos)
        s.set("vel", vel)
        s.tick(1)
        pos = s.get_prefix("pos", nfl)
        vel = s.get_prefix("vel", nfl)
    el = time.perf_counter() - t0
    out.update({"value": value, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": args.workload, "fluid": nf, "boundary": sc.n_boundary,
                                                "impl": "reference CUDA build (sm_100a, -O3) via Solver::tickNsteps",
                                                **(iters or {})},
                "clocks": clocks,
                "cpu_baseline": {"value": value, "unit": METRIC, "cores": 0, "kind": "reference",
                                 "sample": "the reference is GPU code: its own CUDA build timed on this B200"},
                "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    # For information: the same fluid-state round trip per step as the library's e2e.
    out["config"]["state_round_trip"] = {"value": nf * e2e_steps / el / 1e6, "unit": METRIC,
                                         "h2d_bytes_per_step": int(2 * 12 * nfl),
                                         "d2h_bytes_per_step": int(2 * 12 * nfl)}
    return out


def fluid_ranges(scene):
    """(first, count) attach-order ranges of the scene's fluid objects."""
    out, start = [], 0
    for o in scene.objects:
        if o.material == 0 and o.n:
            if out and out[-1][0] + out[-1][1] == start:
                out[-1] = (out[-1][0], out[-1][1] + o.n)
            else:
                out.append((start, o.n))
        start += o.n
    return out


def state_buffers(s, ranges, torch):
    """Page-locked host buffers (vtp_host_alloc) holding the fluid state (pos, vel) of each range."""
    import vtp
    bufs = []
    for first, count in ranges:
        p, v = vtp.HostBuffer((count, 3)), vtp.HostBuffer((count, 3))
        s.get_state_range_ptr(first, count, p.ptr, v.ptr)
        bufs.append((first, count, p, v))
    return bufs


def state_bytes(bufs) -> int:
    return int(sum(p.nbytes + v.nbytes for _, _, p, v in bufs))


def frame_buffers(s, ranges):
    """Page-locked host buffers holding the state (pos, vel) of several attach-order ranges back
    to back, filled with the current state."""
    import vtp
    total = sum(c for _, c in ranges)
    p, v = vtp.HostBuffer((total, 3)), vtp.HostBuffer((total, 3))
    off = 0
    for first, count in ranges:
        s.get_state_range_ptr(first, count, p.ptr + 12 * off, v.ptr + 12 * off)
        off += count
    return ranges, p, v


def frame_round_trip(s, fb):
    """One e2e step of several ranges: one vtp_solver_step_state_ranges call (upload, one
    substep, read back, one synchronisation)."""
    ranges, p, v = fb
    assert s.step_state_ranges_ptr(ranges, p.ptr, v.ptr, 1, p.ptr, v.ptr), s.last_error


def state_round_trip(s, bufs):
    """One e2e step: fluid state host -> device, one substep, fluid state device -> host (one
    library call, vtp_solver_step_state_range, when the fluid is one attach-order range)."""
    if len(bufs) == 1:
        first, count, p, v = bufs[0]
        assert s.step_state_range_ptr(first, count, p.ptr, v.ptr, 1, p.ptr, v.ptr), s.last_error
        return
    for first, count, p, v in bufs:
        s.set_state_range_ptr(first, count, p.ptr, v.ptr)
    assert s.tickNsteps(1), s.last_error
    for first, count, p, v in bufs:
        s.get_state_range_ptr(first, count, p.ptr, v.ptr)


def run_batched(args, rank, world, local, dist, torch):
    """64 independent scenes (48 PBF + 16 DFSPH): one solver per solver type advances all its
    scenes together (scene-offset kernels, one CUDA graph per substep).  Compared with the plain
    per-scene loop (one solver per scene, scenes one after another) on the same GPU."""
    import numpy as np
    import vtp
    from vtp.dist import scene_share
    mix = batched_mix(args.workload)
    mine = scene_share(mix, world, rank)
    # per solver type: --extra, or the autotuned block of that half of the mix
    extras = {}
    for kind in ("PBF", "DFSPH"):
        e = json.loads(args.extra) if args.extra else default_extra(f"batched_{kind.lower()}")
        if args.block:
            e["blockSize"] = args.block
        extras[kind] = e or None
    groups = {}
    for k in mine:
        groups.setdefault(mix[k].solver, []).append(k)
    batches = []
    for kind in ("PBF", "DFSPH"):
        if kind not in groups:
            continue
        idx = groups[kind]
        b, ranges = vtp.solver_from_scenes([mix[k] for k in idx], extras[kind])
        assert b.initialize(), b.last_error
        batches.append((kind, idx, b, ranges))
    for _, _, b, _ in batches:
        if args.warmup:
            assert b.tickNsteps(args.warmup), b.last_error
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = Clocks(local if world > 1 else 0)
    clk.start()
    # The batches advance concurrently, each on its own stream (vtp.solver.tick_together);
    # the device time is the span between two events recorded on an idle GPU before the first
    # substep is submitted and after the last one has finished.
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    ev0.synchronize()
    t0 = time.perf_counter()
    from vtp.solver import tick_together
    assert tick_together([b for _, _, b, _ in batches], args.steps), [b.last_error for _, _, b, _ in batches]
    wall = time.perf_counter() - t0
    torch.cuda.synchronize()
    ev1.record()
    ev1.synchronize()
    dev_ms = ev0.elapsed_time(ev1)
    launches = sum(b.launch_count() for _, _, b, _ in batches)
    batch_ms = {kind: b.stage_times()[2] for kind, _, b, _ in batches}
    clocks = clk.stop()
    t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    nf_all = sum(m.n_fluid for m in mix)
    value = nf_all * args.steps / (max_ms / 1e3) / 1e6
    final = {}
    for kind, idx, b, ranges in batches:
        pos = b.get_field("pos")
        for k, (lo, hi) in zip(idx, ranges):
            final[k] = pos[lo:hi].copy()

    # Roofline of the dominant kernel (per-launch CUDA events), with the work model of the
    # batch that launches it.
    prof = {}
    cands = []
    for kind, idx, b, _ in batches:
        for name, (ms, n) in b.profile_kernels(args.profile_steps).items():
            pm, pn = prof.get(name, (0.0, 0))
            prof[name] = (pm + ms, pn + n)
            cands.append((ms, n, name, kind, idx, b))
    kernels = {k: {"ms_total": round(v[0], 4), "launches": v[1],
                   "share": round(v[0] / sum(x[0] for x in prof.values()), 4)}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    d_ms, d_n, dom_name, d_kind, d_idx, d_b = max(cands, key=lambda c: c[0])
    roofline = batch_roofline(d_b, d_kind, [mix[k] for k in d_idx], dom_name, d_ms / max(d_n, 1), clocks)

    # e2e through the public API: every step each batch's fluid state (positions and velocities
    # of the fluid objects of all its scenes; boundary particles are static scene data) goes
    # host -> device, one substep runs, and the new state comes back: one
    # vtp_solver_step_state_ranges call per batch and step.
    def fluid_of(idx, ranges):
        out = []
        for k, (lo, _) in zip(idx, ranges):
            out += [(lo + f, c) for f, c in fluid_ranges(mix[k])]
        return out

    hbuf = [frame_buffers(b, fluid_of(idx, ranges)) for _, idx, b, ranges in batches]
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else min(args.steps, 20)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()

    failures = []

    def e2e_run(k):
        b, fb = batches[k][2], hbuf[k]
        try:
            for _ in range(e2e_steps):
                frame_round_trip(b, fb)
        except BaseException as e:
            failures.append(e)

    threads = [threading.Thread(target=e2e_run, args=(k,)) for k in range(len(batches))]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if failures:
        raise failures[0]
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_val = nf_all * e2e_steps / float(te.item()) / 1e6
    io_bytes = int(sum(p.nbytes + v.nbytes for _, p, v in hbuf))
    for _, _, b, _ in batches:
        b.destroy()

    cfg = {"workload": args.workload, "scenes": len(mix), "pbf_scenes": sum(m.solver == "PBF" for m in mix),
           "fluid": nf_all, "boundary": sum(m.n_boundary for m in mix), "scenes_this_rank": len(mine),
           "parallelism": f"scenes-lpt{world}", "wall_ms_per_step": 1e3 * wall / args.steps, "b200": extras,
           "batches": "PBF and DFSPH batches on their own streams, advanced concurrently",
           "batch_ms_per_step": {k: v / args.steps for k, v in batch_ms.items()},
           "l2": "inputs larger than L2 (~9.2M particles of state and neighbour lists)"}
    if world == 1 and not args.no_loop_baseline:
        # The plain per-scene loop: one solver per scene, scenes one after another.
        loop_ms = 0.0
        same = True
        for k, m in enumerate(mix):
            s = vtp.solver_from_scene(m, extras[m.solver])
            assert s.initialize(), s.last_error
            if args.warmup:
                assert s.tickNsteps(args.warmup), s.last_error
            assert s.tickNsteps(args.steps), s.last_error
            loop_ms += s.stage_times()[2]
            same = same and np.array_equal(s.get_field("pos"), final[k])
            s.destroy()
        cfg["per_scene_loop_value"] = nf_all * args.steps / (loop_ms / 1e3) / 1e6
        cfg["per_scene_loop_ms_per_step"] = loop_ms / args.steps
        cfg["speedup_vs_per_scene_loop"] = cfg["per_scene_loop_value"] and value / cfg["per_scene_loop_value"]
        cfg["identical_per_scene"] = bool(same)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg, "clocks": clocks,
        "gpu_launches": int(launches),
        "roofline": roofline,
        "kernels": kernels,
        "e2e": {"value": e2e_val, "unit": METRIC, "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
    }
    return line


def grid_buckets(req, extra=None) -> int:
    """Cell buckets of one scene's grid as the library allocates them (cells 0..g per axis,
    the reference's inclusive upper bound): 64-cell bricks, or the reference's linear key range
    for "cellOrder": "linear" and grids under 4 cells wide in x or y; plus the outside bucket."""
    import numpy as np
    h = float(np.float32(np.float32(req["particleRadius"]) * np.float32(4)))
    gx, gy, gz = [int(np.ceil(np.float32(np.float32(v) / np.float32(h)))) for v in req["simSpaceSize"]]
    linear = (extra or {}).get("cellOrder", "brick") == "linear" or gx < 4 or gy < 4
    if linear:
        return gz * gy * gx + gy * gx + gx + 1 + 1
    return 64 * ((gx + 4) // 4) * ((gy + 4) // 4) * ((gz + 4) // 4) + 1


def batch_roofline(b, kind, batch_scenes, name, per_launch_ms, clocks) -> dict:
    """Roofline of kernel `name` of one batched solver: the work model of the whole batch
    (all its scenes' rows, buckets and measured mean neighbour count)."""
    import numpy as np
    from vtp.bytes_model import kernel_bytes, kernel_flops
    c = b.counts()
    req = batch_scenes[0].config[kind]["Required"]
    fluid = np.asarray(b.get_field("mat")).reshape(-1) == 0
    cnt, _ = b.get_neighbors(int(req["maxNeighborNum"]))
    k_mean = float(np.mean(np.maximum(cnt[fluid].astype(np.float64) - 1.0, 0.0))) if fluid.any() else 0.0
    K = sum(grid_buckets(m.config[kind]["Required"]) for m in batch_scenes)  # default cell order
    bts = kernel_bytes(kind, name, c["total"], c["fluid"], K, k_mean)
    peak, peak_kind = peaks()
    out = roofline_of(name, bts, kernel_flops(name, c["fluid"], k_mean), per_launch_ms, peak, peak_kind, clocks,
                      "batched")
    out["batch"] = {"solver": kind, "scenes": len(batch_scenes), "rows": c["total"], "fluid": c["fluid"],
                    "mean_neighbors": round(k_mean, 2)}
    return out


def run_diff(args, torch) -> dict:
    """Differentiable PBF, 64k fluid particles: forward with checkpoints every k substeps, then the
    adjoint (per-segment recompute + hand-written adjoint passes).  value = adjoint throughput;
    config carries the forward throughput and the adjoint / forward cost ratio, and an FD check of
    the adjoint (FP64 CPU oracle, lists frozen to the GPU's) over a shorter horizon."""
    import numpy as np
    import vtp
    from vtp import diff
    sc = vtp.scenes.diff_pbf()
    mask = diff.fluid_mask(sc)
    nf = int(mask.sum())
    target = np.array([0.8, 0.2, 0.6])
    extra = json.loads(args.extra) if args.extra else (default_extra("diff_pbf") or None)

    def loss_grad(pos):
        m = pos[mask].astype(np.float64).mean(0)
        g = np.zeros(pos.shape, np.float32)
        g[mask] = 2.0 * (m - target) / nf
        return float(((m - target) ** 2).sum()), g

    s = diff.pbf_solver(sc, extra=extra)   # initialized
    x_init, v_init = s.get_field("pos"), s.get_field("vel")
    if args.warmup:
        # One recorded rollout of the timed shape and its adjoint on this solver: it allocates the
        # checkpoints and the tape, which later rollouts of the same shape reuse, and captures the
        # backward's segment graph; then the initial state is written back, as a training loop
        # restarts every rollout from its initial state.
        diff.diff_forward(s, args.steps, args.checkpoint_every)
        _, g = loss_grad(s.get_field("pos"))
        diff.diff_backward(s, g, None)
        s.set_field("pos", x_init)
        s.set_field("vel", v_init)
    # plain forward of the same rollout (no checkpoints): the cost the adjoint is compared with;
    # one substep first captures its substep graphs outside the timed region, then the
    # rollout's initial state is written back
    p = diff.pbf_solver(sc, extra=extra)
    p.tickNsteps(1)
    p.set_field("pos", x_init)
    p.set_field("vel", v_init)
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.start()
    tp = time.perf_counter()
    assert p.tickNsteps(args.steps), p.last_error
    plain_s = time.perf_counter() - tp
    p.destroy()
    t0 = time.perf_counter()
    diff.diff_forward(s, args.steps, args.checkpoint_every)
    t1 = time.perf_counter()
    loss, g = loss_grad(s.get_field("pos"))
    t2 = time.perf_counter()
    gx, gv, gk = diff.diff_backward(s, g, None)
    t3 = time.perf_counter()
    clocks = clk.stop()
    fwd_s, bwd_s = t1 - t0, t3 - t2
    s.destroy()
    # value: gradients per second in particle-steps, i.e. the recorded forward plus the backward
    value = nf * args.steps / (fwd_s + bwd_s) / 1e6
    cfg = {"workload": "diff_pbf", "fluid": nf, "boundary": int((~mask).sum()), "substeps": args.steps, "b200": extra,
           "checkpoint_every": args.checkpoint_every, "loss": loss, "dl_dxsph_k": gk,
           "forward_value": nf * args.steps / plain_s / 1e6, "recorded_forward_value": nf * args.steps / fwd_s / 1e6,
           "adjoint_over_forward": (fwd_s + bwd_s) / plain_s,
           "adjoint_over_forward_definition": "(recorded forward + backward) / plain forward, wall clock",
           "recorded_forward_over_forward": fwd_s / plain_s, "backward_over_forward": bwd_s / plain_s,
           "grad_v0_norm": float(np.linalg.norm(gv[mask])),
           "timing": "host wall clock around each synchronous C-ABI call (inputs resident on the device)",
           "l2": "per-segment tapes (~0.5 GB) larger than L2"}
    # FD check of the adjoint over a shorter horizon, FP64 CPU oracle with the GPU's frozen lists.
    if args.fd_steps > 0 and args.fd_directions > 0:
        from oracle import oracle as O
        T = min(args.fd_steps, args.steps)
        s = diff.pbf_solver(sc, extra=extra)
        maxnbr = int(sc.config["PBF"]["Required"]["maxNeighborNum"])
        diff.diff_forward(s, T, args.checkpoint_every, keep_lists=True)
        lists = [diff.diff_lists(s, t, maxnbr) for t in range(T)]
        _, g = loss_grad(s.get_field("pos"))
        _, gv, gk = diff.diff_backward(s, g, None)
        s.destroy()
        d = O.PbfDiff(sc)
        x0, v0 = d.base.pos.copy(), d.base.vel.copy()
        rng = np.random.default_rng(5006)
        k0 = d.p.xsph_k
        errs = []
        for _ in range(args.fd_directions):
            dv = np.zeros_like(v0)
            dv[mask] = rng.normal(size=(nf, 3))
            dk = rng.normal()
            nrm = np.sqrt((dv ** 2).sum() + dk * dk)
            dv, dk = dv / nrm, dk / nrm

            def L(e):
                d.p.xsph_k = k0 + e * dk
                x, _, _, _ = d.rollout(x0, v0 + e * dv, T, lists=lists)
                d.p.xsph_k = k0
                m = x[mask].mean(0)
                return float(((m - target) ** 2).sum())
            fd = (L(1e-4) - L(-1e-4)) / 2e-4
            ad = float((gv.astype(np.float64) * dv).sum() + gk * dk)
            errs.append(abs(ad - fd) / abs(fd))
        cfg["fd_check"] = {"substeps": T, "directions": args.fd_directions, "eps": 1e-4,
                           "max_rel_err": max(errs), "rel_errs": errs, "reference": "FP64 CPU oracle, frozen lists"}
    return {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * (fwd_s + bwd_s) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "clocks": clocks}


def run_diff_dfsph(args, torch) -> dict:
    """Differentiable DFSPH, 64k fluid particles: forward with checkpoints every k substeps
    (the last segments recorded into resident tapes), then the adjoint of the whole substep
    (per-segment recompute where no tape holds the segment, hand-written adjoint passes).
    value = (recorded forward + backward) throughput; config carries the plain forward's, the
    cost ratio, the GPU adjoint against the FP64 adjoint of the same discrete map, and FP64
    central differences (FP64 CPU oracle, the GPU's lists and iteration counts frozen) over a
    shorter horizon."""
    import numpy as np
    import vtp
    from vtp import diff
    sc = vtp.scenes.diff_dfsph()
    mask = diff.fluid_mask(sc)
    nf = int(mask.sum())
    target = np.array([0.4, 0.1, 0.3])
    extra = json.loads(args.extra) if args.extra else (default_extra("diff_dfsph") or None)

    def loss_grad(pos):
        m = pos[mask].astype(np.float64).mean(0)
        g = np.zeros(pos.shape, np.float32)
        g[mask] = 2.0 * (m - target) / nf
        return float(((m - target) ** 2).sum()), g

    def solver():
        s = vtp.solver_from_scene(sc, extra=extra)
        assert s.initialize(), s.last_error
        return s

    every = min(args.checkpoint_every, 10)
    s = solver()
    x_init, v_init = s.get_field("pos"), s.get_field("vel")
    if args.warmup:
        # one rollout of the timed shape allocates checkpoints, tapes and iteration records,
        # which later rollouts of the same shape reuse; the initial state is written back
        diff.diff_forward(s, args.steps, every)
        _, g = loss_grad(s.get_field("pos"))
        diff.diff_backward(s, g, None)
        s.set_field("pos", x_init)
        s.set_field("vel", v_init)
    # plain forward of the same rollout: its substep graphs captured by one substep outside the
    # timed region, then the rollout's initial state written back
    p = solver()
    p.tickNsteps(1)
    p.set_field("pos", x_init)
    p.set_field("vel", v_init)
    it0 = p.stats()
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.start()
    tp = time.perf_counter()
    assert p.tickNsteps(args.steps), p.last_error
    plain_s = time.perf_counter() - tp
    it1 = p.stats()
    plain_iters = {k: it1[k] - it0[k] for k in ("total_div_iters", "total_incomp_iters")}
    p.destroy()
    t0 = time.perf_counter()
    diff.diff_forward(s, args.steps, every)
    t1 = time.perf_counter()
    loss, g = loss_grad(s.get_field("pos"))
    t2 = time.perf_counter()
    gx, gv, gvis = diff.diff_backward(s, g, None)
    t3 = time.perf_counter()
    clocks = clk.stop()
    fwd_s, bwd_s = t1 - t0, t3 - t2
    s.destroy()
    value = nf * args.steps / (fwd_s + bwd_s) / 1e6
    cfg = {"workload": "diff_dfsph", "fluid": nf, "boundary": int((~mask).sum()), "substeps": args.steps,
           "b200": extra, "checkpoint_every": every, "loss": loss, "dl_dviscosity": gvis,
           "pressure_iterations": {"div": int(plain_iters["total_div_iters"]),
                                   "incomp": int(plain_iters["total_incomp_iters"])},
           "forward_value": nf * args.steps / plain_s / 1e6, "recorded_forward_value": nf * args.steps / fwd_s / 1e6,
           "adjoint_over_forward": (fwd_s + bwd_s) / plain_s,
           "adjoint_over_forward_definition": "(recorded forward + backward) / plain forward, wall clock",
           "recorded_forward_over_forward": fwd_s / plain_s, "backward_over_forward": bwd_s / plain_s,
           "grad_v0_norm": float(np.linalg.norm(gv[mask])), "grad_x0_norm": float(np.linalg.norm(gx[mask])),
           "timing": "host wall clock around each synchronous C-ABI call (inputs resident on the device)",
           "l2": "per-substep tapes (lists 15 MB, iteration records 2 MB each) larger than L2 in total"}
    if args.fd_steps > 0 and args.fd_directions > 0:
        from oracle import oracle as O
        T = min(args.fd_steps, args.steps)
        s = solver()
        x0, v0 = s.get_field("pos").astype(np.float64), s.get_field("vel").astype(np.float64)
        maxnbr = int(sc.config["DFSPH"]["Required"]["maxNeighborNum"])
        diff.diff_forward(s, T, every, keep_lists=True)
        lists = [diff.diff_lists(s, t, maxnbr) for t in range(T)]
        iters = [diff.diff_iterations(s, t) for t in range(T)]
        _, g = loss_grad(s.get_field("pos"))
        gx, gv, gvis = diff.diff_backward(s, g, None)
        s.destroy()
        d = O.DfsphDiff(sc)
        xT, _, states, used = d.rollout(x0, v0, T, iters, lists=lists, record=True)
        _, g64 = loss_grad(xT)
        ox, ov, ovis = d.adjoint(states, used, g64.astype(np.float64), np.zeros_like(x0))
        rel = lambda a, b: float(np.linalg.norm(a[mask] - b[mask]) / np.linalg.norm(b[mask]))
        rng = np.random.default_rng(5006)
        errs, errs64 = [], []
        for _ in range(args.fd_directions):
            dv = np.zeros_like(v0)
            dv[mask] = rng.normal(size=(nf, 3))
            dv /= np.linalg.norm(dv)

            def L(e):
                x, _, _, _ = d.rollout(x0, v0 + e * dv, T, iters, lists=lists)
                m = x[mask].mean(0)
                return float(((m - target) ** 2).sum())
            fd = (L(1e-4) - L(-1e-4)) / 2e-4
            errs.append(abs(float((gv.astype(np.float64) * dv).sum()) - fd) / abs(fd))
            errs64.append(abs(float((ov * dv).sum()) - fd) / abs(fd))
        # A central difference whose step moves a particle's compression error across the clamp
        # delta = max(delta, 0) of a pressure-solve iteration sees a kink the adjoint does not;
        # the FP64 adjoint of the same map shows which departures are the secant's.
        cfg["fd_check"] = {"substeps": T, "iterations": iters, "directions": args.fd_directions, "eps": 1e-4,
                           "max_rel_err": max(errs), "rel_errs": errs, "fp64_adjoint_rel_errs": errs64,
                           "vs_fp64_adjoint": {"x0": rel(gx, ox), "v0": rel(gv, ov)},
                           # dL/dnu of a centre-of-mass loss is a cancellation residue: viscosity
                           # conserves momentum, so a uniform adjoint sees none of it
                           "dl_dviscosity": {"gpu": gvis, "fp64": ovis},
                           "reference": "FP64 CPU oracle, the GPU's lists and iteration counts frozen"}
    return {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * (fwd_s + bwd_s) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "clocks": clocks}


DEFAULT_STEPS = {"dfsph_1m": 200, "pbf": 1000, "pbf_m1": 1000, "immct_500k": 30, "batched": 200, "batched_m1": 200,
                 "diff_pbf": 200, "diff_dfsph": 100, "dfsph_1m_dd": 50}
# "B200" keys a workload always runs with, beside the autotuned ones: the DFSPH 1M scene steps
# with the adaptive CFL 0.4 rule capped at its 1 ms timeStep, as the benchmark's configuration
# states (the dam break stays below 4 m/s over the timed substeps, so the step is the cap
# throughout, the same work as the reference's fixed step).
FIXED_EXTRA = {"dfsph_1m": {"cfl": 0.4}}


def run_domains(args, rank, world, dist, torch) -> dict:
    """dfsph_1m_dd: the DFSPH 1M scene decomposed into slabs along x (vtp/domain.py), one slab per
    rank under torchrun (NCCL point-to-point and all-reduce between the GPUs) or, in one process,
    --domains slabs as threads on this GPU.  Strong scaling: the whole scene's particle-steps over
    the slowest rank's CUDA-event time.  The configuration of the dfsph_1m workload, its adaptive
    step included (one max all-reduce of |v|^2 per substep)."""
    from vtp import domain, scenes
    sc = scenes.dfsph_1m()
    extra = json.loads(args.extra) if args.extra else default_extra("dfsph_1m")
    arrays = domain.scene_arrays(sc)
    arrays.config = json.loads(json.dumps(arrays.config))
    arrays.config["B200"] = extra
    ranks = world if world > 1 else max(1, args.domains)
    plan = domain.plan_slabs(arrays, ranks)
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else args.steps

    def timed(r):
        r.step(args.warmup)
        before = r.stages.launches
        ms = r.timed_steps(args.steps)
        return {"ms": ms, "launches": r.stages.launches - before, "iters": list(r.iters[-args.steps:]),
                "owned": int(r.pos.shape[0])}

    def e2e(r):
        # the same substeps on fresh ranks; every substep each rank's owned state goes
        # device -> page-locked host -> device around it
        r.step(args.warmup)
        cap = r.stages.capacity
        hp = torch.empty((cap, 3), dtype=torch.float32, pin_memory=True)
        hv = torch.empty((cap, 3), dtype=torch.float32, pin_memory=True)
        io = 0
        torch.cuda.current_stream().synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            n = r.pos.shape[0]
            hp[:n].copy_(r.pos, non_blocking=True)
            hv[:n].copy_(r.vel, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            r.pos = hp[:n].to(r.pos.device, non_blocking=True)
            r.vel = hv[:n].to(r.vel.device, non_blocking=True)
            io += 24 * n
            r.substep()
        torch.cuda.current_stream().synchronize()
        return {"e2e_s": time.perf_counter() - t0, "io": io}

    clk = Clocks(int(os.environ.get("LOCAL_RANK", 0)) if world > 1 else 0)
    clk.start()
    if world > 1:
        with torch.cuda.stream(torch.cuda.Stream()):
            r = domain.DomainRank(arrays, plan, domain.TorchComm())
            res = [timed(r)]
            r.close()
            r = domain.DomainRank(arrays, plan, domain.TorchComm())
            ee = [e2e(r)]
            r.close()
        t = torch.tensor([res[0]["ms"], ee[0]["e2e_s"], res[0]["launches"], ee[0]["io"]], dtype=torch.float64,
                         device="cuda")
        tm = t[:2].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        ts = t[2:].clone()
        dist.all_reduce(ts, op=dist.ReduceOp.SUM)
        max_ms, e2e_s, launches, io = float(tm[0]), float(tm[1]), int(ts[0]), float(ts[1])
        owned = None
    else:
        res = domain.local_ranks(arrays, plan, timed)
        ee = domain.local_ranks(arrays, plan, e2e)
        max_ms = max(x["ms"] for x in res)
        e2e_s = max(x["e2e_s"] for x in ee)
        launches = sum(x["launches"] for x in res)
        io = sum(x["io"] for x in ee)
        owned = [x["owned"] for x in res]
    clocks = clk.stop()
    nf = sc.n_fluid
    iters = res[0]["iters"]
    value = nf * args.steps / (max_ms / 1e3) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "dfsph_1m_dd", "fluid": nf, "boundary": sc.n_boundary, "dt": 1e-3,
                   "halo": "peer stores" if ranks > 1 else "none (one slab)",
                   "parallelism": f"slabs{ranks}" + ("" if world > 1 else " (threads on one GPU)"),
                   "slab_axis": plan.axis, "slab_bounds": list(plan.bounds), "ghost": plan.ghost,
                   "owned_at_end": owned,
                   "div_iters_total": sum(i[0] for i in iters), "incomp_iters_total": sum(i[1] for i in iters),
                   "b200": extra, "l2": "working set above L2 (1.45M particles); no flush between substeps"},
        "clocks": clocks,
        "gpu_launches": launches,
        "roofline": None,
        "e2e": {"value": nf * e2e_steps / e2e_s / 1e6, "unit": METRIC, "h2d_bytes_per_step": io / e2e_steps,
                "d2h_bytes_per_step": io / e2e_steps, "steps": e2e_steps},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc, args.cpu_seconds)
    return line


def default_extra(workload: str) -> dict:
    """The "B200" block a workload runs with when --extra is not given: the autotuner's cached
    launch configuration for it on this GPU (vtp/tuned.json, written by vtp/autotune.py --write)
    plus the workload's fixed keys."""
    from vtp import autotune
    extra = autotune.tuned_extra(workload)
    extra.update(FIXED_EXTRA.get(workload, {}))
    return extra


L2_BYTES = 126e6


def neighbor_pass(kind, prof, substeps, nf, K, k_mean, peak, peak_kind) -> dict:
    """The whole neighbour pass of one substep (hash, scan, scatter, rank/reorder, list build:
    per-kernel CUDA events) against the HBM ceiling, with the bytes of the neighbour-pass work
    model (fluid re-bin and cell tables; the list writes beside it)."""
    from vtp.bytes_model import UGNS_KERNELS, neighbor_pass_bytes
    ms = sum(prof.get(k, (0.0, 0))[0] for k in UGNS_KERNELS) / max(substeps, 1)
    sort_ms = sum(prof.get(k, (0.0, 0))[0] for k in UGNS_KERNELS[:-1]) / max(substeps, 1)
    b = neighbor_pass_bytes(kind, nf, K)
    lists = 4.0 * k_mean * nf
    gbs = b / (ms / 1e3) / 1e9 if ms else None
    return {"kernels": list(UGNS_KERNELS), "ms_per_substep": ms, "sort_ms_per_substep": sort_ms,
            "bytes_per_substep": b, "achieved": gbs, "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
            "frac": gbs / peak if gbs else None, "list_bytes_per_substep": lists,
            "frac_with_lists": (b + lists) / (ms / 1e3) / 1e9 / peak if ms else None,
            "sort_frac": b / (sort_ms / 1e3) / 1e9 / peak if sort_ms else None}


def l2_note(s, req) -> str:
    """Working set of one substep (state arrays, both buffers, plus the fluid
    neighbour lists) against the 126 MB L2; substeps run back to back without a
    flush, as a simulation runs them."""
    c = s.counts()
    ws = c["total"] * 160 + c["fluid"] * int(req["maxNeighborNum"]) * 4
    rel = "larger than" if ws > L2_BYTES else "smaller than"
    return f"working set ~{ws / 1e6:.0f} MB per replica, {rel} L2 (126 MB); no flush between substeps"


def launch_ranks(n: int) -> int:
    """`--gpus N` without a launcher: start N ranks of this same command, one process per GPU,
    through torch.distributed.run on 127.0.0.1 (each rank then initialises NCCL and reads
    RANK / LOCAL_RANK / WORLD_SIZE like under an outer torchrun).  Rank 0 prints the line; the
    process group's own timeout ends ranks that wait for one another, `timeout` bounds the rest."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.steps is None:
        args.steps = DEFAULT_STEPS[args.workload]
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.scene_index < 0:
        return launch_ranks(args.gpus)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        # one GPU per process: the library and torch both see only this rank's device
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    import numpy as np
    import torch

    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import vtp
    vtp.lib()
    if args.workload in ("diff_pbf", "diff_dfsph"):
        if rank == 0:
            run = run_diff if args.workload == "diff_pbf" else run_diff_dfsph
            print(json.dumps(run(args, torch)), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    if args.workload == "dfsph_1m_dd":
        line = run_domains(args, rank, world, dist, torch)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return 0
    if args.workload in ("batched", "batched_m1"):
        line = run_batched(args, rank, world, local, dist, torch)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            mix = batched_mix(args.workload)
            a = cpu_baseline(mix[0], args.cpu_seconds / 2)
            d = cpu_baseline(mix[48], args.cpu_seconds / 2)
            # combined rate: fluid particle-steps of both samples over their summed time
            t_a = 1.0 / a["value"] if a["value"] else 0.0
            t_d = 1.0 / d["value"] if d["value"] else 0.0
            line["cpu_baseline"] = {"value": 2.0 / (t_a + t_d) if t_a + t_d else 0.0, "unit": METRIC,
                                    "cores": a["cores"], "kind": "port",
                                    "sample": f"scene 0 (PBF): {a['sample']}; scene 48 (DFSPH): {d['sample']}"}
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return 0
    sc = make_scene(args.workload)
    extra = json.loads(args.extra) if args.extra else default_extra(args.workload)
    if args.block:
        extra["blockSize"] = args.block
    s = vtp.solver_from_scene(sc, extra=extra or None)
    assert s.initialize(), s.last_error
    if args.warmup:
        assert s.tickNsteps(args.warmup), s.last_error
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = Clocks(local if world > 1 else 0)
    clk.start()
    t0 = time.perf_counter()
    ok = s.tickNsteps(args.steps)
    wall = time.perf_counter() - t0
    clocks = clk.stop()
    assert ok, s.last_error
    torch.cuda.synchronize()
    dev_ms = s.stage_times()[2]
    launches = s.launch_count()
    st = s.stats()
    t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    nf = sc.n_fluid
    value = nf * args.steps * world / (max_ms / 1e3) / 1e6

    # Per-kernel device times over a few extra substeps (CUDA events around each launch).
    prof = s.profile_kernels(args.profile_steps)
    cnt, nb = None, None
    k_mean = 0.0
    try:
        cnt_all, _ = s.get_neighbors(int(sc.config[sc.solver]["Required"]["maxNeighborNum"]))
        fmask = np.concatenate([np.full(o.n, o.material == 0) for o in sc.objects])
        k_mean = float(np.mean(np.maximum(cnt_all[fmask].astype(np.float64) - 1.0, 0.0)))
    except Exception:
        pass
    from vtp.bytes_model import kernel_bytes, kernel_flops
    req = sc.config[sc.solver]["Required"]
    h = float(np.float32(np.float32(req["particleRadius"]) * np.float32(4)))
    K = grid_buckets(req, extra)
    N = sc.n_total
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_launches) = dom
    per_launch_ms = dom_ms / max(dom_launches, 1)
    P = len(req.get("phaseRestDensity", [])) or 1
    b = kernel_bytes(sc.solver, dom_name, N, nf, K, k_mean, P)
    peak, peak_kind = peaks()
    roofline = roofline_of(dom_name, b, kernel_flops(dom_name, nf, k_mean), per_launch_ms, peak, peak_kind,
                           clocks, args.workload)
    kernels = {k: {"ms_total": round(v[0], 4), "launches": v[1], "share": round(v[0] / sum(x[0] for x in prof.values()), 4)}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    npass = neighbor_pass(sc.solver, prof, args.profile_steps, nf, K, k_mean, peak, peak_kind)

    l2 = l2_note(s, req)
    cons = s.conservation()
    s.destroy()

    # e2e through the public API, over the same substeps as the timed run (a fresh solver of
    # the same scene, the same warm-up): every step the fluid state (positions and velocities
    # of the fluid objects; boundary particles are static) goes host -> device from pinned
    # memory, one substep runs, and the new fluid state comes back device -> host.
    s = vtp.solver_from_scene(sc, extra=extra or None)
    assert s.initialize(), s.last_error
    if args.warmup:
        assert s.tickNsteps(args.warmup), s.last_error
    bufs = state_buffers(s, fluid_ranges(sc), torch)
    e2e_steps = args.e2e_steps if args.e2e_steps > 0 else args.steps
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        state_round_trip(s, bufs)
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_val = nf * e2e_steps * world / float(te.item()) / 1e6

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "fluid": nf, "boundary": sc.n_boundary,
                   "dt": req["timeStep"], "dt_last": st.get("last_dt"), "parallelism": f"replicas{world}",
                   "div_iters_total": st["total_div_iters"], "incomp_iters_total": st["total_incomp_iters"],
                   "mean_neighbors": round(k_mean, 2),
                   "mean_density_error": cons["mean_density_error"],
                   "l2": l2,
                   "b200": extra,
                   "wall_ms_per_step": 1e3 * wall / args.steps},
        "clocks": clocks,
        "gpu_launches": int(launches),
        "roofline": roofline,
        "neighbor_pass": npass,
        "kernels": kernels,
        "e2e": {"value": e2e_val, "unit": METRIC, "h2d_bytes_per_step": state_bytes(bufs),
                "d2h_bytes_per_step": state_bytes(bufs), "steps": e2e_steps,
                "substeps": f"{args.warmup + 1}-{args.warmup + e2e_steps} of a fresh solver"},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc, args.cpu_seconds)
    s.destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
