#!/usr/bin/env python3
"""Throughput of the mCDFCI iteration on one B200 (N ranks = N replicas).

Workload: the synthetic 24-orbital, 6 alpha + 6 beta electron Hamiltonian
(~1.8e10 determinants, mcdfci_b200.synth "n24_6a6b", seed 0) with
num_of_coordinate = estimate = 32, max_memory = 64 GB, z_threshold = 1e-9,
FP64.  A step is one iteration of the hot path: pick 32 coordinates, generate
their 32 Hamiltonian columns (16,471 entries each), solve the 33x33 subspace
eigenproblem, apply x += dx and z += H_col * dx in the hash wavefunction.

  value        coordinate updates/s over all ranks (32 per step per rank),
               from CUDA events on the solver's stream around the product
               path (CUDA graphs of 64 iterations), max over ranks; a pass of
               direct launches with an event between the two kernels of every
               iteration gives the per-kernel times of the roofline
  e2e          the same metric through the C ABI a user calls
               (mcd_create_from_fcidump from host data + mcd_solve + read of
               the result), wall clock, host<->device copies inside
  roofline     column kernel: 40 algorithmic bytes per column entry (16-byte
               key probe, 8-byte x read, 8-byte z read, 8-byte z write) over
               its average device time, against the measured HBM copy peak
  cpu_baseline the reference cdfci_omp, compiled from its sources, on a
               bounded sample of the same workload on this host's cores
  table_growth_timed
               the table growths inside value's timed iterations (they count
               in it): how many, their host time and its rehash part
  aged         value's timing repeated after --aged-iterations iterations in
               all, on the grown table (load factor stated)
  e2e_detail   the end-to-end run's stages: host tables, device allocation,
               upload, table fill, graph builds, growths (with their
               allocation, rehash and frees), report read-backs

  batched      the 32-point dissociation curve (synthetic n16_5a5b points,
               k = m = 16, 1 GB table each): coordinate updates/s of all 32
               instances advanced together (mcd_batch_*) against one instance
               on its own, from CUDA events

Multi-GPU: the iteration does not shard (a sequential block Gauss-Southwell
chain), so --gpus N runs N independent replicas with no collective on the
data path ("weak" scaling).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  python bench.py --workload curve [--curve-iterations N]
      time for the whole 32-point curve, batched against one point after
      another, both through the public API, and the time until every point's
      energy is within 1e-6 Ha of the energy it reaches after N iterations
"""
import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "coord updates/s"
UNIT = "coordinate_updates/s"
WORKLOAD = "n24_6a6b"
BYTES_PER_ENTRY = 40
REF_EXE = os.path.join(HERE, "oracle", "_ref", "cdfci_omp")
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=400)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--k", type=int, default=32)
    ap.add_argument("--m", type=int, default=32)
    ap.add_argument("--max-memory", type=float, default=64.0)
    ap.add_argument("--z-threshold", type=float, default=1e-9)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample", type=int, default=600, help="reference iterations timed for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--groups", type=int, default=0, help="CTAs per Hamiltonian column (0: the library's choice)")
    ap.add_argument("--workload", choices=["n24", "curve"], default="n24")
    ap.add_argument("--curve-points", type=int, default=32)
    ap.add_argument("--curve-iterations", type=int, default=20000)
    ap.add_argument("--curve-report", type=int, default=1000)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-curve throughput object")
    ap.add_argument("--aged-iterations", type=int, default=2000,
                    help="iterations in all before the aged-table timing (0: skip it)")
    ap.add_argument("--aged-steps", type=int, default=256)
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuner object")
    ap.add_argument("--phases", action="store_true",
                    help="print where the device time of an iteration goes (leader and column phase timers) "
                         "on --phase-workload instead of the bench line")
    ap.add_argument("--phase-workload", default="n24_6a6b")
    ap.add_argument("--eig-method", type=int, default=2, choices=[0, 1, 2],
                    help="subspace eigenproblem: 1 shifted inverse iteration first, 0 the full reduction")
    ap.add_argument("--scatter-sweep", action="store_true",
                    help="with --phases: also sweep the table's scattered-access probe")
    return ap.parse_args()


def config(args):
    return {
        "workload": f"{WORKLOAD}: norb=24, 6a/6b (~1.8e10 dets), synthetic seed {args.seed}",
        "num_of_coordinate": args.k,
        "estimate": args.m,
        "max_memory_gb": args.max_memory,
        "z_threshold": args.z_threshold,
        "step": "one mCDFCI iteration",
        "l2": "inputs larger than L2: the hash wavefunction (at least 2^27 slots x 32 B = 4.3 GB, growing "
              "as it fills up to 2^31 slots = 68.7 GB for 64 GB) vs 126 MB L2",
        "parallelism": "replicas",
    }


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
             "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    """DRAM bytes per column-kernel launch from the committed ncu summary."""
    p = os.path.join(HERE, "profiles", "column_kernel_n24_6a6b.md")
    try:
        txt = open(p).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


CURVE = "n16_5a5b"
CURVE_K = 16
CURVE_GB = 1.0


def write_curve(d, points, seed):
    """The dissociation-curve points: integrals interpolated between two
    endpoints, the second with its off-diagonal couplings scaled x3."""
    from mcdfci_b200 import synth

    paths = []
    for i in range(points):
        t = i / (points - 1) if points > 1 else 0.0
        p = os.path.join(d, f"{CURVE}_t{i:02d}.fcidump")
        synth.write_fcidump(p, CURVE, seed=seed, t=t)
        paths.append(p)
    return paths


CURVE_FIXTURE = os.path.join(HERE, "tests", "golden", "curve_energies.json")
CURVE_TOL = 1e-6


def curve_reference():
    """Energies the reference reached on each curve point (its compiled solver
    run by tests/golden/make_curve.py), or None when the fixture lacks points."""
    try:
        with open(CURVE_FIXTURE) as f:
            data = json.load(f)
    except OSError:
        return None
    pts = {p["point"]: p for p in data["points"]}
    return pts if len(pts) == 32 else None


def curve_time_to_reference(mc, paths, local_rank, ref, report=200, max_iterations=200000, sample=8):
    """Wall time through the public API until every point's energy is within
    1e-6 Ha of (at or below) the reference's energy on that point.  Batched:
    mcd_batch_create + mcd_batch_solve, each instance retired at its first
    report past its target, until the last gets there.  Plain: mcd_create +
    mcd_solve point after point, each stopped at its first report past its
    target, on `sample` evenly spaced points, summed and scaled to all of them.
    Both include the set-up (Hamiltonian tables, tables, fills).  A point on
    which the reference stopped early ("Factorization fails!") has its last
    reported energy as the target; one that stopped before its first report
    has none: the batch retires it at its first report and the plain sample
    leaves it out."""
    n = len(paths)
    targets = [None if ref[i]["energy"] is None else ref[i]["energy"] + CURVE_TOL for i in range(n)]
    with_target = [i for i in range(n) if targets[i] is not None]
    opts = dict(num_of_coordinate=CURVE_K, estimate=CURVE_K, max_memory=CURVE_GB, z_threshold=0.0,
                threshold=0.0, device=local_rank, num_iterations=max_iterations, report_interval=report)
    fc = [mc.Fcidump(p) for p in paths]
    reached_b = {}
    t0 = time.perf_counter()
    b = mc.CDFCIBatch(fc, **opts)

    def bcb(i, r):
        if targets[i] is None:
            return "retire"
        if r["energy"] <= targets[i]:
            reached_b[i] = (time.perf_counter() - t0, r["iteration"], r["energy"])
            return "retire"
        return False

    b.solve(callback=bcb)
    t_batch = time.perf_counter() - t0
    b.close()
    nt = len(with_target)
    idx = sorted({with_target[round(j * (nt - 1) / (sample - 1))] for j in range(sample)})
    plain = []
    for i in idx:
        t1 = time.perf_counter()
        s = mc.CDFCI(fc[i], **opts)
        got = {}

        def pcb(r, i=i, got=got):
            if r["energy"] <= targets[i]:
                got["it"] = r["iteration"]
                return True
            return False

        s.solve(callback=pcb)
        plain.append((i, time.perf_counter() - t1, got.get("it")))
        s.close()
    plain_s = sum(t for _, t, _ in plain) * nt / len(plain)
    ok_b = sorted(reached_b) == with_target
    ok_p = all(it is not None for _, _, it in plain)
    return {
        "metric": "time to E within 1e-6 Ha of the reference, batched vs plain", "unit": "s",
        "batched_s": t_batch if ok_b else None, "plain_s": plain_s if ok_p else None,
        "speedup": (plain_s / t_batch) if (ok_b and ok_p) else None,
        "points_reached_batched": len(reached_b),
        "points_with_target": nt,
        "reference_failed": [{"point": i, "message": ref[i]["failed"]["message"],
                              "last_report": ref[i]["reports"][-1]["iteration"] if ref[i]["reports"] else None}
                             for i in range(n) if "failed" in ref[i]],
        "iterations_to_target_batched": {"min": min(v[1] for v in reached_b.values()) if reached_b else None,
                                         "max": max(v[1] for v in reached_b.values()) if reached_b else None},
        "plain_sample": [{"point": i, "seconds": t, "iterations": it} for i, t, it in plain],
        "target": ("per point, the reference's final energy (its last reported one where it stopped early) + "
                   "1e-6 Ha, the reference (the solver compiled from its "
                   "sources, tests/golden/make_curve.py) after " + str(ref[0]["iterations"]) + " iterations at k = "
                   + str(ref[0]["k"]) + "; checked at reports every " + str(report) + " iterations"),
        "plain_is": (f"sum over {len(plain)} evenly spaced points (of those with a target) of create + solve to "
                     f"the target, times {nt}/{len(plain)}"),
    }


def curve_throughput(mc, paths, local_rank, steps=500, warmup=500):
    """Device-timed coordinate updates/s: the whole curve as one batch, and
    one point on its own."""
    opts = dict(num_of_coordinate=CURVE_K, estimate=CURVE_K, max_memory=CURVE_GB, z_threshold=0.0,
                threshold=0.0, device=local_rank)
    fc = [mc.Fcidump(p) for p in paths]
    b = mc.CDFCIBatch(fc, **opts)
    b.reset()
    b.run_iterations(warmup)
    tb = b.run_iterations_timed(steps)["total_ms"]
    b.close()
    s = mc.CDFCI(fc[0], **opts)
    s.reset()
    s.run_iterations(warmup)
    ts = s.run_iterations_timed(steps)["total_ms"]
    s.close()
    batched = len(paths) * CURVE_K * steps / (tb / 1000.0)
    plain = CURVE_K * steps / (ts / 1000.0)
    return {"workload": f"{len(paths)} x {CURVE} curve points, k = m = {CURVE_K}, {CURVE_GB} GB table each",
            "batched_updates_per_s": batched, "one_point_updates_per_s": plain,
            "batched_ms_per_iteration": tb / steps, "one_point_ms_per_iteration": ts / steps,
            "speedup_over_one_point_at_a_time": batched / plain,
            "timing": f"CUDA events, {steps} iterations after {warmup}"}


def curve_arm(args, local_rank):
    """The curve solved both ways through the public API (create + solve +
    reports + result, wall clock), and the time until every point is within
    1e-6 Ha of the energy the batch reaches after N iterations."""
    import mcdfci_b200 as mc

    n_it, rep = args.curve_iterations, args.curve_report
    opts = dict(num_of_coordinate=CURVE_K, estimate=CURVE_K, max_memory=CURVE_GB, z_threshold=0.0,
                threshold=0.0, device=local_rank, num_iterations=n_it, report_interval=rep)
    tmp = tempfile.mkdtemp(prefix="mcd_curve_")
    try:
        paths = write_curve(tmp, args.curve_points, args.seed)
        fc = [mc.Fcidump(p) for p in paths]
        t0 = time.perf_counter()
        b = mc.CDFCIBatch(fc, **opts)
        t_ready = time.perf_counter()
        eb = b.solve()
        t_batch = time.perf_counter() - t0
        hist_b = [[(r["time_s"], r["energy"]) for r in reps] for reps in b.reports]
        b.close()
        plain_times, hist_p, ep = [], [], []
        for f in fc:
            t1 = time.perf_counter()
            s = mc.CDFCI(f, **opts)
            ts_ready = time.perf_counter() - t1
            ep.append(s.solve())
            plain_times.append(time.perf_counter() - t1)
            hist_p.append([(ts_ready + r["time_s"], r["energy"]) for r in s.reports])
            s.close()
        tol = 1e-6
        # Away from convergence the two runs of a point follow different
        # trajectories (the pick order depends on the order of concurrent
        # atomic updates), so each point's target is the energy level both
        # of its runs reach: max(final batched, final plain) + 1e-6 Ha.
        level = [max(a, c) + tol for a, c in zip(eb, ep)]

        def first_at(hist, lvl):
            for t, e in hist:
                if e <= lvl:
                    return t
            return None

        tb = [first_at(h, level[i]) for i, h in enumerate(hist_b)]
        tp = [first_at(h, level[i]) for i, h in enumerate(hist_p)]
        t_b = (t_ready - t0) + max(tb) if all(x is not None for x in tb) else None
        t_p = sum(tp) if all(x is not None for x in tp) else None
        out = {
            "metric": "time to E within 1e-6 Ha, batched vs plain", "unit": "s", "higher_is_better": False,
            "value": t_b, "plain_value": t_p, "speedup": (t_p / t_b) if (t_b and t_p) else None,
            "target": (f"per point, the energy both its batched and its one-at-a-time run reach in {n_it} "
                       "iterations, within 1e-6 Ha; batched: set-up + the time the last point gets there; "
                       "plain: sum over points of set-up + time to get there"),
            "curve_wall_s": {"batched": t_batch, "plain_sum": sum(plain_times)},
            "max_abs_energy_difference_batched_vs_plain": max(abs(a - c) for a, c in zip(eb, ep)),
            "energies": {"first": eb[0], "last": eb[-1]},
            "config": {"workload": f"{len(paths)} x {CURVE} points (t = 0..1), k = m = {CURVE_K}, "
                                   f"{CURVE_GB} GB table each", "iterations": n_it, "report_interval": rep},
            "n_gpus": 1, "dtype": "f64", "data": "synthetic (mcdfci_b200.synth)",
        }
        print(json.dumps(out))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


def phases_arm(args, local_rank):
    """Per-iteration device time of the two kernels (CUDA events) and the SM
    cycles of each leader phase (one CTA), of each column-kernel phase per
    round of 256 entries (thread 0 of each CTA), and per column-kernel CTA its
    prelude and list merge, with the column's final merge by its last CTA."""
    import mcdfci_b200 as mc
    from mcdfci_b200 import synth

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, args.phase_workload + ".fcidump")
        synth.write_fcidump(path, args.phase_workload, seed=args.seed)
        s = mc.CDFCI(mc.Fcidump(path), num_of_coordinate=args.k, estimate=args.m, max_memory=args.max_memory,
                     z_threshold=args.z_threshold, threshold=0.0, groups=args.groups, device=local_rank,
                     eig_method=args.eig_method, num_iterations=args.warmup + args.steps)
        s.reset()
        s.run_iterations(args.warmup)
        rb = s.report()
        s.leader_sections()
        s.column_sections(enable=True)
        n = args.steps
        t = s.run_iterations_timed(n)
        lead = s.leader_sections()
        col = s.column_sections(enable=False)
        rounds = max(col.pop("rounds"), 1)
        ctas = max(col.pop("ctas"), 1)
        merges = max(col.pop("merges"), 1)
        per_cta = {"prelude": round(col.pop("prelude") / ctas), "post": round(col.pop("post") / ctas),
                   "merge": round(col.pop("merge") / merges)}
        scatter = []
        if args.scatter_sweep:
            for mode, name in enumerate(s.SCATTER_MODES):
                for entries in (527072, 8433152):
                    for cps in (3, 8):
                        for ilp in (1, 4):
                            r = s.scatter_rate(entries, 10, ilp, cps, mode)
                            scatter.append({"mode": name, "slots": entries, "ctas_per_sm": cps, "ilp": ilp,
                                            "slots_per_s": r, "us_per_launch": entries / r * 1e6})
        rep = s.report()
        eig = {"fast_updates": rep["inv_updates"] - rb["inv_updates"],
               "fast_steps_avg": (rep["inv_steps"] - rb["inv_steps"]) / max(1, rep["inv_updates"] - rb["inv_updates"]),
               "fallbacks": rep["eig_fallbacks"] - rb["eig_fallbacks"], "max_residual": rep["max_residual"]}
        groups = s.launch_info()["groups"]
        s.close()
    print(json.dumps({
        "workload": args.phase_workload, "k": args.k, "m": args.m, "max_memory_gb": args.max_memory,
        "warmup": args.warmup, "iterations": n, "groups": groups,
        "leader_us_per_iteration": 1000.0 * t["leader_ms"] / n,
        "column_us_per_iteration": 1000.0 * t["column_ms"] / n,
        "leader_cycles_per_iteration": {k: round(v / n) for k, v in lead.items()},
        "column_cycles_per_round": {k: round(v / rounds) for k, v in col.items()},
        "column_cycles_per_cta": per_cta,
        "column_rounds_per_cta": round(rounds / ctas, 2),
        "energy": rep["energy"], "z_size": rep["z_size"], "eig": eig, "eig_method": args.eig_method,
        "scatter_probe": scatter,
    }, indent=1))
    return 0


def curve_sharded_arm(args, rank, world, local_rank):
    """The curve spread over the node's GPUs (mcdfci_b200.curve): point i on
    rank i mod world, each rank's share solved as one batch, energies gathered
    to rank 0; wall time from a barrier before the first creation to a
    barrier after the last solve, max over ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    from mcdfci_b200 import curve
    from mcdfci_b200.replicas import max_over_ranks

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    tmp = tempfile.mkdtemp(prefix="mcd_curve_")
    try:
        paths = write_curve(tmp, args.curve_points, args.seed)
        opts = dict(num_of_coordinate=CURVE_K, estimate=CURVE_K, max_memory=CURVE_GB, z_threshold=0.0,
                    threshold=0.0, device=local_rank, num_iterations=args.curve_iterations,
                    report_interval=args.curve_report)
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = curve.solve_curve(len(paths), curve.batch_solver(paths, **opts), dist)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        wall = max_over_ranks(dt, dist, "cuda")
        if rank == 0:
            print(json.dumps({
                "metric": "curve wall time, points spread over GPUs", "unit": "s", "value": wall,
                "higher_is_better": False, "n_gpus": world, "scaling": "strong",
                "points": len(paths), "energies": [r["energy"] for r in out],
                "config": {"workload": f"{len(paths)} x {CURVE} points (t = 0..1), k = m = {CURVE_K}, "
                                       f"{CURVE_GB} GB table each", "iterations": args.curve_iterations,
                           "report_interval": args.curve_report, "sharding": "point i on rank i mod world"},
                "dtype": "f64", "data": "synthetic (mcdfci_b200.synth)"}))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        dist.destroy_process_group()
    return 0


def autotune_object(mc, tmp, args, local_rank):
    """CTAs per column chosen by the autotuner against the fixed rule, from
    its timed trials (16 iterations per candidate, column-kernel device time),
    on three workloads."""
    from mcdfci_b200 import synth

    out = {}
    for name, k, mem, zt in (("n24_6a6b", 32, 8.0, 1e-9), ("n16_5a5b", 16, 1.0, 0.0), ("n42_24a24b", 64, 100.0, 1e-5)):
        p = os.path.join(tmp, f"tune_{name}.fcidump")
        synth.write_fcidump(p, name, seed=args.seed)
        s = mc.CDFCI(mc.Fcidump(p), num_of_coordinate=k, estimate=k, max_memory=mem, z_threshold=zt, threshold=0.0,
                     device=local_rank, autotune=True, num_iterations=256)
        try:
            s.reset()
            s.run_iterations(16 * 10)
            info = s.autotune_info()
        except mc.McdError as e:
            out[name] = {"k": k, "error": str(e)}
            continue
        finally:
            s.close()
        rule_us = next((t["column_us"] for t in info["trials"] if t["groups"] == info["rule"]), None)
        best_us = min((t["column_us"] for t in info["trials"]), default=None)
        out[name] = {"k": k, "rule_groups": info["rule"], "chosen_groups": info["chosen"],
                     "rule_column_us": rule_us, "chosen_column_us": best_us, "trials": info["trials"]}
    return out


def write_workload(d, seed):
    from mcdfci_b200 import synth

    path = os.path.join(d, WORKLOAD + ".fcidump")
    synth.write_fcidump(path, WORKLOAD, seed=seed)
    return path


# ---------------------------------------------------------------------------
# The reference solver, built from its sources (oracle/Makefile).

REF_ATTEMPTS = 4


def run_reference(fcidump, k, m, zt, warmup, steps, max_memory, threads):
    """Runs cdfci_omp for warmup+steps iterations; returns (updates/s, k_eff,
    seconds) measured from its own cumulative timer between the report at
    `warmup` and the one at `warmup+steps`.  The reference's OpenMP runs do
    not repeat one another, and some stop with "Factorization fails!" (exit
    status 255, src/solver.h:444-450); such a run is started again, up to
    REF_ATTEMPTS runs in all."""
    r = math.gcd(warmup, steps) if warmup > 0 else steps
    with tempfile.TemporaryDirectory() as d:
        deck = os.path.join(d, "input.json")
        with open(deck, "w") as f:
            json.dump({"hamiltonian": {"fcidump_path": fcidump, "threshold": 0.0},
                       "solver": {"cdfci": {"num_iterations": warmup + steps, "report_interval": r,
                                            "z_threshold": zt, "z_threshold_search": False,
                                            "max_memory": max_memory, "coordinate_pick": "gcd_grad",
                                            "coordinate_update": "eig", "num_of_coordinate": k,
                                            "estimate": m}}}, f)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
        for attempt in range(REF_ATTEMPTS):
            res = subprocess.run([REF_EXE, deck], capture_output=True, text=True, env=env, timeout=1800)
            if res.returncode == 0 or "Factorization fails" not in res.stdout:
                break
    if res.returncode != 0:
        raise RuntimeError(f"reference failed ({attempt + 1} runs): " + (res.stderr or res.stdout)[-500:])
    k_eff = k
    m_warn = re.search(r"Not enough processes\. Set k = (\d+)", res.stdout)
    if m_warn:
        k_eff = int(m_warn.group(1))
    times = {}
    for line in res.stdout.splitlines():
        p = line.split()
        if len(p) >= 9 and re.match(r"^\d+$", p[0]) and re.match(r"^-?\d+\.\d+$", p[1]):
            times[int(p[0])] = float(p[7])
    t0 = times.get(warmup, 0.0)
    t1 = times[warmup + steps]
    dt = t1 - t0
    return k_eff * steps / dt, k_eff, dt


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    if not os.path.exists(REF_EXE):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cdfci_omp not built (needs the reference sources)"}))
        return 0
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        path = write_workload(d, args.seed)
        # The reference allocates its whole table in host RAM up front; a
        # smaller max_memory keeps the run within this host's memory and
        # does not change the per-iteration work until the table fills.
        mem = min(args.max_memory, 4.0)
        # The reference's timer prints hundredths of a second: at least 600
        # iterations keep that resolution well below the measured interval.
        # (at least 100 warm-up iterations, and a count they divide, keep its
        # reports few).
        w_eff = max(args.warmup, 100)
        n_meas = -(-max(args.steps, 600) // w_eff) * w_eff
        rate, k_eff, dt = run_reference(path, args.k, args.m, args.z_threshold, w_eff, n_meas, mem, threads)
    sample = (f"{n_meas} iterations after {w_eff} warm-up, k={k_eff} (capped at the core count), "
              f"max_memory {mem} GB, OMP_NUM_THREADS={threads}, OPENBLAS_NUM_THREADS=1, timed by the "
              "reference's own report clock")
    out = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / n_meas,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (mcdfci_b200.synth)", "config": config(args),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------

def b200_arm(args, rank, world, local_rank):
    import torch

    import mcdfci_b200 as mc
    from mcdfci_b200.replicas import max_over_ranks, replica_rate

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

    tmp = tempfile.mkdtemp(prefix="mcd_bench_")
    try:
        path = write_workload(tmp, args.seed)
        fc = mc.Fcidump(path)
        # End to end first: the process holds no earlier solver whose
        # teardown (the release of its tables) the clock would catch.
        e2e = None
        if not args.no_e2e:
            torch.cuda.synchronize()
            e2e = e2e_run(mc, fc, args, local_rank)
            if dist:
                e2e["value"] = replica_rate(args.k * e2e["iterations"], e2e["seconds"], world, dist, "cuda")
        # num_iterations: the iterations this run makes (the first table is
        # sized for them, up to two 64-iteration chunks).
        solver = mc.CDFCI(fc, num_of_coordinate=args.k, estimate=args.m, max_memory=args.max_memory,
                          z_threshold=args.z_threshold, threshold=0.0, device=local_rank, groups=args.groups,
                          num_iterations=args.warmup + 2 * args.steps + max(args.aged_iterations, 0) + args.aged_steps)
        solver.reset()
        solver.run_iterations(args.warmup)
        r0 = solver.report()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local_rank)
        sampler.start()
        time.sleep(0.3)
        # Per-kernel device times (direct launches with an event between the
        # two kernels of every iteration), for the roofline.
        t = solver.run_iterations_timed(args.steps)
        r_mid = solver.report()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        # The timed steps: the product path, CUDA graphs of 64 iterations on
        # the solver's stream, bracketed by events on that stream.
        ext = torch.cuda.ExternalStream(solver.stream)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        g0, st0 = solver.table_info()["growths"], solver.setup_times()
        ev0.record(ext)
        solver.run_iterations(args.steps)
        ev1.record(ext)
        ev1.synchronize()
        torch.cuda.synchronize()
        sampler.stop()
        st1 = solver.setup_times()
        growth_timed = {"growths": solver.table_info()["growths"] - g0,
                        "ms": st1["growth"] - st0["growth"],
                        "rehash_ms": st1["growth_rehash"] - st0["growth_rehash"],
                        "slots_after": solver.table_info()["capacity"]}
        if dist:
            dist.barrier()
        r1 = solver.report()
        clocks = sampler.summary()
        total_s = ev0.elapsed_time(ev1) / 1000.0
        entries = r_mid["emitted_total"] - r0["emitted_total"]
        updates = args.k * args.steps
        col_ms_avg = t["column_ms"] / args.steps
        total_max = max_over_ranks(total_s, dist, "cuda")
        value = replica_rate(updates, total_s, world, dist, "cuda")
        # The scattered-access ceiling of the same table: as many pseudo-random
        # slots as a launch has entries, each touched the way an entry touches
        # its slot (key, x, atomic z add of zero), 1 or 4 in flight per thread.
        per_launch = max(1, int(entries / args.steps))
        scatter = max(solver.scatter_rate(per_launch, 20, 1), solver.scatter_rate(per_launch, 20, 4))
        table_main = solver.table_info()
        # The same timing on an aged table: iterate on to --aged-iterations
        # iterations in all (the table grows as it fills), then time the
        # product path again.
        aged = None
        if args.aged_iterations > 0:
            done = r1["iteration"]
            if args.aged_iterations > done:
                solver.run_iterations(args.aged_iterations - done)
            ra0 = solver.report()
            n_aged = args.aged_steps
            ev0.record(ext)
            solver.run_iterations(n_aged)
            ev1.record(ext)
            ev1.synchronize()
            ra1 = solver.report()
            ta = ev0.elapsed_time(ev1) / 1000.0
            ti = solver.table_info()
            aged = {"iterations_before": ra0["iteration"], "steps": n_aged, "ms_per_step": 1000.0 * ta / n_aged,
                    "updates_per_s": args.k * n_aged / ta, "z_size": ra1["z_size"], "occupied": ra1["occupied"],
                    "table_slots": ti["capacity"], "load_factor": ra1["occupied"] / ti["capacity"],
                    "table_growths": ti["growths"], "energy": ra1["energy"],
                    "entries_per_step": (ra1["emitted_total"] - ra0["emitted_total"]) / n_aged,
                    "timing": "CUDA events on the solver's stream around the product path (graphs of 64 "
                              "iterations), table growths inside the timed steps included"}
        solver.close()

        peak, peak_kind = hbm_peak()
        achieved = (entries / args.steps) * BYTES_PER_ENTRY / (col_ms_avg / 1000.0) / 1e9
        traffic = ncu_traffic()
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "peak_source": peak_kind,
                    "kernel": "column_kernel", "entries_per_launch": entries / args.steps,
                    "algorithmic_bytes_per_entry": BYTES_PER_ENTRY, "avg_launch_ms": col_ms_avg,
                    "leader_ms_per_step": t["leader_ms"] / args.steps,
                    "table_slots": table_main["capacity"],
                    "scatter_ceiling": {"slots_per_s": scatter,
                                        "column_entries_per_s": (entries / args.steps) / (col_ms_avg / 1000.0),
                                        "frac": (entries / args.steps) / (col_ms_avg / 1000.0) / scatter,
                                        "probe": "mcd_debug_scatter_rate on the same table, best of 1 and 4 "
                                                 "slots in flight per thread, 148 x 8 CTAs of 256"}}


        tuned = None
        if not args.no_autotune:
            tuned = autotune_object(mc, tmp, args, local_rank)

        batched = None
        if not args.no_batched:
            ctmp = tempfile.mkdtemp(prefix="mcd_curve_", dir=tmp)
            cpaths = write_curve(ctmp, args.curve_points, args.seed)
            batched = curve_throughput(mc, cpaths, local_rank)
            ref = curve_reference()
            if ref is not None and args.curve_points == 32:
                batched["time_to_reference"] = curve_time_to_reference(mc, cpaths, local_rank, ref)
            else:
                batched["time_to_reference"] = {"unavailable": "tests/golden/curve_energies.json lacks points"}

        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_EXE):
            threads = os.cpu_count() or 1
            n = args.cpu_sample
            w = max(100, n // 5)
            try:
                rate, k_eff, dt = run_reference(path, args.k, args.m, args.z_threshold, w, n, 4.0, threads)
                cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                       "sample": f"{n} iterations after {w} warm-up of the same workload, k={k_eff} "
                                 f"(the reference caps k at the core count), max_memory 4 GB, "
                                 f"OMP_NUM_THREADS={threads}, {dt:.1f} s"}
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": f"failed: {e}"}

        if rank == 0:
            out = {
                "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * total_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (mcdfci_b200.synth)",
                "config": config(args),
                "e2e": {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step")} if e2e else None,
                "gpu_launches": 2 * args.steps,
                "roofline": roofline,
                "cpu_baseline": cpu,
                "batched": batched,
                "clocks": clocks,
                "energy": r1["energy"],
                "z_size": r1["z_size"],
                "table_growth_timed": growth_timed,
                "aged": aged,
                "autotune": tuned,
                "e2e_detail": e2e,
            }
            print(json.dumps(out))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


def e2e_run(mc, fc, args, local_rank):
    """create (host tables -> device) + solve (reports read back) + result."""
    import ctypes

    iters = args.steps
    interval = max(1, iters // 10)
    # Warm-up: one small solve through the same calls (7 orbitals, the same
    # k and m), so that the clock below sees a process whose kernels are
    # loaded, as the warm-up steps precede the device-timed value.
    from mcdfci_b200 import synth

    wpath = os.path.join(os.path.dirname(fc.path), "warmup_n7.fcidump")
    synth.write_fcidump(wpath, "n7_5a5b", seed=0)
    w = mc.CDFCI(mc.Fcidump(wpath), num_of_coordinate=args.k, estimate=args.m, max_memory=0.001,
                 threshold=0.0, device=local_rank, num_iterations=10, report_interval=5)
    w.solve()
    w.close()
    t0 = time.perf_counter()
    s = mc.CDFCI(fc, num_of_coordinate=args.k, estimate=args.m, max_memory=args.max_memory,
                 z_threshold=args.z_threshold, threshold=0.0, device=local_rank, num_iterations=iters,
                 report_interval=interval, groups=args.groups)
    t_created = time.perf_counter()
    s.solve()
    energy = s.result_energy
    dt = time.perf_counter() - t0  # the result is in hand; releasing the solver is not part of it
    stages = s.setup_times()
    table = s.table_info()
    s.close()
    create_ms = 1000.0 * (t_created - t0)
    breakdown = {
        "create_ms": create_ms,
        "create_host_tables_ms": stages["host_tables"],
        "create_device_alloc_ms": stages["device_alloc"],
        "create_upload_ms": stages["upload"],
        "create_device_setup_ms": stages["device_setup"],
        "create_upload_copy_ms": stages["upload_copy"],
        "create_upload_sync_ms": stages["upload_sync"],
        "solve_ms": 1000.0 * dt - create_ms,
        "solve_table_fill_ms": stages["table_fill"],
        "solve_graph_build_ms": stages["graph_build"],
        "solve_table_growth_ms": stages["growth"],
        "solve_table_growth_alloc_ms": stages["growth_alloc"],
        "solve_table_growth_rehash_ms": stages["growth_rehash"],
        "solve_table_growth_free_ms": stages["growth_free"],
        "solve_report_readback_ms": stages["reports"],
        "table_slots": table["capacity"], "table_slots_max": table["max_capacity"],
        "table_growths": table["growths"],
    }
    n = fc.norb
    nsp = n // 2
    table_bytes = 8 * (n + n * n + 2 * nsp * nsp + 2 * nsp * nsp * n + 2 * nsp + 2 * (nsp * (nsp - 1) // 2) ** 2 + nsp ** 4)
    state_bytes = 16 * 1024
    h2d = table_bytes + state_bytes
    d2h = (iters // interval) * (state_bytes + 8)
    return {"value": args.k * iters / dt, "unit": UNIT, "h2d_bytes_per_step": h2d / iters,
            "d2h_bytes_per_step": d2h / iters, "seconds": dt, "iterations": iters, "energy": energy,
            "stages": breakdown,
            "what": "mcd_create_from_fcidump (Hamiltonian tables host->device, hash table allocation) + mcd_solve "
                    f"(table fill, {iters} iterations, a report read back every {interval}) + mcd_result; "
                    "mcd_destroy after the clock; after one 10-iteration warm-up solve of a 7-orbital problem "
                    "in the same process (kernels loaded)"}


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.phases:
        if world > 1 and rank != 0:
            return 0
        import torch

        torch.cuda.set_device(local_rank)
        return phases_arm(args, local_rank)
    if args.workload == "curve":
        import torch

        torch.cuda.set_device(local_rank)
        if world > 1:
            return curve_sharded_arm(args, rank, world, local_rank)
        return curve_arm(args, local_rank)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        return b200_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
