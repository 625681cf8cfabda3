"""Where the device time of an iteration goes: the phase timers of the leader
kernel and of the column kernel, on a synthetic workload.

    python -m mcdfci_b200.phase_clocks [--workload n24_6a6b] [--k 32] [--m 32]
        [--max-memory 16] [--warmup 300] [--iterations 300] [--groups 0] [--scatter]

Prints, per iteration, the device time of the two kernels (CUDA events) and
the SM cycles of each leader phase (one CTA); per round of 256 column entries,
of each column-kernel phase (thread 0 of each CTA); and per column-kernel CTA
its prelude and list merge, with the column's final merge by its last CTA.
"""
import argparse
import json
import os
import tempfile

import mcdfci_b200 as m
from mcdfci_b200 import synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="n24_6a6b")
    ap.add_argument("--k", type=int, default=32)
    ap.add_argument("--m", type=int, default=32)
    ap.add_argument("--max-memory", type=float, default=16.0)
    ap.add_argument("--z-threshold", type=float, default=1e-9)
    ap.add_argument("--warmup", type=int, default=300)
    ap.add_argument("--iterations", type=int, default=300)
    ap.add_argument("--groups", type=int, default=0, help="CTAs per column (0: the library's choice)")
    ap.add_argument("--scatter", action="store_true",
                    help="also sweep the table's scattered-access probe (slots per launch, CTAs per SM, "
                         "slots in flight per thread)")
    args = ap.parse_args()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, args.workload + ".fcidump")
        synth.write_fcidump(path, args.workload, seed=0)
        s = m.CDFCI(m.Fcidump(path), num_of_coordinate=args.k, estimate=args.m, max_memory=args.max_memory,
                    z_threshold=args.z_threshold, threshold=0.0, groups=args.groups)
        s.reset()
        s.run_iterations(args.warmup)
        s.report()
        s.leader_sections()
        s.column_sections(enable=True)
        n = args.iterations
        t = s.run_iterations_timed(n)
        lead = s.leader_sections()
        col = s.column_sections(enable=False)
        rounds = max(col.pop("rounds"), 1)
        ctas = max(col.pop("ctas"), 1)
        merges = max(col.pop("merges"), 1)
        per_cta = {"prelude": round(col.pop("prelude") / ctas), "post": round(col.pop("post") / ctas),
                   "merge": round(col.pop("merge") / merges)}
        scatter = []
        if args.scatter:
            for entries in (527072, 2108288, 8433152, 33732608):
                for cps in (3, 8):
                    for ilp in (1, 4):
                        r = s.scatter_rate(entries, 10, ilp, cps)
                        scatter.append({"slots": entries, "ctas_per_sm": cps, "ilp": ilp, "slots_per_s": r,
                                        "us_per_launch": entries / r * 1e6})
        print(json.dumps({
            "workload": args.workload, "k": args.k, "iterations": n, "groups": s.launch_info()["groups"],
            "leader_us_per_iteration": 1000.0 * t["leader_ms"] / n,
            "column_us_per_iteration": 1000.0 * t["column_ms"] / n,
            "leader_cycles_per_iteration": {k: round(v / n) for k, v in lead.items()},
            "column_cycles_per_round": {k: round(v / rounds) for k, v in col.items()},
            "column_cycles_per_cta": per_cta,
            "column_rounds_per_cta": round(rounds / ctas, 2),
            "scatter_probe": scatter,
        }, indent=1))


if __name__ == "__main__":
    main()
