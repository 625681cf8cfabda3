"""Reference energies of the 32-point dissociation curve, from the reference.

Each point is the synthetic 16-orbital, 5 + 5 electron FCIDUMP of
mcdfci_b200.synth ("n16_5a5b", seed 0) at t = i/31, i = 0..31 (integrals
interpolated between two endpoints, the second with its off-diagonal
couplings scaled x3).  The reference solves a curve one point after another
(experiments/4.4-binding-curve/dissociation.sh:2-9); this script does the
same with oracle/_ref/cdfci_omp (the reference compiled from its sources by
``make -C oracle ref REF=<checkout>``):

    python tests/golden/make_curve.py [--iterations 60000] [--jobs 2] [--threads 4]

Deck per point: gcd_grad, eig, num_of_coordinate = estimate = 16 (the
reference lowers k to its host's processor count; the effective k is
recorded), max_memory 1 GB, z_threshold 0, hamiltonian threshold 0, report
every 1000 iterations.  Output: curve_energies.json, one record per point with
t, the effective k, the iterations, the energy of every report and the last
one.  On some points the reference stops before its last iteration: its
inverse-iteration refinement prints "Factorization fails!" and exits with
status 255 (src/solver.h:444-450).  Such a point is recorded with
"failed" (the message and the exit status), the reports it printed, and
"energy" = its last reported energy (null when it printed none).
Points are written as they finish, so an interrupted run keeps what it did;
a rerun skips the points already recorded with the same settings.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from mcdfci_b200 import synth  # noqa: E402

CDFCI = os.path.join(REPO, "oracle", "_ref", "cdfci_omp")
OUT = os.path.join(HERE, "curve_energies.json")
POINTS = 32
WORKLOAD = "n16_5a5b"


def run_point(i, iterations, threads, report):
    t = i / (POINTS - 1)
    with tempfile.TemporaryDirectory() as d:
        fcidump = os.path.join(d, "FCIDUMP")
        synth.write_fcidump(fcidump, WORKLOAD, seed=0, t=t)
        deck = os.path.join(d, "input.json")
        with open(deck, "w") as f:
            json.dump({"hamiltonian": {"fcidump_path": fcidump, "threshold": 0.0},
                       "solver": {"cdfci": {"num_iterations": iterations, "report_interval": report,
                                            "z_threshold": 0.0, "z_threshold_search": False, "max_memory": 1.0,
                                            "coordinate_pick": "gcd_grad", "coordinate_update": "eig",
                                            "num_of_coordinate": 16, "estimate": 16}}}, f)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
        res = subprocess.run([CDFCI, deck], capture_output=True, text=True, env=env)
    failed = None
    if res.returncode != 0:
        msg = [ln.strip() for ln in (res.stdout + res.stderr).splitlines() if "fail" in ln.lower()]
        if not msg:
            raise RuntimeError(f"point {i}: the reference exited with status {res.returncode}:\n{res.stdout[-2000:]}")
        failed = {"message": msg[-1], "exit_status": res.returncode}
    k_eff = 16
    m = re.search(r"Not enough processes\. Set k = (\d+)", res.stdout)
    if m:
        k_eff = int(m.group(1))
    reports = []
    for line in res.stdout.splitlines():
        p = line.split()
        if len(p) >= 9 and re.match(r"^\d+$", p[0]) and re.match(r"^-?\d+\.\d+$", p[1]):
            reports.append({"iteration": int(p[0]), "energy": float(p[1]), "z_size": int(p[4]),
                            "time_s": float(p[7])})
    rec = {"point": i, "t": t, "k": k_eff, "iterations": iterations, "report_interval": report, "reports": reports,
           "energy": reports[-1]["energy"] if reports else None}
    if failed:
        rec["failed"] = failed
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=60000)
    ap.add_argument("--report", type=int, default=1000)
    ap.add_argument("--jobs", type=int, default=2)
    ap.add_argument("--threads", type=int, default=4)
    ap.add_argument("--points", type=int, nargs="*", default=list(range(POINTS)))
    args = ap.parse_args()
    if not os.path.exists(CDFCI):
        sys.exit(f"missing {CDFCI}: run `make -C oracle ref REF=<checkout>` first")
    data = {"workload": f"{POINTS} x {WORKLOAD} (mcdfci_b200.synth, seed 0, t = i/{POINTS - 1})",
            "deck": {"num_of_coordinate": 16, "estimate": 16, "max_memory": 1.0, "z_threshold": 0.0,
                     "threshold": 0.0, "report_interval": args.report},
            "source": "oracle/_ref/cdfci_omp, OPENBLAS_NUM_THREADS=1", "points": []}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data["deck"]["report_interval"] = args.report
    data["points"] = [p for p in data["points"]
                      if p["iterations"] == args.iterations and p.get("report_interval") == args.report]
    done = {p["point"] for p in data["points"]}
    todo = [i for i in args.points if i not in done]

    def save():
        data["points"].sort(key=lambda p: p["point"])
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)
            f.write("\n")

    with ThreadPoolExecutor(max_workers=args.jobs) as ex:
        futs = {ex.submit(run_point, i, args.iterations, args.threads, args.report): i for i in todo}
        for fu in futs:
            rec = fu.result()
            data["points"] = [p for p in data["points"] if p["point"] != rec["point"]] + [rec]
            save()
            print(json.dumps({"point": rec["point"], "energy": rec["energy"], "k": rec["k"],
                              "failed": rec.get("failed")}), flush=True)
    save()


if __name__ == "__main__":
    main()
