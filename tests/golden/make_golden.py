"""Regenerate the golden fixtures in this directory from the reference itself.

Run in a container that has the reference checkout, after
``make -C oracle ref REF=<checkout>``:

    python tests/golden/make_golden.py --ref <checkout>   (or MCDFCI_REFERENCE=<checkout>)

It uses oracle/_ref/ref_dump (oracle/ref_dump.cpp compiled against the
reference headers) and oracle/_ref/cdfci_omp (the reference solver compiled
from its sources).  Outputs:

  h2o_sto3g.fcidump.gz        the reference's example FCIDUMP (example_h2o_sto3g/),
                              copied as an input fixture so GPU-side tests can run
                              without the reference checkout
  n7_5a5b.fcidump.gz          synthetic 7-orbital 5a/5b FCIDUMP (mcdfci_b200.synth, seed 0)
  n33_2a1b.fcidump.gz         synthetic 33-orbital 2a/1b FCIDUMP: 66 spin-orbitals, so the
                              reference stores each determinant in two 64-bit words
  cols_*.json.gz              get_column / get_diagonal output for a random walk of dets
  hsub_*.json.gz              get_hamiltonian_submatrix output for random det sets
  eig_*.json.gz               CoordinateUpdateEig inputs/outputs captured in real runs
  energies.json               converged energies printed by the reference solver
  trajectories.json           report energies of small-k solves (--only trajectories)

Determinants in these files use the reference layout: interleaved spin-orbital
bits (bit 2p = alpha p, bit 2p+1 = beta p) in 64-bit words, word 0 first.
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from mcdfci_b200 import synth  # noqa: E402

REF_DUMP = os.path.join(REPO, "oracle", "_ref", "ref_dump")
CDFCI = os.path.join(REPO, "oracle", "_ref", "cdfci_omp")


def gz_copy(src: str, dst: str) -> None:
    with open(src, "rb") as fi, gzip.GzipFile(dst, "wb", mtime=0) as fo:
        shutil.copyfileobj(fi, fo)


def gunzip_to(src: str, dst: str) -> None:
    with gzip.open(src, "rb") as fi, open(dst, "wb") as fo:
        shutil.copyfileobj(fi, fo)


def run(cmd, cwd=None) -> str:
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    res = subprocess.run(cmd, cwd=cwd, env=env, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"{cmd} failed ({res.returncode}):\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")
    return res.stdout


def dump(mode_args, out_name: str, tmp: str) -> None:
    out = os.path.join(tmp, out_name)
    if mode_args[0] == "eig":
        cmd = [REF_DUMP, "eig", mode_args[1], out] + mode_args[2:]
    else:
        cmd = [REF_DUMP] + mode_args + [out]
    run(cmd)
    with open(out, "rb") as fi, gzip.GzipFile(os.path.join(HERE, out_name + ".gz"), "wb", mtime=0) as fo:
        shutil.copyfileobj(fi, fo)


def final_energy(stdout: str) -> float:
    rows = [l for l in stdout.splitlines() if re.match(r"^\d+\s+-?\d+\.\d+", l)]
    return float(rows[-1].split()[1])


def report_energies(stdout: str):
    rows = [l for l in stdout.splitlines() if re.match(r"^\d+\s+-?\d+\.\d+", l)]
    return [[int(l.split()[0]), float(l.split()[1])] for l in rows]


def trajectories() -> None:
    """trajectories.json: the reference's report energies (every 250
    iterations) on the 7-orbital fixture for k = 1 (m = 1) and k = 2 (m = 4)."""
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        n7 = os.path.join(tmp, "n7.fcidump")
        gunzip_to(os.path.join(HERE, "n7_5a5b.fcidump.gz"), n7)
        for k, m in ((1, 1), (2, 4)):
            j = os.path.join(tmp, "n7_k%d.json" % k)
            write_input(j, n7, num_iterations=2000, report_interval=250, z_threshold=0,
                        z_threshold_search=False, max_memory=0.001, coordinate_pick="gcd_grad",
                        coordinate_update="eig", num_of_coordinate=k, estimate=m)
            out["n7_5a5b k%d m%d" % (k, m)] = report_energies(run([CDFCI, j]))
    with open(os.path.join(HERE, "trajectories.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(json.dumps(out, indent=1))


def write_input(path, fcidump, **kw):
    synth.write_input_json(path, fcidump, **kw)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MCDFCI_REFERENCE"),
                    help="the reference checkout (default: $MCDFCI_REFERENCE)")
    ap.add_argument("--only", choices=["all", "trajectories"], default="all")
    args = ap.parse_args()
    if args.only == "trajectories":
        return trajectories()
    if not args.ref:
        sys.exit("give the reference checkout: --ref <path> or MCDFCI_REFERENCE=<path>")
    for exe in (REF_DUMP, CDFCI):
        if not os.path.exists(exe):
            sys.exit(f"missing {exe}: run `make -C oracle ref` first")

    # Input fixtures.
    gz_copy(os.path.join(args.ref, "example_h2o_sto3g", "FCIDUMP"), os.path.join(HERE, "h2o_sto3g.fcidump.gz"))
    with tempfile.TemporaryDirectory() as tmp:
        synth.write_fcidump(os.path.join(tmp, "n7"), "n7_5a5b", seed=0)
        gz_copy(os.path.join(tmp, "n7"), os.path.join(HERE, "n7_5a5b.fcidump.gz"))
        spec33 = synth.SynthSpec(33, 2, 1, -5.0, 2.0, 0.05, 8, decay=1.0)
        synth.write_fcidump(os.path.join(tmp, "n33"), spec33, seed=3, drop_below=1e-5)
        gz_copy(os.path.join(tmp, "n33"), os.path.join(HERE, "n33_2a1b.fcidump.gz"))

        h2o = os.path.join(tmp, "h2o.fcidump")
        n7 = os.path.join(tmp, "n7.fcidump")
        n33 = os.path.join(tmp, "n33.fcidump")
        gunzip_to(os.path.join(HERE, "h2o_sto3g.fcidump.gz"), h2o)
        gunzip_to(os.path.join(HERE, "n7_5a5b.fcidump.gz"), n7)
        gunzip_to(os.path.join(HERE, "n33_2a1b.fcidump.gz"), n33)

        # Columns and diagonals.
        dump(["columns", h2o, "0.0", "1", "16"], "cols_h2o.json", tmp)
        dump(["columns", h2o, "1e-3", "2", "6"], "cols_h2o_thr1e-3.json", tmp)
        dump(["columns", n7, "0.0", "3", "32"], "cols_n7.json", tmp)
        dump(["columns", n33, "0.0", "4", "3"], "cols_n33.json", tmp)
        # Sub-matrices.
        dump(["hsub", h2o, "0.0", "5", "8", "6"], "hsub_h2o.json", tmp)
        dump(["hsub", h2o, "0.0", "6", "24", "2"], "hsub_h2o_k24.json", tmp)
        dump(["hsub", n7, "0.0", "7", "8", "6"], "hsub_n7.json", tmp)
        dump(["hsub", n33, "0.0", "8", "8", "4"], "hsub_n33.json", tmp)

        # Eig-update records inside real solves, and converged energies.
        energies = {}
        j_h2o = os.path.join(tmp, "h2o.json")
        write_input(j_h2o, h2o, num_iterations=20000, report_interval=1000, z_threshold=0,
                    z_threshold_search=False, max_memory=0.005, coordinate_pick="gcd_grad",
                    coordinate_update="eig", num_of_coordinate=8, estimate=8)
        dump(["eig", j_h2o, "0", "1", "2", "3", "4", "10", "100", "1000", "5000", "19999"], "eig_h2o.json", tmp)
        energies["h2o_sto3g k8 m8 20000it"] = final_energy(run([CDFCI, j_h2o]))

        j_n7 = os.path.join(tmp, "n7.json")
        write_input(j_n7, n7, num_iterations=1000, report_interval=250, z_threshold=0,
                    z_threshold_search=False, max_memory=0.001, coordinate_pick="gcd_grad",
                    coordinate_update="eig", num_of_coordinate=8, estimate=8)
        dump(["eig", j_n7, "0", "1", "2", "3", "50", "500"], "eig_n7.json", tmp)
        energies["n7_5a5b seed0 k8 m8 1000it"] = final_energy(run([CDFCI, j_n7]))

        j_h2o_zt = os.path.join(tmp, "h2o_zt.json")
        write_input(j_h2o_zt, h2o, num_iterations=20000, report_interval=1000, z_threshold=1e-5,
                    z_threshold_search=False, max_memory=0.005, coordinate_pick="gcd_grad",
                    coordinate_update="eig", num_of_coordinate=8, estimate=8)
        energies["h2o_sto3g k8 m8 20000it z_threshold=1e-5"] = final_energy(run([CDFCI, j_h2o_zt]))

        j_h2o_k4 = os.path.join(tmp, "h2o_k4.json")
        write_input(j_h2o_k4, h2o, num_iterations=40000, report_interval=1000, z_threshold=0,
                    z_threshold_search=False, max_memory=0.005, coordinate_pick="gcd_grad",
                    coordinate_update="eig", num_of_coordinate=4, estimate=6)
        energies["h2o_sto3g k4 m6 40000it"] = final_energy(run([CDFCI, j_h2o_k4]))

    with open(os.path.join(HERE, "energies.json"), "w") as f:
        json.dump(energies, f, indent=2, sort_keys=True)
        f.write("\n")
    print(json.dumps(energies, indent=2))


if __name__ == "__main__":
    main()
