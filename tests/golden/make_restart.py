"""Fixture for the z_threshold_search restart, from the reference itself.

Runs oracle/_ref/cdfci_omp (the reference solver compiled from its sources by
``make -C oracle ref REF=<checkout>``) on the H2O example FCIDUMP kept in this
directory with z_threshold_search on, and records what it printed:

    python tests/golden/make_restart.py

Settings: k = m = 8, report_interval 1000 (the reference's minimum with the
search on, src/run_wrapper.h:117-120), max_memory 0.002 GB (2^16 slots, so
max_wavefunction_size = 51,773 and the restart window 0.7 * 51,773 < |z| at a
report, src/solver.h:802-809), starting z_threshold 7e-5.  At iteration 1000
|z| = 38,518 lies in that window, the reference restarts once with
z_threshold 1.4e-4 (src/solver.h:882-888) and then runs to the end.  Starting
values from 6e-5 to 8e-5 and 2, 4 or 8 OpenMP threads give the same single
restart (|z| at iteration 1000 between 36.9k and 40.3k), so the case is not on
an edge.

Output: restart_h2o.json with the deck, the restarts (iteration, |z|, new
z_threshold), the report table after the last restart (iteration, energy,
|x|, |z|) and the final energy.
"""
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
CDFCI = os.path.join(REPO, "oracle", "_ref", "cdfci_omp")

DECK = {"num_iterations": 20000, "report_interval": 1000, "z_threshold": 7e-5, "z_threshold_search": True,
        "max_memory": 0.002, "coordinate_pick": "gcd_grad", "coordinate_update": "eig",
        "num_of_coordinate": 8, "estimate": 8}


def parse(out: str):
    restarts, tables, cur = [], [], []
    for line in out.splitlines():
        m = re.search(r"Increase z_threhold to ([0-9.eE+-]+)", line)
        if m:
            restarts.append({"at_iteration": cur[-1]["iteration"] if cur else None,
                             "z_size": cur[-1]["z_size"] if cur else None,
                             "new_z_threshold": float(m.group(1))})
            tables.append(cur)
            cur = []
            continue
        p = line.split()
        if len(p) >= 9 and re.match(r"^\d+$", p[0]) and re.match(r"^-?\d+\.\d+$", p[1]):
            cur.append({"iteration": int(p[0]), "energy": float(p[1]), "x_size": int(p[3]), "z_size": int(p[4])})
    tables.append(cur)
    return restarts, tables


def main():
    if not os.path.exists(CDFCI):
        sys.exit(f"missing {CDFCI}: run `make -C oracle ref REF=<checkout>` first")
    with tempfile.TemporaryDirectory() as d:
        fcidump = os.path.join(d, "FCIDUMP")
        with gzip.open(os.path.join(HERE, "h2o_sto3g.fcidump.gz"), "rb") as fi, open(fcidump, "wb") as fo:
            shutil.copyfileobj(fi, fo)
        deck = os.path.join(d, "input.json")
        with open(deck, "w") as f:
            json.dump({"hamiltonian": {"fcidump_path": fcidump, "threshold": 0.0}, "solver": {"cdfci": DECK}}, f)
        env = dict(os.environ, OMP_NUM_THREADS="8", OPENBLAS_NUM_THREADS="1")
        res = subprocess.run([CDFCI, deck], capture_output=True, text=True, env=env, check=True)
    restarts, tables = parse(res.stdout)
    final = tables[-1]
    out = {"fcidump": "h2o_sto3g.fcidump.gz", "threshold": 0.0, "deck": DECK, "restarts": restarts,
           "reports_before_restart": tables[:-1], "reports": final, "energy": final[-1]["energy"],
           "source": "oracle/_ref/cdfci_omp, OMP_NUM_THREADS=8, OPENBLAS_NUM_THREADS=1"}
    with open(os.path.join(HERE, "restart_h2o.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps({"restarts": restarts, "energy": out["energy"]}))


if __name__ == "__main__":
    main()
