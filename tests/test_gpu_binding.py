"""The reference-side binding, compiled: oracle/run_cdfci_gpu.cpp is the
run_cdfci_gpu a maintainer adds to the reference's src/run_wrapper.h,
built against the reference's own headers (its Option, read_input,
check_argument) and linked with libmcdfci.so.  Run on the reference's H2O
example deck, it prints the report table and ends at the reference's energy
(1e-6 Ha); a deck the reference rejects is rejected the same way."""
import json
import os
import subprocess

import pytest

from conftest import REPO, load_golden

pytestmark = pytest.mark.gpu

EXE = os.path.join(REPO, "oracle", "_ref", "run_cdfci_gpu")


def _deck(tmp_path, fcidump, **cdfci):
    d = {"num_iterations": 20000, "report_interval": 1000, "z_threshold": 0, "z_threshold_search": False,
         "max_memory": 0.005, "coordinate_pick": "gcd_grad", "coordinate_update": "eig",
         "num_of_coordinate": 8, "estimate": 8}
    d.update(cdfci)
    p = os.path.join(str(tmp_path), "input.json")
    with open(p, "w") as f:
        json.dump({"hamiltonian": {"fcidump_path": fcidump, "threshold": 0.0}, "solver": {"cdfci": d}}, f)
    return p


@pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/run_cdfci_gpu is built with the reference checkout")
def test_binding_runs_reference_deck(fcidumps, tmp_path):
    res = subprocess.run([EXE, _deck(tmp_path, fcidumps["h2o_sto3g"])], capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.split() and l.split()[0].isdigit() and "." in l]
    assert len(lines) == 20
    e = float(res.stdout.split("run_cdfci_gpu energy:")[1].split()[0])
    assert abs(e - load_golden("energies.json")["h2o_sto3g k8 m8 20000it"]) < 1e-6


@pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/run_cdfci_gpu is built with the reference checkout")
def test_binding_rejects_what_the_reference_rejects(fcidumps, tmp_path):
    # z_threshold_search needs report_interval >= 1000 (src/run_wrapper.h:117-120)
    res = subprocess.run([EXE, _deck(tmp_path, fcidumps["h2o_sto3g"], z_threshold_search=True, report_interval=10)],
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 1
    assert "report_interval >= 1000" in res.stderr
