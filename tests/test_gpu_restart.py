"""z_threshold_search restarts against the reference's own run.

The fixture (tests/golden/restart_h2o.json, made by make_restart.py from the
reference compiled from its sources) is the H2O example with the search on,
max_memory 0.002 GB and a starting z_threshold of 7e-5: at the report of
iteration 1000 |z| lies between 0.7 and 0.79 of max_wavefunction_size and
has grown by more than one entry per candidate per 1000 iterations, so the
reference restarts with twice the threshold (src/solver.h:802-809,882-888) and
then converges.  The GPU solve must take the same restarts at the same
report with the same thresholds, keep |z| within 3 % of the reference's at
every report, and end within 1e-6 Ha of the reference's energy.
"""
import pytest

import mcdfci_b200 as m
from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_restart_sequence_and_energy_match_reference(fcidumps):
    g = load_golden("restart_h2o.json")
    d = g["deck"]
    s = m.CDFCI(m.Fcidump(fcidumps["h2o_sto3g"]), threshold=g["threshold"], num_iterations=d["num_iterations"],
                report_interval=d["report_interval"], z_threshold=d["z_threshold"], z_threshold_search=True,
                max_memory=d["max_memory"], num_of_coordinate=d["num_of_coordinate"], estimate=d["estimate"])
    e = s.solve()
    reps = s.reports
    s.close()
    # Split the report table at the restarts (the iteration count starts over).
    runs, cur = [], []
    for r in reps:
        if cur and r["iteration"] <= cur[-1]["iteration"]:
            runs.append(cur)
            cur = []
        cur.append(r)
    runs.append(cur)
    assert len(runs) == len(g["restarts"]) + 1
    zt = d["z_threshold"]
    for run, rs in zip(runs[:-1], g["restarts"]):
        assert run[-1]["iteration"] == rs["at_iteration"]
        assert abs(run[-1]["z_size"] - rs["z_size"]) <= 0.03 * rs["z_size"]
        assert run[0]["z_threshold"] == pytest.approx(zt, rel=1e-12)
        zt = rs["new_z_threshold"]
    last = runs[-1]
    assert last[0]["z_threshold"] == pytest.approx(zt, rel=1e-12)
    assert [r["iteration"] for r in last] == [r["iteration"] for r in g["reports"]]
    for mine, ref in zip(last, g["reports"]):
        assert abs(mine["z_size"] - ref["z_size"]) <= 0.03 * ref["z_size"], (mine["iteration"], mine["z_size"])
    assert abs(e - g["energy"]) < 1e-6
