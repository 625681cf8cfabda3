"""Checkpoint / restart (mcd_checkpoint_save / mcd_checkpoint_load): a solve
stopped, saved, loaded into a new solver (with a different table size) and
continued ends where the uninterrupted solve ends, and a checkpoint of another
problem is refused."""
import os

import pytest

import mcdfci_b200 as m

pytestmark = pytest.mark.gpu

OPTS = dict(num_of_coordinate=8, estimate=8, threshold=0.0)


def test_restart_continues_the_solve(fcidumps, tmp_path):
    path = fcidumps["h2o_sto3g"]
    ck = os.path.join(str(tmp_path), "h2o.ckpt")
    a = m.CDFCI(m.Fcidump(path), max_memory=0.005, **OPTS)
    a.reset()
    a.run_iterations(3000)
    r_mid = a.report()
    a.save(ck)
    a.run_iterations(2000)
    r_a = a.report()
    b = m.CDFCI(m.Fcidump(path), max_memory=0.01, **OPTS)
    b.load(ck)
    r_b0 = b.report()
    assert r_b0["iteration"] == r_mid["iteration"]
    assert r_b0["energy"] == r_mid["energy"]
    assert (r_b0["x_size"], r_b0["z_size"]) == (r_mid["x_size"], r_mid["z_size"])
    b.run_iterations(2000)
    r_b = b.report()
    assert r_b["iteration"] == r_a["iteration"]
    assert abs(r_b["energy"] - r_a["energy"]) < 1e-9
    assert b.table_sums()["occupied"] == a.table_sums()["occupied"]


def test_checkpoint_of_another_problem_is_refused(fcidumps, tmp_path):
    ck = os.path.join(str(tmp_path), "n7.ckpt")
    a = m.CDFCI(m.Fcidump(fcidumps["n7_5a5b"]), max_memory=0.005, **OPTS)
    a.reset()
    a.run_iterations(10)
    a.save(ck)
    b = m.CDFCI(m.Fcidump(fcidumps["h2o_sto3g"]), max_memory=0.005, **OPTS)
    with pytest.raises(m.McdError) as e:
        b.load(ck)
    assert e.value.code == m.MCD_ERR_INVALID
