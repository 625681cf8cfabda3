"""Several instances in one batch (mcd_batch_*): each instance of uneven size
converges to its own dense FP64 ground-state energy (1e-8 Ha), H2O to the
reference's energy (1e-6 Ha), and an instance in a batch ends where it ends
when solved alone (1e-9 Ha, both converged)."""
import os
from itertools import combinations

import numpy as np
import pytest

from conftest import load_golden
from oracle.oracle import Oracle

import mcdfci_b200 as m
from mcdfci_b200 import synth

pytestmark = pytest.mark.gpu

ENERGIES = load_golden("energies.json")
SMALL_6 = synth.SynthSpec(6, 3, 3, -20.0, 1.0, 0.1, 12)   # 400 determinants
OPEN_8 = synth.SynthSpec(8, 4, 3, -20.0, 1.0, 0.1, 16)    # 3920 determinants, ms2 = 1


def _dense(path, norb, na, nb):
    o = Oracle(path, 0.0)
    dets = [(sum(1 << p for p in a), sum(1 << p for p in b)) for a in combinations(range(norb), na)
            for b in combinations(range(norb), nb)]
    idx = {d: i for i, d in enumerate(dets)}
    H = np.zeros((len(dets), len(dets)))
    for d in dets:
        cd, cv = o.column_ab(*d)
        for e, v in zip(cd, cv):
            H[idx[e], idx[d]] = v
    return np.linalg.eigvalsh(H)[0]


@pytest.fixture(scope="module")
def batch_paths(tmp_path_factory, fcidumps):
    d = tmp_path_factory.mktemp("batch")
    p6 = os.path.join(str(d), "small6.fcidump")
    p8 = os.path.join(str(d), "open8.fcidump")
    synth.write_fcidump(p6, SMALL_6, seed=1)
    synth.write_fcidump(p8, OPEN_8, seed=2)
    return [fcidumps["n7_5a5b"], fcidumps["h2o_sto3g"], p6, p8]


OPTS = dict(num_of_coordinate=8, estimate=8, max_memory=0.005, threshold=0.0, num_iterations=20000,
            report_interval=5000)


def test_batch_uneven_instances_match_dense(batch_paths):
    b = m.CDFCIBatch([m.Fcidump(p) for p in batch_paths], **OPTS)
    e = b.solve()
    assert len(e) == 4
    assert abs(e[0] - _dense(batch_paths[0], 7, 5, 5)) < 1e-8
    assert abs(e[1] - ENERGIES["h2o_sto3g k8 m8 20000it"]) < 1e-6
    assert abs(e[2] - _dense(batch_paths[2], 6, 3, 3)) < 1e-8
    assert abs(e[3] - _dense(batch_paths[3], 8, 4, 3)) < 1e-8
    # Reports: one per instance per interval, in iteration order.
    for reps in b.reports:
        assert [r["iteration"] for r in reps] == [5000, 10000, 15000, 20000]


def test_batch_instance_matches_single_solve(batch_paths):
    b = m.CDFCIBatch([m.Fcidump(p) for p in batch_paths], **OPTS)
    eb = b.solve()
    for i in (0, 3):
        s = m.CDFCI(m.Fcidump(batch_paths[i]), **OPTS)
        assert abs(s.solve() - eb[i]) < 1e-9


def test_batch_of_one_and_report(batch_paths):
    b = m.CDFCIBatch([m.Fcidump(batch_paths[0])], **OPTS)
    b.reset()
    b.run_iterations(3000)
    r = b.report(0)
    assert r["iteration"] == 3000
    assert abs(r["energy"] - _dense(batch_paths[0], 7, 5, 5)) < 1e-8


def test_batch_callback_stops(batch_paths):
    b = m.CDFCIBatch([m.Fcidump(p) for p in batch_paths[:2]], **OPTS)
    seen = []
    b.solve(callback=lambda i, r: seen.append((i, r["iteration"])) or r["iteration"] >= 10000)
    assert seen == [(0, 5000), (1, 5000), (0, 10000), (1, 10000)]


def test_batch_retires_instances(batch_paths):
    """An instance retired by the callback (MCD_CB_RETIRE) stops advancing and
    keeps its energy; the others run on without it, to the energies they
    reach in the full batch, and the solve ends when none is left."""
    b = m.CDFCIBatch([m.Fcidump(p) for p in batch_paths], **OPTS)
    full = b.solve()
    b.close()
    b = m.CDFCIBatch([m.Fcidump(p) for p in batch_paths], **OPTS)
    retire_at = {0: 5000, 2: 10000, 1: 15000, 3: 20000}
    e = b.solve(callback=lambda i, r: "retire" if r["iteration"] >= retire_at[i] else False)
    for i, reps in enumerate(b.reports):
        assert [r["iteration"] for r in reps] == list(range(5000, retire_at[i] + 1, 5000)), i
        assert e[i] == reps[-1]["energy"]
    assert abs(e[3] - full[3]) < 1e-9
    assert abs(e[1] - full[1]) < 1e-6
    b.close()
