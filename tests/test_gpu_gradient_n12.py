"""Energy gradient at the scale of the gradient workload: 12 orbitals, 6 + 6
electrons (853,776 determinants, mcdfci_b200.synth "n12_6a6b", seed 0).

The solve runs with z_threshold = 0 until ||H c - E c|| / ||c|| < 1e-9
(mcd_residual), and dE/d(value of a FCIDUMP line) comes from mcd_rdm
(dE/dh_PQ = rdm1, dE/d(PR|QS) = rdm2 / 2, summed over the symmetric images a
line stands for).  Against it: central finite differences with step 1e-5 on
64 seeded lines (one- and two-electron), each perturbed FCIDUMP converged to
the same residual; the 128 perturbed solves run as two batches of 64
(mcd_batch_*).  Tolerance 1e-6 (the energies' convergence error is about
residual^2 / gap, far below step x 1e-6).  The reference has no RDMs; the
finite differences are the oracle, and the RDM kernel itself is checked
against the CPU restatement and dense RDMs in test_gpu_rdm.py.

Setting MCD_GRADIENT_REPORT=<path> writes the iterations, residuals and
every entry's two derivatives to that JSON file.
"""
import json
import os

import numpy as np
import pytest

from oracle import rdm as ordm

import mcdfci_b200 as m
from mcdfci_b200 import synth

pytestmark = pytest.mark.gpu

RESIDUAL = 1e-9
STEP = 1e-5
ENTRIES = 64
K = 32
CHUNK = 8000
MAX_ITERATIONS = 400000
OPTS = dict(num_of_coordinate=K, estimate=K, max_memory=0.1, threshold=0.0, z_threshold=0.0)


def _write_with(lines, out, line_ids, values):
    new = list(lines)
    for li, v in zip(line_ids, values):
        t = new[li].split()
        t[0] = repr(float(v))
        new[li] = " ".join(t)
    with open(out, "w") as f:
        f.write("\n".join(new))


def _converge_batch(paths):
    b = m.CDFCIBatch([m.Fcidump(p) for p in paths], **OPTS)
    b.reset()
    it = 0
    res = [1.0] * len(paths)
    while it < MAX_ITERATIONS:
        b.run_iterations(CHUNK)
        it += CHUNK
        res = [b.residual(i) for i in range(len(paths))]
        if max(res) < RESIDUAL:
            break
    # The energy of each final vector from double-double sums over its table
    # (sum x z / sum x^2), not the solve's running xz, which carries the
    # rounding of every iteration's update.
    e = []
    for i in range(len(paths)):
        t = b.table_sums(i)
        e.append(float((np.longdouble(t["xz"][0]) + np.longdouble(t["xz"][1])) /
                       (np.longdouble(t["xx"][0]) + np.longdouble(t["xx"][1]))))
    b.close()
    return e, res, it


def test_rdm_gradient_matches_finite_differences_n12(tmp_path):
    d = str(tmp_path)
    path = os.path.join(d, "n12.fcidump")
    synth.write_fcidump(path, "n12_6a6b", seed=0)
    s = m.CDFCI(m.Fcidump(path), **OPTS)
    s.reset()
    it = 0
    res = 1.0
    while it < MAX_ITERATIONS and res >= RESIDUAL:
        s.run_iterations(CHUNK)
        it += CHUNK
        res = s.residual()
    assert res < RESIDUAL, (it, res)
    e0 = s.report()["energy"]
    g1, g2 = s.rdm()
    s.close()

    lines = open(path).read().split("\n")
    start = next(i for i, l in enumerate(lines) if "&END" in l.upper()) + 1
    # integral lines: "v i j k l" with (j, k, l) not all 0 (those are orbital
    # energies and the core energy); eight one-electron lines (k = 0), the
    # rest two-electron
    body = [i for i in range(start, len(lines))
            if len(lines[i].split()) == 5 and lines[i].split()[2:] != ["0", "0", "0"]]
    one = [i for i in body if lines[i].split()[3] == "0"]
    two = [i for i in body if lines[i].split()[3] != "0"]
    rng = np.random.default_rng(17)
    ids = [int(i) for i in rng.choice(one, size=8, replace=False)] + \
          [int(i) for i in rng.choice(two, size=ENTRIES - 8, replace=False)]
    idx = [[int(v) for v in lines[i].split()[1:]] for i in ids]
    grad = [ordm.fcidump_gradient(g1, g2, *ij) for ij in idx]
    v0 = [float(lines[i].split()[0]) for i in ids]

    paths = []
    for j in range(ENTRIES):
        for sgn in (1.0, -1.0):
            p = os.path.join(d, f"fd{j}_{'p' if sgn > 0 else 'm'}.fcidump")
            _write_with(lines, p, [ids[j]], [v0[j] + sgn * STEP])
            paths.append(p)
    energies, residuals, iters = [], [], []
    for b0 in range(0, len(paths), 64):
        e, r, n = _converge_batch(paths[b0:b0 + 64])
        energies += e
        residuals += r
        iters.append(n)
    fd = [(energies[2 * j] - energies[2 * j + 1]) / (2 * STEP) for j in range(ENTRIES)]
    err = [abs(a - b) for a, b in zip(fd, grad)]
    rep = os.environ.get("MCD_GRADIENT_REPORT")
    if rep:
        with open(rep, "w") as f:
            json.dump({"workload": "n12_6a6b seed 0 (853,776 determinants)", "k": K, "energy": e0,
                       "base_iterations": it, "base_residual": res, "fd_step": STEP,
                       "fd_batch_iterations": iters, "fd_max_residual": max(residuals),
                       "max_abs_error": max(err),
                       "entries": [{"line": lines[i].split()[1:], "rdm": g, "fd": f}
                                   for i, g, f in zip(ids, grad, fd)]}, f, indent=1)
    assert max(residuals) < RESIDUAL, max(residuals)
    assert max(err) < 1e-6, max(err)
