"""The CPU RDM restatement (oracle/rdm.py) pinned on the 441-determinant
case: the energy from its RDMs equals the dense ground-state energy of the
Hamiltonian the reference's column generation defines (oracle columns,
bit-exact with the reference's), and its integral gradients equal central
finite differences of that dense energy (Hellmann-Feynman)."""
import os
import shutil

import numpy as np
import pytest

from oracle import rdm
from oracle.oracle import Oracle

NORB, NA, NB = 7, 5, 5


def _dense(path):
    o = Oracle(path, 0.0)
    dets = rdm.determinants(NORB, NA, NB)
    idx = {d: i for i, d in enumerate(dets)}
    H = np.zeros((len(dets), len(dets)))
    for d in dets:
        cd, cv = o.column_ab(*d)
        for e, v in zip(cd, cv):
            H[idx[e], idx[d]] = v
    w, V = np.linalg.eigh(H)
    return dets, w[0], V[:, 0]


@pytest.fixture(scope="module")
def n7(fcidumps):
    dets, e0, c = _dense(fcidumps["n7_5a5b"])
    gamma, Gamma = rdm.rdms(NORB, dets, c)
    g1, g2 = rdm.spin_summed(gamma, Gamma)
    return fcidumps["n7_5a5b"], e0, g1, g2


def test_rdm_energy_equals_dense(n7):
    path, e0, g1, g2 = n7
    n, ne, ms2, h, eri, ecore = rdm.read_fcidump(path)
    assert abs(rdm.energy(h, eri, ecore, g1, g2) - e0) < 1e-10
    assert abs(np.trace(g1) - ne) < 1e-12
    assert abs(np.einsum("pqpq", g2) - ne * (ne - 1)) < 1e-10


def _perturbed(path, tmpdir, line_idx, delta):
    lines = open(path).read().split("\n")
    t = lines[line_idx].split()
    t[0] = repr(float(t[0].replace("D", "E")) + delta)
    lines[line_idx] = " ".join(t)
    out = os.path.join(str(tmpdir), "pert.fcidump")
    with open(out, "w") as f:
        f.write("\n".join(lines))
    return out


def test_rdm_gradient_equals_finite_differences(n7, tmp_path):
    path, e0, g1, g2 = n7
    lines = open(path).read().split("\n")
    start = next(i for i, l in enumerate(lines) if "&END" in l.upper() or l.strip() == "/") + 1
    body = [i for i in range(start, len(lines)) if len(lines[i].split()) == 5]
    rng = np.random.default_rng(3)
    picks = list(rng.choice(body[:-1], size=16, replace=False))
    h = 1e-5
    for li in picks:
        t = lines[li].split()
        ij = [int(x) for x in t[1:]]
        if ij[1:] == [0, 0, 0]:
            continue  # core or orbital energy
        _, ep, _ = _dense(_perturbed(path, tmp_path, li, +h))
        _, em, _ = _dense(_perturbed(path, tmp_path, li, -h))
        fd = (ep - em) / (2 * h)
        an = rdm.fcidump_gradient(g1, g2, *ij)
        assert abs(fd - an) < 1e-6, (lines[li], fd, an)
