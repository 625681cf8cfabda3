"""RDMs on the GPU (mcd_rdm) and the energy gradient they give.

- Parity: the GPU RDMs of the converged wavefunction equal the CPU
  restatement's (oracle/rdm.py, explicit fermionic operators) computed from the
  same exported coefficients, to 1e-12.
- The energy from the RDMs equals the solver's energy (1e-9 Ha), and the RDMs
  of the converged vector equal those of the dense FP64 ground state (1e-5).
- Gradient: a torch.autograd.Function defined here, in the test harness only,
  whose forward solves the FCIDUMP with some line values replaced and whose
  backward returns dE/d(line values) from mcd_rdm, matches central finite
  differences (step 1e-5) of converged energies to 1e-6.
"""
import os

import numpy as np
import pytest
import torch

from oracle import rdm as ordm
from oracle.oracle import Oracle

import mcdfci_b200 as m

pytestmark = pytest.mark.gpu

NORB, NA, NB = 7, 5, 5
OPTS = dict(num_of_coordinate=8, estimate=8, max_memory=0.001, threshold=0.0, num_iterations=12000,
            report_interval=4000)


def _solve(path):
    s = m.CDFCI(m.Fcidump(path), **OPTS)
    e = s.solve()
    return s, e


@pytest.fixture(scope="module")
def n7(fcidumps):
    path = fcidumps["n7_5a5b"]
    s, e = _solve(path)
    g1, g2 = s.rdm()
    a, b, x = s.wavefunction()
    return path, s, e, g1, g2, a, b, x


def test_rdm_matches_cpu_restatement_on_same_vector(n7):
    path, s, e, g1, g2, a, b, x = n7
    dets = [(int(p), int(q)) for p, q in zip(a, b)]
    gamma, Gamma = ordm.rdms(NORB, dets, x)
    c1, c2 = ordm.spin_summed(gamma, Gamma)
    assert np.max(np.abs(g1 - c1)) < 1e-12
    assert np.max(np.abs(g2 - c2)) < 1e-12


def test_rdm_energy_and_traces(n7):
    path, s, e, g1, g2, a, b, x = n7
    n, ne, ms2, h, eri, ecore = ordm.read_fcidump(path)
    assert abs(ordm.energy(h, eri, ecore, g1, g2) - e) < 1e-9
    assert abs(np.trace(g1) - ne) < 1e-12
    assert abs(np.einsum("pqpq", g2) - ne * (ne - 1)) < 1e-10
    assert np.max(np.abs(g1 - g1.T)) < 1e-12


def test_rdm_matches_dense_ground_state(n7):
    path, s, e, g1, g2, a, b, x = n7
    o = Oracle(path, 0.0)
    dets = ordm.determinants(NORB, NA, NB)
    idx = {d: i for i, d in enumerate(dets)}
    H = np.zeros((len(dets), len(dets)))
    for d in dets:
        cd, cv = o.column_ab(*d)
        for f, v in zip(cd, cv):
            H[idx[f], idx[d]] = v
    w, V = np.linalg.eigh(H)
    assert abs(w[0] - e) < 1e-9
    c1, c2 = ordm.spin_summed(*ordm.rdms(NORB, dets, V[:, 0]))
    assert np.max(np.abs(g1 - c1)) < 1e-5
    assert np.max(np.abs(g2 - c2)) < 1e-5


# ---------------------------------------------------------------------------
# The gradient as an autograd function (test harness only).

def _write_with(path, out, line_ids, values):
    lines = open(path).read().split("\n")
    for li, v in zip(line_ids, values):
        t = lines[li].split()
        t[0] = repr(float(v))
        lines[li] = " ".join(t)
    with open(out, "w") as f:
        f.write("\n".join(lines))


class FcidumpEnergy(torch.autograd.Function):
    """E(values of some FCIDUMP lines); backward from mcd_rdm."""

    @staticmethod
    def forward(ctx, values, path, out, line_ids, indices):
        _write_with(path, out, line_ids, values.tolist())
        s, e = _solve(out)
        g1, g2 = s.rdm()
        grads = [ordm.fcidump_gradient(g1, g2, *ij) for ij in indices]
        ctx.save_for_backward(torch.tensor(grads, dtype=torch.float64))
        return torch.tensor(e, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None, None


def test_gradient_matches_finite_differences(fcidumps, tmp_path):
    path = fcidumps["n7_5a5b"]
    lines = open(path).read().split("\n")
    start = next(i for i, l in enumerate(lines) if "&END" in l.upper()) + 1
    body = [i for i in range(start, len(lines))
            if len(lines[i].split()) == 5 and lines[i].split()[2:] != ["0", "0", "0"]]
    rng = np.random.default_rng(11)
    ids = [int(i) for i in rng.choice(body, size=6, replace=False)]
    indices = [[int(v) for v in lines[i].split()[1:]] for i in ids]
    v0 = torch.tensor([float(lines[i].split()[0]) for i in ids], dtype=torch.float64, requires_grad=True)
    out = os.path.join(str(tmp_path), "x.fcidump")
    e = FcidumpEnergy.apply(v0, path, out, ids, indices)
    e.backward()
    h = 1e-5
    for j in range(len(ids)):
        vp = v0.detach().clone()
        vm = v0.detach().clone()
        vp[j] += h
        vm[j] -= h
        _write_with(path, out, ids, vp.tolist())
        ep = _solve(out)[1]
        _write_with(path, out, ids, vm.tolist())
        em = _solve(out)[1]
        fd = (ep - em) / (2 * h)
        assert abs(fd - float(v0.grad[j])) < 1e-6, (lines[ids[j]], fd, float(v0.grad[j]))


def test_rdm_energy_identity_n12(synth_fcidumps):
    """The gradient workload (12 orbitals, 6 + 6 electrons, 853,776
    determinants): after 3000 iterations the RDMs of the current vector give
    the solver's energy (with z_threshold = 0 both are its Rayleigh quotient)."""
    path = synth_fcidumps["n12_6a6b"]
    s = m.CDFCI(m.Fcidump(path), num_of_coordinate=32, estimate=32, max_memory=1.0, threshold=0.0,
                z_threshold=0.0)
    s.reset()
    s.run_iterations(3000)
    e = s.report()["energy"]
    g1, g2 = s.rdm()
    n, ne, ms2, h, eri, ecore = ordm.read_fcidump(path)
    assert abs(ordm.energy(h, eri, ecore, g1, g2) - e) < 1e-8
    assert abs(np.trace(g1) - ne) < 1e-10
