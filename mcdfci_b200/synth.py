"""Seeded synthetic FCIDUMP generator for the benchmark and parity workloads.

There is no public benchmark suite for this path; the workloads are synthetic
molecular-like Hamiltonians with the shapes and value distributions below.

* ``h1`` is symmetric: diagonal ~ U[diag_lo, diag_hi], off-diagonal ~ N(0, off_sigma).
* ``eri[p,q,r,s] = sum_P L[P,p,q] * L[P,r,s]`` (chemists' notation (pq|rs)), with
  each ``L[P]`` symmetric, N(0, chol_sigma) scaled by ``exp(-|p-q|/decay)``.  The
  tensor therefore has the 8-fold permutational symmetry of real orbitals and is
  positive semi-definite as a (pq),(rs) matrix.
* The FCIDUMP holds the 8-fold-unique two-electron entries, the lower triangle
  of ``h1``, orbital energies equal to the ``h1`` diagonal (so the Hartree-Fock
  determinant fills the lowest diagonal entries), and the core energy last.
* The solver needs a negative ground-state energy (it takes sqrt(-lambda) of the
  subspace eigenvalue).  If the Hartree-Fock energy with the nominal core energy
  is not below -1 Ha, the core energy is lowered to ``-E_HF(no core) - 50``.

Every array is drawn from ``numpy.random.default_rng(seed)`` (PCG64, stable
across numpy versions) in a fixed order, so a (workload, seed) pair always
produces the same FCIDUMP bytes.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, Optional

import numpy as np


@dataclasses.dataclass(frozen=True)
class SynthSpec:
    norb: int
    nalpha: int
    nbeta: int
    diag_lo: float
    diag_hi: float
    off_sigma: float
    nchol: int
    chol_sigma: float = 0.3
    decay: float = 3.0
    ecore: float = 9.0

    @property
    def nelec(self) -> int:
        return self.nalpha + self.nbeta

    @property
    def ms2(self) -> int:
        return self.nalpha - self.nbeta


# Workloads, named by what they are.
SPECS: Dict[str, SynthSpec] = {
    # 441 determinants; small enough for dense FP64 diagonalisation.
    "n7_5a5b": SynthSpec(7, 5, 5, -20.0, 1.0, 0.1, 14),
    # ~1.8e10 determinants; the single-GPU throughput workload.
    "n24_6a6b": SynthSpec(24, 6, 6, -5.0, 2.0, 0.05, 48),
    # ~1.9e7 determinants per point of the dissociation curve.
    "n16_5a5b": SynthSpec(16, 5, 5, -20.0, 1.0, 0.1, 32),
    # ~8.5e5 determinants; the energy-gradient workload.
    "n12_6a6b": SynthSpec(12, 6, 6, -20.0, 1.0, 0.1, 24),
    # 42 orbitals, 48 electrons; needs alpha/beta strings wider than 32 bits.
    "n42_24a24b": SynthSpec(42, 24, 24, -3.0, 1.0, 0.08, 84, decay=6.0),
}


def _draw(spec: SynthSpec, rng: np.random.Generator, off_scale: float = 1.0):
    n = spec.norb
    h1 = np.zeros((n, n))
    diag = rng.uniform(spec.diag_lo, spec.diag_hi, size=n)
    off = rng.normal(0.0, spec.off_sigma, size=(n, n))
    off = np.triu(off, 1)
    h1 = off + off.T
    h1 *= off_scale
    h1[np.diag_indices(n)] = diag
    idx = np.arange(n)
    decay = np.exp(-np.abs(idx[:, None] - idx[None, :]) / spec.decay)
    L = rng.normal(0.0, spec.chol_sigma, size=(spec.nchol, n, n))
    L = np.triu(L)
    L = L + np.transpose(np.triu(L, 1), (0, 2, 1))
    L = L * decay[None]
    if off_scale != 1.0:
        offmask = ~np.eye(n, dtype=bool)
        L[:, offmask] *= off_scale
    eri = np.einsum("Ppq,Prs->pqrs", L, L, optimize=True)
    return h1, eri


def hf_energy(h1: np.ndarray, eri: np.ndarray, nalpha: int, nbeta: int) -> float:
    """Energy of the determinant filling the lowest ``h1`` diagonal orbitals
    (no core energy): sum h_ii + sum_{i<j} <ij||ij> over spin-orbitals."""
    order = np.argsort(np.diag(h1), kind="stable")
    occa, occb = order[:nalpha], order[:nbeta]
    e = h1[occa, occa].sum() + h1[occb, occb].sum()
    J = np.einsum("iijj->ij", eri)
    K = np.einsum("ijji->ij", eri)
    e += 0.5 * (J[np.ix_(occa, occa)].sum() - K[np.ix_(occa, occa)].sum())
    e += 0.5 * (J[np.ix_(occb, occb)].sum() - K[np.ix_(occb, occb)].sum())
    e += J[np.ix_(occa, occb)].sum()
    return float(e)


def make_integrals(name_or_spec, seed: int = 0, t: Optional[float] = None):
    """Return (spec, h1, eri, ecore).  ``t`` in [0,1] selects a point on the
    dissociation curve between endpoint A (seed) and endpoint B (seed+1000,
    off-diagonal couplings x3): h(t) = (1-t) h_A + t h_B, eri likewise."""
    spec = SPECS[name_or_spec] if isinstance(name_or_spec, str) else name_or_spec
    rng = np.random.default_rng(seed)
    h1, eri = _draw(spec, rng)
    if t is not None:
        rng_b = np.random.default_rng(seed + 1000)
        h1b, erib = _draw(spec, rng_b, off_scale=3.0)
        h1 = (1.0 - t) * h1 + t * h1b
        eri = (1.0 - t) * eri + t * erib
    ecore = spec.ecore
    ehf = hf_energy(h1, eri, spec.nalpha, spec.nbeta)
    if ehf + ecore > -1.0:
        ecore = float(np.floor(-ehf - 50.0))
    return spec, h1, eri, ecore


def fcidump_text(spec: SynthSpec, h1: np.ndarray, eri: np.ndarray, ecore: float,
                 drop_below: float = 0.0) -> str:
    """FCIDUMP text.  Two-electron entries with |value| <= ``drop_below`` are
    left out (absent entries read as zero); the default keeps every entry."""
    n = spec.norb
    lines = [
        f"&FCI NORB={n},NELEC={spec.nelec},MS2={spec.ms2},",
        " ORBSYM=" + ",".join(["1"] * n) + ",",
        " ISYM=1,",
        " UHF=.FALSE.,",
        "&END",
    ]
    out = []
    for i in range(n):
        for j in range(i + 1):
            ij = i * (i + 1) // 2 + j
            for k in range(n):
                for l in range(k + 1):
                    kl = k * (k + 1) // 2 + l
                    if kl > ij or abs(eri[i, j, k, l]) <= drop_below:
                        continue
                    out.append(f"{eri[i, j, k, l]: .16e} {i + 1:4d} {j + 1:4d} {k + 1:4d} {l + 1:4d}")
    for i in range(n):
        for j in range(i + 1):
            out.append(f"{h1[i, j]: .16e} {i + 1:4d} {j + 1:4d}    0    0")
    for i in range(n):
        out.append(f"{h1[i, i]: .16e} {i + 1:4d}    0    0    0")
    out.append(f"{ecore: .16e}    0    0    0    0")
    return "\n".join(lines + out) + "\n"


def write_fcidump(path: str, name_or_spec, seed: int = 0, t: Optional[float] = None,
                  drop_below: float = 0.0) -> SynthSpec:
    spec, h1, eri, ecore = make_integrals(name_or_spec, seed, t)
    tmp = path + ".tmp%d" % os.getpid()
    with open(tmp, "w") as f:
        f.write(fcidump_text(spec, h1, eri, ecore, drop_below))
    os.replace(tmp, path)
    return spec


def write_input_json(path: str, fcidump_path: str, **cdfci) -> None:
    import json

    opts = {
        "hamiltonian": {"fcidump_path": fcidump_path, "threshold": 0.0},
        "solver": {"cdfci": dict(cdfci)},
    }
    with open(path, "w") as f:
        json.dump(opts, f, indent=4)
