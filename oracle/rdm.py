"""Reduced density matrices and integral gradients on the CPU, from explicit
fermionic operators on occupation bit strings.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU RDM
path; the product never imports it.

Conventions (spin-orbitals interleaved as in the reference, src/input.h:242-243:
spin-orbital 2P is spatial orbital P with spin alpha, 2P+1 with spin beta;
operators ordered by that index, Jordan-Wigner signs):

    gamma[p][q]      = <a+_p a_q>
    Gamma[p][q][r][s] = <a+_p a+_q a_s a_r>
    E = sum h[p][q] gamma[p][q] + 1/2 sum <pq|rs> Gamma[p][q][r][s] + E_core

Spin-summed spatial forms: g1[P][Q] = sum_s gamma[Ps][Qs],
g2[P][Q][R][S] = sum_{s,t} Gamma[Ps][Qt][Rs][St], so that
E = sum h_PQ g1[P][Q] + 1/2 sum (PR|QS) g2[P][Q][R][S] + E_core.
"""
from __future__ import annotations

from itertools import combinations
from typing import Dict, List, Tuple

import numpy as np


def read_fcidump(path: str):
    """Spatial integrals of an RHF FCIDUMP with the 8-fold symmetry of real
    orbitals filled in: (norb, nelec, ms2, h[n,n], eri[n,n,n,n] chemist
    (ij|kl), ecore).  An independent parse of the format, kept minimal."""
    with open(path) as f:
        text = f.read()
    head, body = text.split("&END", 1) if "&END" in text else text.split("/", 1)
    import re

    def field(name):
        m = re.search(name + r"\s*=\s*(-?\d+)", head, flags=re.I)
        return int(m.group(1)) if m else None

    n, ne, ms2 = field("NORB"), field("NELEC"), field("MS2") or 0
    h = np.zeros((n, n))
    eri = np.zeros((n, n, n, n))
    ecore = 0.0
    for line in body.split("\n"):
        t = line.split()
        if len(t) != 5:
            continue
        v = float(t[0].replace("D", "E").replace("d", "e"))
        i, j, k, l = (int(x) for x in t[1:])
        if i == 0 and j == 0 and k == 0 and l == 0:
            ecore = v
        elif j == 0 and k == 0 and l == 0:
            continue  # orbital energy
        elif k == 0 and l == 0:
            h[i - 1, j - 1] = h[j - 1, i - 1] = v
        else:
            a, b, c, d = i - 1, j - 1, k - 1, l - 1
            for (p, q, r, s) in ((a, b, c, d), (b, a, c, d), (a, b, d, c), (b, a, d, c),
                                 (c, d, a, b), (d, c, a, b), (c, d, b, a), (d, c, b, a)):
                eri[p, q, r, s] = v
    return n, ne, ms2, h, eri, ecore


def determinants(norb: int, na: int, nb: int) -> List[Tuple[int, int]]:
    """(alpha, beta) occupation strings of the full determinant space."""
    return [(sum(1 << p for p in a), sum(1 << p for p in b)) for a in combinations(range(norb), na)
            for b in combinations(range(norb), nb)]


def _to_so(a: int, b: int, norb: int) -> int:
    bits = 0
    for p in range(norb):
        if (a >> p) & 1:
            bits |= 1 << (2 * p)
        if (b >> p) & 1:
            bits |= 1 << (2 * p + 1)
    return bits


def _apply(bits: int, create: int, annihilate: int):
    """a+_create a_annihilate |bits> -> (sign, bits') or None."""
    if not (bits >> annihilate) & 1:
        return None
    s = bin(bits & ((1 << annihilate) - 1)).count("1")
    bits ^= 1 << annihilate
    if (bits >> create) & 1:
        return None
    s += bin(bits & ((1 << create) - 1)).count("1")
    return (-1.0 if s & 1 else 1.0), bits | (1 << create)


def rdms(norb: int, dets: List[Tuple[int, int]], c: np.ndarray):
    """Spin-orbital gamma[2n,2n] and Gamma[2n,2n,2n,2n] of the normalised
    vector c over `dets`, with Gamma_pqrs = <E_pr E_qs> - delta_qr gamma_ps
    and E_pr = a+_p a_r."""
    nso = 2 * norb
    so = [_to_so(a, b, norb) for a, b in dets]
    index: Dict[int, int] = {d: i for i, d in enumerate(so)}
    c = np.asarray(c, dtype=np.float64) / np.linalg.norm(c)
    # w[(p, r)] = E_pr c
    W = np.zeros((nso * nso, len(dets)))
    for p in range(nso):
        for r in range(nso):
            col = W[p * nso + r]
            for i, bits in enumerate(so):
                res = _apply(bits, p, r)
                if res is not None:
                    s, nb = res
                    j = index.get(nb)
                    if j is not None:
                        col[j] += s * c[i]
    gamma = (W @ c).reshape(nso, nso)  # <c|E_pr|c>
    G = W @ W.T  # G[(r,p),(q,s)] = <E_rp c, E_qs c> = <c|E_pr E_qs|c>
    Gamma = np.zeros((nso, nso, nso, nso))
    for p in range(nso):
        for q in range(nso):
            for r in range(nso):
                for s in range(nso):
                    v = G[r * nso + p, q * nso + s]
                    if q == r:
                        v -= gamma[p, s]
                    Gamma[p, q, r, s] = v
    return gamma, Gamma


def spin_summed(gamma: np.ndarray, Gamma: np.ndarray):
    n = gamma.shape[0] // 2
    g1 = np.zeros((n, n))
    g2 = np.zeros((n, n, n, n))
    for s in range(2):
        g1 += gamma[s::2, s::2]
        for t in range(2):
            g2 += Gamma[s::2, t::2, s::2, t::2]
    return g1, g2


def energy(h: np.ndarray, eri: np.ndarray, ecore: float, g1: np.ndarray, g2: np.ndarray) -> float:
    """E = sum h_PQ g1_PQ + 1/2 sum (PR|QS) g2_PQRS + E_core."""
    return float(np.einsum("pq,pq", h, g1) + 0.5 * np.einsum("prqs,pqrs", eri, g2) + ecore)


def fcidump_gradient(g1: np.ndarray, g2: np.ndarray, i: int, j: int, k: int = 0, l: int = 0) -> float:
    """dE / d(value of the FCIDUMP line 'v i j k l') (1-based indices, k = l =
    0 for a one-electron line), the line's value entering every position the
    8-fold (resp. 2-fold) symmetry gives it; 0 for orbital-energy lines
    'v i 0 0 0', which do not enter the energy."""
    if j == 0 and k == 0 and l == 0:
        return 0.0  # orbital energy or core energy line (the core energy's gradient is 1)
    if k == 0 and l == 0:
        a, b = i - 1, j - 1
        return float(g1[a, b] + (g1[b, a] if a != b else 0.0))
    a, b, c, d = i - 1, j - 1, k - 1, l - 1
    perms = {(a, b, c, d), (b, a, c, d), (a, b, d, c), (b, a, d, c),
             (c, d, a, b), (d, c, a, b), (c, d, b, a), (d, c, b, a)}
    # A position (x0 x1|x2 x3) is (PR|QS) with P = x0, R = x1, Q = x2, S = x3.
    return float(sum(0.5 * g2[x[0], x[2], x[1], x[3]] for x in perms))
