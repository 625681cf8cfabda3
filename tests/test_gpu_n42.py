"""The 42-orbital, 24 + 24 electron workload: alpha and beta strings wider
than 32 bits, and 84 spin-orbitals, which the reference keeps in two 64-bit
words (interleaved).  Columns (271,945 entries) are bit-exact with the oracle
along a walk of determinants, and a k = 64 solve runs with a decreasing
energy."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, interleaved_to_ab

import mcdfci_b200 as m
from mcdfci_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def n42(tmp_path_factory):
    d = tmp_path_factory.mktemp("n42")
    p = os.path.join(str(d), "n42.fcidump")
    synth.write_fcidump(p, "n42_24a24b", seed=0)
    return p


def test_n42_columns_vs_oracle(n42):
    o = Oracle(n42, 0.0)
    assert o.nw == 2
    s = m.CDFCI(m.Fcidump(n42), max_memory=0.05, num_of_coordinate=8, estimate=8, threshold=0.0)
    a, b = interleaved_to_ab(o.hartree_fock(), o.nw)
    assert a >> 32 and b >> 32  # strings wider than 32 bits
    rng = np.random.default_rng(2)
    for _ in range(3):
        dets, vals = o.column_ab(a, b)
        ref = {d: v for d, v in zip(dets, vals)}
        ca, cb, cv = s.column(m.Determinant(a, b))
        mine = {(int(x), int(y)): float(v) for x, y, v in zip(ca, cb, cv)}
        assert len(mine) == len(ca) == len(ref) == 271945
        assert set(mine) == set(ref)
        for k, v in ref.items():
            if k != (a, b):
                assert mine[k] == v
        a, b = dets[int(rng.integers(1, len(dets)))]


def test_n42_solve_k64(n42):
    # Every early iteration inserts most of its 64 x 271,945 column entries.
    s = m.CDFCI(m.Fcidump(n42), max_memory=32.0, num_of_coordinate=64, estimate=64, threshold=0.0,
                z_threshold=1e-6, num_iterations=24, report_interval=8)
    s.solve()
    es = [r["energy"] for r in s.reports]
    assert len(es) == 3
    assert es[0] > es[1] > es[2]
    assert s.reports[-1]["last_k"] == 64
