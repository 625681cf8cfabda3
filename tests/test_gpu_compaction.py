"""Compaction under max_memory (mcd_options.compaction, mcd_debug_compact):
it removes only entries with x = 0 and |z scale| <= z_threshold, so the
coefficients and the sums xx = sum x^2 and xz = sum x z are unchanged, the
iteration continues from the compacted table, and a solve whose table would
overflow completes with a raised z_threshold."""
import numpy as np
import pytest

import mcdfci_b200 as m

pytestmark = pytest.mark.gpu


def test_compaction_keeps_coefficients_and_sums(synth_fcidumps):
    s = m.CDFCI(m.Fcidump(synth_fcidumps["n12_6a6b"]), num_of_coordinate=16, estimate=16, max_memory=0.5,
                threshold=0.0, z_threshold=0.0)
    s.reset()
    s.run_iterations(800)
    e0 = s.report()["energy"]
    t0 = s.table_sums()
    a0, b0, x0 = s.wavefunction()
    occ = s.compact(1e-6)
    t1 = s.table_sums()
    a1, b1, x1 = s.wavefunction()
    assert occ < t0["occupied"]
    assert occ == t1["occupied"]
    before = {(int(a), int(b)): float(x) for a, b, x in zip(a0, b0, x0)}
    after = {(int(a), int(b)): float(x) for a, b, x in zip(a1, b1, x1)}
    assert before == after
    xx0, xx1 = sum(t0["xx"]), sum(t1["xx"])
    xz0, xz1 = sum(t0["xz"]), sum(t1["xz"])
    assert abs(xx1 - xx0) <= 1e-14 * abs(xx0)
    assert abs(xz1 - xz0) <= 1e-14 * abs(xz0)
    r = s.report()
    assert r["z_threshold"] == 1e-6 and r["z_size"] == occ
    assert abs(r["energy"] - e0) <= 1e-12 * abs(e0)
    s.run_iterations(400)
    assert s.report()["energy"] < e0


def test_solve_with_compaction_under_small_max_memory(synth_fcidumps):
    """16 orbitals, 5 + 5 electrons (1.9e7 determinants): a table half the size
    the run needs overflows without compaction and completes with it; reports
    every 10 iterations keep one interval's growth below the margin between
    the 60% trigger and the occupancy limit."""
    path = synth_fcidumps["n16_5a5b"]
    opts = dict(num_of_coordinate=16, estimate=16, threshold=0.0, z_threshold=0.0, num_iterations=400,
                report_interval=10)
    big = m.CDFCI(m.Fcidump(path), max_memory=4.0, **opts)
    e_big = big.solve()
    need = big.reports[-1]["z_size"]
    small_gb = need * 24 * 0.5 / 1e9  # 24 bytes per determinant at one word per string
    with pytest.raises(m.McdError) as err:
        m.CDFCI(m.Fcidump(path), max_memory=small_gb, **opts).solve()
    assert err.value.code == m.MCD_ERR_OVERFLOW
    small = m.CDFCI(m.Fcidump(path), max_memory=small_gb, compaction=True, **opts)
    e_small = small.solve()
    assert small.reports[-1]["z_threshold"] > 0.0
    assert abs(e_small - e_big) < 1e-3
