"""The hash table that grows on demand (mcd_options.table_growth, the default).

The table starts at the size that two 64-iteration chunks of worst-case
inserts need and doubles by rehashing as it fills (when the worst case could
pass 3/4, or the load passes 1/4), up to the table max_memory gives.  Growth
changes where determinants sit, not what the iteration computes:

- with k = 1 (one column per iteration, so no two adds race on a slot) a solve
  that grows reports the same energies, sizes and counters as one that holds
  the whole table from the start;
- after growths (k = 1 on the 16-orbital workload: a first table of 2^20
  slots that grows within 3000 iterations), the solver's xx and xz still
  equal the sums over the table
  (WaveFunctionCuckoo::debug_calculate_xx_xz, src/wavefunction.h:640-667);
- a checkpoint with more entries than a fresh solver's first table loads into
  it (the table grows first) and continues the solve;
- a doubling by runs of clusters (rehash_double_kernel, in shared memory or by
  global compare-and-swap) keeps every determinant with its x and z, and the
  solve after it follows the fill-and-insert rehash's exactly (k = 1).
"""
import os

import pytest

import mcdfci_b200 as m

pytestmark = pytest.mark.gpu


def _reports(path, growth, **kw):
    s = m.CDFCI(m.Fcidump(path), table_growth=growth, **kw)
    s.solve()
    info = s.table_info()
    reps = s.reports
    s.close()
    return reps, info


def test_growth_gives_the_same_solve_k1(synth_fcidumps):
    path = synth_fcidumps["n16_5a5b"]
    kw = dict(num_of_coordinate=1, estimate=16, max_memory=1.0, threshold=0.0, z_threshold=0.0,
              num_iterations=3000, report_interval=500)
    grown, gi = _reports(path, True, **kw)
    whole, wi = _reports(path, False, **kw)
    assert gi["growths"] >= 1 and gi["capacity"] > 1 << 20
    assert wi["growths"] == 0 and wi["capacity"] == wi["max_capacity"] == gi["max_capacity"]
    assert len(grown) == len(whole) == 6
    for a, b in zip(grown, whole):
        assert a["iteration"] == b["iteration"]
        assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(b["energy"])
        for f in ("x_size", "z_size", "cols_size", "updates", "emitted_total", "updates_total", "occupied"):
            assert a[f] == b[f], f


def test_scalars_match_table_after_growth(synth_fcidumps):
    path = synth_fcidumps["n16_5a5b"]
    s = m.CDFCI(m.Fcidump(path), num_of_coordinate=1, estimate=16, max_memory=1.0, threshold=0.0,
                z_threshold=0.0)
    s.reset()
    cap0 = s.table_info()["capacity"]
    s.run_iterations(3000)
    info = s.table_info()
    assert info["growths"] >= 1 and info["capacity"] > cap0
    sc = s.scalars()
    t = s.table_sums()
    r = s.report()
    assert t["occupied"] == r["occupied"]
    xx, txx = sum(sc["xx"]), sum(t["xx"])
    xz, txz = sum(sc["xz"]), sum(t["xz"])
    assert abs(xx - txx) <= 1e-12 * abs(xx)
    assert abs(xz - txz) <= 1e-10 * abs(xz)
    s.close()


def test_checkpoint_loads_into_a_smaller_first_table(synth_fcidumps, tmp_path):
    path = synth_fcidumps["n16_5a5b"]
    ck = os.path.join(str(tmp_path), "n16.ckpt")
    kw = dict(num_of_coordinate=1, estimate=16, max_memory=1.0, threshold=0.0, z_threshold=0.0)
    a = m.CDFCI(m.Fcidump(path), **kw)
    a.reset()
    a.run_iterations(3000)
    r_mid = a.report()
    a.save(ck)
    a.run_iterations(200)
    r_a = a.report()
    cap_a = a.table_info()["capacity"]
    a.close()
    b = m.CDFCI(m.Fcidump(path), **kw)
    assert b.table_info()["capacity"] < cap_a
    b.load(ck)
    assert r_mid["occupied"] <= 0.75 * b.table_info()["capacity"]
    r_b0 = b.report()
    assert (r_b0["iteration"], r_b0["z_size"], r_b0["occupied"]) == (r_mid["iteration"], r_mid["z_size"],
                                                                      r_mid["occupied"])
    b.run_iterations(200)
    r_b = b.report()
    assert r_b["iteration"] == r_a["iteration"]
    assert abs(r_b["energy"] - r_a["energy"]) < 1e-9
    b.close()


def _sorted_slots(s):
    import numpy as np

    a, b, x, z = s.slots()
    o = np.lexsort((b, a))
    return a[o], b[o], x[o], z[o]


@pytest.mark.parametrize("mode", [0, 1])
def test_doubling_rehash_keeps_every_entry(synth_fcidumps, mode):
    """A doubling moves runs of whole clusters (mode 0: placed in shared
    memory; mode 1: every entry by global compare-and-swap), and writes every
    slot of the new table: the same determinants with the same x and z, the
    same occupancy, and (k = 1) the same solve afterwards as the fill and
    insert of mode 2."""
    import numpy as np

    path = synth_fcidumps["n16_5a5b"]
    kw = dict(num_of_coordinate=1, estimate=16, max_memory=1.0, threshold=0.0, z_threshold=0.0)
    solvers, wraps = {}, {}
    for md in (mode, 2):
        s = m.CDFCI(m.Fcidump(path), **kw)
        s.reset()
        s.run_iterations(1500)
        before = _sorted_slots(s)
        occ0 = s.report()["occupied"]
        cap0 = s.table_info()["capacity"]
        wraps[md] = [s.grow(md), s.grow(md)]
        assert s.table_info()["capacity"] == 4 * cap0
        after = _sorted_slots(s)
        for u, v in zip(before, after):
            assert np.array_equal(u, v)
        r = s.report()
        assert r["occupied"] == occ0 == len(before[0])
        assert s.table_sums()["occupied"] == occ0
        solvers[md] = s
    # The occupied slots of linear probing do not depend on the insertion
    # order, so both solvers saw the same clusters at the table ends.
    assert wraps[mode] == wraps[2]
    reps = {}
    for md, s in solvers.items():
        out = []
        for _ in range(3):
            s.run_iterations(200)
            out.append(s.report())
        reps[md] = out
        s.close()
    for a, b in zip(reps[mode], reps[2]):
        assert a["iteration"] == b["iteration"]
        assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(b["energy"])
        for f in ("x_size", "z_size", "cols_size", "updates", "emitted_total", "updates_total", "occupied"):
            assert a[f] == b[f], f
