"""The product column kernel checked directly, one iteration at a time.

The table is exported (mcd_debug_slots) before and after exactly one
iteration of the product path (leader_kernel + column_kernel, the launches a
solve makes), and every change is compared with the oracle's Hamiltonian
columns of the picked determinants times their dx, the update of
WaveFunctionCuckoo::update_z_and_get_sub (src/wavefunction.h:499-552) and
update_x (src/wavefunction.h:425-451):

- keys: the determinants after the iteration are those before plus the ones
  the insertion rule admits (some column's |H dx scale| > z_threshold),
  bit-exact;
- x: unchanged except x[D_c] + dx_c on the picked determinants, bit-exact;
- z: z + sum_c H[D, D_c] dx_c on every other determinant, within 1e-12 of the
  terms' magnitude (the adds of different columns to one determinant are FP64
  atomics in the order the CTAs reach them); on a determinant that the
  iteration inserts, a below-threshold term of another column lands only if
  that column's probe comes after the insert, so such terms bound the
  difference;
- the picked determinants' z: the exact recompute sum_D' H[D', D_c] x[D']
  over the column with the updated x (src/wavefunction.h:557-565).

Workloads: 24 orbitals, 6 + 6 electrons (16,471 entries per column), k = 32,
with z_threshold 0 and 1e-7; 42 orbitals, 24 + 24 electrons (271,945 entries,
strings wider than 32 bits), k = 8.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle

import mcdfci_b200 as m
from mcdfci_b200 import synth

pytestmark = pytest.mark.gpu

KEY = np.dtype([("a", "<u8"), ("b", "<u8")])


def _keys(a, b):
    k = np.empty(len(a), dtype=KEY)
    k["a"] = a
    k["b"] = b
    return k


def _lookup(sorted_keys, q):
    """Index of each q in sorted_keys, -1 where absent."""
    i = np.searchsorted(sorted_keys, q)
    i = np.minimum(i, len(sorted_keys) - 1)
    hit = sorted_keys[i] == q
    return np.where(hit, i, -1)


def _abs_scaled(scale, dz):
    """|scale * dz| in double, scale = (hi, lo); it can differ from the
    kernel's double-double test only within 1e-13 of the threshold, which the
    checks below leave open."""
    return np.abs(scale[0] * dz + scale[1] * dz)


def _check_one_iteration(path, k, zt, warm, max_memory):
    o = Oracle(path, 0.0)
    s = m.CDFCI(m.Fcidump(path), num_of_coordinate=k, estimate=k, max_memory=max_memory, threshold=0.0,
                z_threshold=zt)
    s.reset()
    s.run_iterations(warm)
    a0, b0, x0, z0 = s.slots()
    s.run_iterations(1)
    a1, b1, x1, z1 = s.slots()
    pa, pb, dx = s.picked()
    sc = s.scalars()["scale"]
    s.close()
    assert len(pa) == k

    k0 = _keys(a0, b0)
    o0 = np.argsort(k0, kind="stable")
    k0s = k0[o0]
    k1 = _keys(a1, b1)
    o1 = np.argsort(k1, kind="stable")
    k1s = k1[o1]
    x0s, z0s, x1s, z1s = x0[o0], z0[o0], x1[o1], z1[o1]
    assert len(np.unique(k1s)) == len(k1s)

    # Contributions of every column.
    ta, tb, tv = [], [], []
    for c in range(k):
        ca, cb, cv = o.column_ab_arrays(int(pa[c]), int(pb[c]))
        ta.append(ca)
        tb.append(cb)
        tv.append(cv * dx[c])
    tk = _keys(np.concatenate(ta), np.concatenate(tb))
    dz = np.concatenate(tv)
    above = _abs_scaled(sc, dz) > zt
    near = np.abs(_abs_scaled(sc, dz) - zt) <= 1e-13 * max(zt, 1e-300)
    uk, inv = np.unique(tk, return_inverse=True)
    sum_all = np.bincount(inv, weights=dz, minlength=len(uk))
    sum_abs = np.bincount(inv, weights=np.abs(dz), minlength=len(uk))
    any_above = np.bincount(inv, weights=above.astype(float), minlength=len(uk)) > 0
    any_near = np.bincount(inv, weights=near.astype(float), minlength=len(uk)) > 0
    below_abs = np.bincount(inv, weights=np.where(above, 0.0, np.abs(dz)), minlength=len(uk))

    pk = _keys(pa, pb)
    is_picked = np.isin(uk, pk)

    # Keys: before + admitted insertions, nothing else.
    i0 = _lookup(k0s, uk)
    new = i0 < 0
    i1 = _lookup(k1s, uk)
    inserted = new & (i1 >= 0)
    assert np.all((i1 >= 0) | ~any_above | any_near), "a determinant above the threshold was not inserted"
    assert np.all(~inserted | any_above | any_near), "a determinant below the threshold was inserted"
    assert np.all(_lookup(k1s, k0s) >= 0), "a determinant left the table"
    assert len(k1s) == len(k0s) + int(inserted.sum())

    # x: unchanged except on the picked determinants.
    j = _lookup(k1s, k0s)
    xp_i0 = _lookup(k0s, pk)
    assert np.all(xp_i0 >= 0)
    x_exp = x0s.copy()
    x_exp[xp_i0] = x0s[xp_i0] + dx
    assert np.array_equal(x1s[j], x_exp)

    # z on determinants that were present and not picked.
    sel = (~new) & (~is_picked)
    zb = z0s[i0[sel]]
    za = z1s[i1[sel]]
    tol = 1e-12 * (np.abs(zb) + sum_abs[sel]) + 1e-300
    err = np.abs(za - (zb + sum_all[sel]))
    assert np.all(err <= tol), float(np.max(err / tol))
    # z on inserted determinants: the above-threshold terms, plus some of the others.
    sel = inserted & ~is_picked
    za = z1s[i1[sel]]
    above_sum = np.bincount(inv, weights=np.where(above, dz, 0.0), minlength=len(uk))[sel]
    tol = 1e-12 * sum_abs[sel] + below_abs[sel] + 1e-300
    assert np.all(np.abs(za - above_sum) <= tol)
    # Determinants untouched by the iteration keep their z.
    touched = np.zeros(len(k0s), dtype=bool)
    touched[i0[~new]] = True
    untouched = ~touched
    untouched[xp_i0] = False
    assert np.array_equal(z1s[j[untouched]], z0s[untouched])

    # Picked determinants: z is the exact recompute with the updated x.
    for c in range(k):
        ca, cb, cv = o.column_ab_arrays(int(pa[c]), int(pb[c]))
        ii = _lookup(k1s, _keys(ca, cb))
        xv = np.where(ii >= 0, x1s[np.maximum(ii, 0)], 0.0)
        exact = float(np.dot(cv, xv))
        got = float(z1s[_lookup(k1s, pk[c:c + 1])[0]])
        # 1e-11: the diagonal term comes from the leader's own diagonal sum (1e-12 relative)
        assert abs(got - exact) <= 1e-11 * float(np.sum(np.abs(cv * xv))) + 1e-300, (c, got, exact)
    return len(k0s), int(inserted.sum())


@pytest.fixture(scope="module")
def n24(tmp_path_factory):
    p = os.path.join(str(tmp_path_factory.mktemp("n24")), "n24.fcidump")
    synth.write_fcidump(p, "n24_6a6b", seed=0)
    return p


@pytest.fixture(scope="module")
def n42(tmp_path_factory):
    p = os.path.join(str(tmp_path_factory.mktemp("n42")), "n42.fcidump")
    synth.write_fcidump(p, "n42_24a24b", seed=0)
    return p


def test_column_kernel_one_iteration_n24(n24):
    before, inserted = _check_one_iteration(n24, k=32, zt=0.0, warm=6, max_memory=2.0)
    assert inserted > 0


def test_column_kernel_one_iteration_n24_threshold(n24):
    # z_threshold 1e-7: most new entries of a late iteration are below it,
    # so both branches of the insertion rule run.
    before, inserted = _check_one_iteration(n24, k=32, zt=1e-7, warm=40, max_memory=2.0)
    assert inserted > 0


def test_column_kernel_one_iteration_n42(n42):
    before, inserted = _check_one_iteration(n42, k=8, zt=1e-6, warm=3, max_memory=4.0)
    assert inserted > 0
