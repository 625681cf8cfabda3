"""GPU parity: the sm_100a kernels, called through the C ABI, against the
reference's own fixtures and the C restatement in oracle/.

Bars: connected determinants and phases exact; excitation values bit for bit
(the GPU sums single-excitation terms in the reference's order); diagonal
elements within 1e-12 relative (the GPU reduces them across a warp); eig
updates within the tolerances stated in each test."""
import numpy as np
import pytest

from conftest import COLUMN_FIXTURES, HSUB_FIXTURES, load_golden
from oracle.oracle import Oracle, ab_to_interleaved, interleaved_to_ab

import mcdfci_b200 as m

pytestmark = pytest.mark.gpu

DIAG_RTOL = 1e-12


def _solver(path, thr=0.0, **kw):
    opts = dict(max_memory=0.01, num_of_coordinate=8, estimate=8, threshold=thr)
    opts.update(kw)
    return m.CDFCI(m.Fcidump(path), **opts)


def _gpu_column(s, a, b):
    ca, cb, cv = s.column(m.Determinant(a, b))
    return {(int(x), int(y)): float(v) for x, y, v in zip(ca, cb, cv)}, len(ca)


def _check_column(mine, n_mine, ref, diag_key):
    assert n_mine == len(mine), "duplicate determinant in a GPU column"
    assert set(mine) == set(ref)
    for k, v in ref.items():
        if k == diag_key:
            assert abs(mine[k] - v) <= DIAG_RTOL * abs(v)
        else:
            assert mine[k] == v, (k, mine[k], v)


@pytest.mark.parametrize("fixture", sorted(COLUMN_FIXTURES))
def test_columns_vs_reference_fixture(fixture, fcidumps):
    fcid, thr = COLUMN_FIXTURES[fixture]
    g = load_golden(fixture)
    nw = g["n_words"]
    s = _solver(fcidumps[fcid], thr)
    for rec in g["dets"]:
        a, b = interleaved_to_ab(rec["det"], nw)
        mine, n = _gpu_column(s, a, b)
        ref = {interleaved_to_ab(e[0], nw): e[1] for e in rec["col"]}
        _check_column(mine, n, ref, (a, b))


def test_columns_vs_oracle_every_det_n7(fcidumps):
    o = Oracle(fcidumps["n7_5a5b"], 0.0)
    s = _solver(fcidumps["n7_5a5b"])
    from itertools import combinations

    count = 0
    for occa in combinations(range(7), 5):
        for occb in combinations(range(7), 5):
            a = sum(1 << p for p in occa)
            b = sum(1 << p for p in occb)
            dets, vals = o.column_ab(a, b)
            ref = {d: v for d, v in zip(dets, vals)}
            mine, n = _gpu_column(s, a, b)
            _check_column(mine, n, ref, (a, b))
            count += 1
    assert count == 441


@pytest.mark.parametrize("name", ["n12_6a6b", "n16_5a5b", "n24_6a6b"])
def test_columns_vs_oracle_synthetic(name, synth_fcidumps):
    o = Oracle(synth_fcidumps[name], 0.0)
    s = _solver(synth_fcidumps[name])
    rng = np.random.default_rng(1)
    a, b = interleaved_to_ab(o.hartree_fock(), o.nw)
    for _ in range(6):
        dets, vals = o.column_ab(a, b)
        ref = {d: v for d, v in zip(dets, vals)}
        mine, n = _gpu_column(s, a, b)
        _check_column(mine, n, ref, (a, b))
        a, b = dets[int(rng.integers(1, len(dets)))]


@pytest.mark.parametrize("fixture", sorted(HSUB_FIXTURES))
def test_hsub_vs_reference_fixture(fixture, fcidumps):
    fcid, thr = HSUB_FIXTURES[fixture]
    g = load_golden(fixture)
    nw = g["n_words"]
    s = _solver(fcidumps[fcid], thr)
    for rec in g["sets"]:
        dets = [m.Determinant(*interleaved_to_ab(d, nw)) for d in rec["dets"]]
        k = len(dets)
        h = s.hsub(dets)
        ref = np.array(rec["hsub"]).reshape(k, k)
        off = ~np.eye(k, dtype=bool)
        assert np.array_equal(h[off], ref[off])
        assert np.all(np.abs(np.diag(h) - np.diag(ref)) <= DIAG_RTOL * np.abs(np.diag(ref)))


def _dd(p):
    return float(p[0]) + float(p[1])


@pytest.mark.parametrize("fixture", ["eig_h2o.json.gz", "eig_n7.json.gz"])
def test_eig_update_vs_reference_fixture(fixture):
    """CoordinateUpdateEig records captured inside reference solves.  The
    reference solves with LAPACK dsyevr plus one __float128 inverse-iteration
    step; here Householder + multisection + inverse iteration with a
    double-double Rayleigh quotient.  Tolerances: dx within 1e-9 absolute
    (plus 1e-9 relative), xx within 1e-12 relative, |scale| within 1e-12
    relative (the sign of scale follows the arbitrary sign LAPACK gives the
    eigenvector)."""
    g = load_golden(fixture)
    for rec in g["calls"]:
        k = rec["k"]
        H = np.array(rec["hsub"]).reshape(k, k)
        dx, nxx, nsc, branch = m.debug_eig(H, rec["x"], rec["z"], rec["xx"], rec["xz"])
        ref_dx = np.array(rec["dx"])
        assert branch == (2 if rec["call"] == 0 else 1)
        if branch == 2:
            # First iteration: dx = v*sqrt(-lambda) - x, sign of v arbitrary in LAPACK.
            x = np.array(rec["x"])
            alt = -(ref_dx + x) - x
            err = min(np.max(np.abs(dx - ref_dx)), np.max(np.abs(dx - alt)))
        else:
            err = np.max(np.abs(dx - ref_dx) / (1.0 + np.abs(ref_dx)))
        assert err < 1e-9, (rec["call"], err)
        assert abs(_dd(nxx) - _dd(rec["new_xx"])) <= 1e-12 * abs(_dd(rec["new_xx"]))
        assert abs(abs(_dd(nsc)) - abs(_dd(rec["new_scale"]))) <= 1e-12 * abs(_dd(rec["new_scale"]))


@pytest.mark.parametrize("fixture", ["eig_h2o.json.gz", "eig_n7.json.gz"])
def test_eig_update_shifted_vs_reference_fixture(fixture):
    """The leader's first method on the recorded reference calls: shifted
    inverse iteration from a Cholesky factorisation of B - sigma I, with the
    drop a solve would pass (the energy drop of the update itself, read from
    the record: xz/xx - lambda, lambda = -new_xx new_scale^2).  Same
    tolerances as the full reduction; a drop far too small puts sigma above
    lambda_1, the factorisation fails and the reduction gives the result."""
    g = load_golden(fixture)
    taken = 0
    n = 0
    for rec in g["calls"]:
        if rec["call"] == 0:
            continue
        k = rec["k"]
        H = np.array(rec["hsub"]).reshape(k, k)
        lam = -_dd(rec["new_xx"]) * _dd(rec["new_scale"]) ** 2
        drop = _dd(rec["xz"]) / _dd(rec["xx"]) - lam
        for d, expect_shift in ((max(drop, 1e-12), True), (1e-300, False)):
            dx, nxx, nsc, branch, steps = m.debug_eig_shifted(H, rec["x"], rec["z"], rec["xx"], rec["xz"], d)
            assert branch == 1
            if expect_shift:
                n += 1
                taken += steps > 0
            ref_dx = np.array(rec["dx"])
            err = np.max(np.abs(dx - ref_dx) / (1.0 + np.abs(ref_dx)))
            assert err < 1e-9, (rec["call"], d, steps, err)
            assert abs(_dd(nxx) - _dd(rec["new_xx"])) <= 1e-12 * abs(_dd(rec["new_xx"])), (rec["call"], steps)
            assert abs(abs(_dd(nsc)) - abs(_dd(rec["new_scale"]))) <= 1e-12 * abs(_dd(rec["new_scale"]))
    # the shifted solver, not its fallback, handles the recorded calls but
    # the first few (an energy drop near the spectral gap)
    assert taken >= n - 2, (taken, n)


def _eig_reference_numpy(H, x, z, xx, xz):
    """The reference's eig update (src/solver.h:333-609) restated with numpy
    eigh in float64."""
    k = len(x)
    Hx = H @ x
    yy = xx - x @ x
    if abs(yy) > 1e-14:
        y1 = np.sqrt(yy)
        B = np.zeros((k + 1, k + 1))
        B[0, 0] = (xz - 2 * (x @ z) + x @ Hx) / yy
        B[0, 1:] = B[1:, 0] = (z - Hx) / y1
        B[1:, 1:] = H
        w, V = np.linalg.eigh(B)
        v = V[:, 0] * np.sign(V[0, 0])
        lam = -w[0]
        gamma = v[0] / y1
        scale = gamma * np.sqrt(lam)
        return v[1:] / gamma - x, lam / scale ** 2, scale
    w, V = np.linalg.eigh(H)
    v = V[:, 0] * (1 if V[:, 0] @ x >= 0 else -1)
    return v * np.sqrt(-w[0]) - x, -w[0], 1.0


@pytest.mark.parametrize("k", [1, 2, 3, 8, 31, 32, 33, 64, 100, 128])
def test_eig_update_random_vs_numpy(k):
    rng = np.random.default_rng(k)
    A = rng.normal(size=(k, k))
    H = (A + A.T) / 2 - 30 * np.eye(k) + np.diag(rng.uniform(0, 5, k))
    x = rng.normal(size=k) * 0.1
    z = H @ x + rng.normal(size=k) * 0.05
    xx = float(x @ x) + 0.5
    xz = float(x @ z) - 10.0
    dx, nxx, nsc, branch = m.debug_eig(H, x, z, (xx, 0.0), (xz, 0.0))
    rdx, rxx, rsc = _eig_reference_numpy(H, x, z, xx, xz)
    assert branch == 1
    assert np.max(np.abs(dx - rdx) / (1 + np.abs(rdx))) < 1e-9
    assert abs(_dd(nxx) - rxx) < 1e-10 * abs(rxx)
    assert abs(_dd(nsc) - rsc) < 1e-10 * abs(rsc)


@pytest.mark.parametrize("k", [1, 2, 8, 32, 33, 64])
def test_eig_update_shifted_random_vs_numpy(k):
    """Shifted solver on random subproblems near convergence: B is chosen
    first, the current vector is its lowest eigenvector plus 1e-3 noise, and
    (H, x, z, xx, xz) are derived so that the update rebuilds that B.  With
    the exact energy drop and with 30 times it (a lower shift, more steps)."""
    rng = np.random.default_rng(300 + k)
    A = rng.normal(size=(k + 1, k + 1))
    M = 0.05 * (A + A.T) / 2 - 30 * np.eye(k + 1) + np.diag(rng.uniform(0, 5, k + 1))
    M[0, 0] = -33.0
    w, U = np.linalg.eigh(M)
    u = U[:, 0] * np.sign(U[0, 0])
    y1 = 1.3 * u[0]
    x = 1.3 * u[1:] + 1e-3 * rng.normal(size=k)
    H = M[1:, 1:]
    z = H @ x + y1 * M[0, 1:]
    xx = float(y1 * y1 + x @ x)
    xz = float(M[0, 0] * y1 * y1 + 2 * (x @ z) - x @ H @ x)
    rdx, rxx, rsc = _eig_reference_numpy(H, x, z, xx, xz)
    drop = xz / xx + rxx * rsc ** 2
    assert drop > 0
    for d in (drop, 30 * drop):
        dx, nxx, nsc, branch, steps = m.debug_eig_shifted(H, x, z, (xx, 0.0), (xz, 0.0), d)
        assert branch == 1
        assert steps > 0
        assert np.max(np.abs(dx - rdx) / (1 + np.abs(rdx))) < 1e-9
        assert abs(_dd(nxx) - rxx) < 1e-10 * abs(rxx)
        assert abs(abs(_dd(nsc)) - abs(rsc)) < 1e-10 * abs(rsc)


@pytest.mark.parametrize("fixture", ["eig_h2o.json.gz", "eig_n7.json.gz"])
def test_eig_update_bordered_vs_reference_fixture(fixture):
    """The bordered fixed point (eig_method 2) on the recorded reference calls:
    same tolerances as the full reduction.  It certifies its eigenvalue as the
    lowest when the eigenvalue plus the residual norm lies below the Gershgorin
    bound of H_sub; the recorded calls but the first few certify, the others
    take the reduction."""
    g = load_golden(fixture)
    taken = n = 0
    for rec in g["calls"]:
        if rec["call"] == 0:
            continue
        k = rec["k"]
        H = np.array(rec["hsub"]).reshape(k, k)
        dx, nxx, nsc, branch, steps = m.debug_eig_method(H, rec["x"], rec["z"], rec["xx"], rec["xz"], 2)
        assert branch == 1
        n += 1
        taken += steps > 0
        ref_dx = np.array(rec["dx"])
        err = np.max(np.abs(dx - ref_dx) / (1.0 + np.abs(ref_dx)))
        assert err < 1e-9, (rec["call"], steps, err)
        assert abs(_dd(nxx) - _dd(rec["new_xx"])) <= 1e-12 * abs(_dd(rec["new_xx"])), (rec["call"], steps)
        assert abs(abs(_dd(nsc)) - abs(_dd(rec["new_scale"]))) <= 1e-12 * abs(_dd(rec["new_scale"]))
    assert taken >= n - 2, (taken, n)


@pytest.mark.parametrize("k,coupling,certified", [(1, 0.02, True), (2, 0.02, True), (8, 0.02, True),
                                                  (32, 0.02, True), (33, 0.02, True), (64, 0.01, True),
                                                  (16, 1.5, False), (65, 0.01, False)])
def test_eig_update_bordered_random_vs_numpy(k, coupling, certified):
    """Bordered fixed point on random subproblems: B = [[a, b'], [b, C]] with C
    diagonal plus symmetric couplings of the given size, (H, x, z, xx, xz)
    derived so that the update rebuilds B.  Weak couplings keep lambda_1 below
    C's Gershgorin bound (certified, steps > 0); strong ones do not, and k = 65
    is beyond the method's 64 rows: the reduction runs (steps = 0).  Both
    against numpy eigh."""
    rng = np.random.default_rng(500 + k)
    A = rng.normal(size=(k, k))
    C = coupling * (A + A.T) / 2
    np.fill_diagonal(C, -30.0 + rng.uniform(0, 5, k))
    M = np.zeros((k + 1, k + 1))
    M[0, 0] = -33.0
    M[0, 1:] = M[1:, 0] = 0.3 * rng.normal(size=k)
    M[1:, 1:] = C
    w, U = np.linalg.eigh(M)
    u = U[:, 0] * np.sign(U[0, 0])
    y1 = 1.3 * u[0]
    x = 1.3 * u[1:] + 1e-3 * rng.normal(size=k)
    H = M[1:, 1:]
    z = H @ x + y1 * M[0, 1:]
    xx = float(y1 * y1 + x @ x)
    xz = float(M[0, 0] * y1 * y1 + 2 * (x @ z) - x @ H @ x)
    rdx, rxx, rsc = _eig_reference_numpy(H, x, z, xx, xz)
    dx, nxx, nsc, branch, steps = m.debug_eig_method(H, x, z, (xx, 0.0), (xz, 0.0), 2)
    assert branch == 1
    assert (steps > 0) == certified, steps
    assert np.max(np.abs(dx - rdx) / (1 + np.abs(rdx))) < 1e-9
    assert abs(_dd(nxx) - rxx) < 1e-10 * abs(rxx)
    assert abs(abs(_dd(nsc)) - abs(rsc)) < 1e-10 * abs(rsc)


@pytest.mark.parametrize("k", [1, 4, 16])
def test_eig_update_first_iteration_branch(k):
    rng = np.random.default_rng(100 + k)
    A = rng.normal(size=(k, k))
    H = (A + A.T) / 2 - 20 * np.eye(k)
    x = np.zeros(k)
    x[0] = 1.0
    dx, nxx, nsc, branch = m.debug_eig(H, x, H @ x, (1.0, 0.0), (H[0, 0], 0.0))
    rdx, rxx, rsc = _eig_reference_numpy(H, x, H @ x, 1.0, H[0, 0])
    assert branch == 2
    assert np.max(np.abs(dx - rdx)) < 1e-9
    assert abs(_dd(nxx) - rxx) < 1e-12 * abs(rxx)
    assert _dd(nsc) == 1.0
