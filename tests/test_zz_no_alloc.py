"""mcd_eig_update_static: the subspace eig update with its device buffers in
a static device array of the library instead of per-call cudaMalloc.  It runs
the same kernel as mcd_debug_eig, so each result is compared with
mcd_debug_eig on the same inputs, on two calls in a row (the second call must
not see anything left by the first), and with the outputs the reference's
CoordinateUpdateEig recorded on the same inputs.  Tolerance: dx, xx and scale within
1e-12 relative (the kernels are the same; the tolerance only allows for a
different reduction order should the two launch shapes ever differ).

Named to be collected last, so that it also runs after every other GPU test
has used the device."""
import numpy as np
import pytest

import mcdfci_b200 as m
from conftest import load_golden

RTOL = 1e-12


def _close(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.all(np.abs(a - b) <= RTOL * (1.0 + np.abs(b)))


def _cases():
    out = []
    for k in (1, 8, 33, 64, 128):
        rng = np.random.default_rng(500 + k)
        A = rng.normal(size=(k, k))
        H = (A + A.T) / 2 - 30 * np.eye(k) + np.diag(rng.uniform(0, 5, k))
        x = rng.normal(size=k) * 0.1
        z = H @ x + rng.normal(size=k) * 0.05
        out.append((H, x, z, (float(x @ x) + 0.5, 0.0), (float(x @ z) - 10.0, 0.0)))
    # First-iteration branch (x = e_0, xx = 1: the k x k problem).
    rng = np.random.default_rng(7)
    A = rng.normal(size=(16, 16))
    H = (A + A.T) / 2 - 20 * np.eye(16)
    x = np.zeros(16)
    x[0] = 1.0
    out.append((H, x, H @ x, (1.0, 0.0), (H[0, 0], 0.0)))
    # Subproblems recorded inside a reference solve.
    for rec in load_golden("eig_h2o.json.gz")["calls"][:4]:
        k = rec["k"]
        out.append((np.array(rec["hsub"]).reshape(k, k), np.array(rec["x"]), np.array(rec["z"]),
                    tuple(rec["xx"]), tuple(rec["xz"])))
    return out


@pytest.mark.gpu
def test_static_eig_matches_debug_eig_twice():
    for H, x, z, xx, xz in _cases():
        ref = m.debug_eig(H, x, z, xx, xz)
        for call in range(2):
            dx, nxx, nsc, branch = m.eig_update_static(H, x, z, xx, xz)
            assert branch == ref[3], (len(x), call)
            assert _close(dx, ref[0]), (len(x), call)
            assert _close(nxx[0] + nxx[1], ref[1][0] + ref[1][1]), (len(x), call)
            assert _close(nsc[0] + nsc[1], ref[2][0] + ref[2][1]), (len(x), call)


@pytest.mark.gpu
def test_static_eig_matches_reference_records_twice():
    """Against the reference itself: the outputs CoordinateUpdateEig produced
    on subproblems recorded inside a reference solve (dx within 1e-9, xx and
    |scale| within 1e-12 relative, the tolerances of the parity tests; the
    first-iteration record's eigenvector sign is arbitrary in LAPACK)."""
    for rec in load_golden("eig_h2o.json.gz")["calls"]:
        k = rec["k"]
        H = np.array(rec["hsub"]).reshape(k, k)
        ref_dx = np.array(rec["dx"])
        x = np.array(rec["x"])
        for call in range(2):
            dx, nxx, nsc, branch = m.eig_update_static(H, x, np.array(rec["z"]), tuple(rec["xx"]),
                                                       tuple(rec["xz"]))
            assert branch == (2 if rec["call"] == 0 else 1)
            if branch == 2:
                err = min(np.max(np.abs(dx - ref_dx)), np.max(np.abs(dx + ref_dx + 2 * x)))
            else:
                err = np.max(np.abs(dx - ref_dx) / (1.0 + np.abs(ref_dx)))
            assert err < 1e-9, (rec["call"], call, err)
            rxx = rec["new_xx"][0] + rec["new_xx"][1]
            rsc = rec["new_scale"][0] + rec["new_scale"][1]
            assert abs(nxx[0] + nxx[1] - rxx) <= 1e-12 * abs(rxx)
            assert abs(abs(nsc[0] + nsc[1]) - abs(rsc)) <= 1e-12 * abs(rsc)


@pytest.mark.gpu
def test_static_eig_alternating_sizes():
    """A small k after a large one reads only its own k x k block."""
    cases = _cases()
    big, small = cases[4], cases[1]
    ref_small = m.debug_eig(*small)
    m.eig_update_static(*big)
    dx, nxx, nsc, branch = m.eig_update_static(*small)
    assert branch == ref_small[3]
    assert _close(dx, ref_small[0])


def test_static_eig_rejects_k_above_its_scratch():
    """Checked before any CUDA call: runs without a GPU."""
    k = 129
    H = -np.eye(k)
    x = np.zeros(k)
    with pytest.raises(m.McdError) as e:
        m.eig_update_static(H, x, x, (1.0, 0.0), (0.0, 0.0))
    assert e.value.code == 5  # MCD_ERR_UNSUPPORTED
    assert "128" in e.value.message
