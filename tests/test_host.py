"""Host-side checks that need no GPU: the C-ABI library loads and exports
every symbol include/mcdfci.h declares, the product's FCIDUMP reader matches
the oracle's, option validation fails before touching CUDA, and the synthetic
generator is deterministic."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO

import mcdfci_b200 as m


def test_header_symbols_exported():
    header = open(os.path.join(REPO, "include", "mcdfci.h")).read()
    declared = set(re.findall(r"^\s*(?:int|void|const char\*)\s+(mcd_\w+)\(", header, flags=re.M))
    assert declared == set(m.EXPORTED_SYMBOLS)
    L = m.library()
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", m.LIB_PATH], capture_output=True, text=True).stdout
    for name in declared:
        assert re.search(rf"\bT {name}$", out, flags=re.M), name


@pytest.mark.parametrize("name", ["h2o_sto3g", "n7_5a5b", "n33_2a1b"])
def test_fcidump_reader_matches_oracle(name, fcidumps):
    from oracle.oracle import Oracle

    f = m.Fcidump(fcidumps[name])
    o = Oracle(fcidumps[name], 0.0)
    assert (f.norb, f.nelec, f.ms2) == (o.nso, o.nelec, o.ms2)
    assert f.core_energy == o.ecore
    h1, g2 = f.arrays()
    oh1, og2 = o.integrals()
    assert np.array_equal(h1, oh1)
    assert np.array_equal(g2, og2)


def test_fcidump_errors(tmp_path):
    with pytest.raises(m.McdError) as e:
        m.Fcidump(str(tmp_path / "missing"))
    assert e.value.code == m.MCD_ERR_INVALID and "Failed to open" in e.value.message
    bad = tmp_path / "bad"
    bad.write_text("&FCI NORB=2,\n NELEC=2,\n&END\n 1.0 1 1 1 1\n")
    with pytest.raises(m.McdError) as e:
        m.Fcidump(str(bad))
    assert "MS2 is not found" in e.value.message
    noend = tmp_path / "noend"
    noend.write_text("&FCI NORB=2, NELEC=2, MS2=0\n")
    with pytest.raises(m.McdError) as e:
        m.Fcidump(str(noend))
    assert "wrong header" in e.value.message
    oob = tmp_path / "oob"
    oob.write_text("&FCI NORB=2,NELEC=2,MS2=0,\n&END\n 1.0 3 1 1 1\n")
    with pytest.raises(m.McdError):
        m.Fcidump(str(oob))


@pytest.mark.parametrize(
    "opts,code,text",
    [
        (dict(max_memory=0.0), m.MCD_ERR_INVALID, "max_memory"),
        (dict(max_memory=0.01, coordinate_update="ls"), m.MCD_ERR_UNSUPPORTED, "ls"),
        (dict(max_memory=0.01, num_of_coordinate=129), m.MCD_ERR_UNSUPPORTED, "num_of_coordinate"),
        (dict(max_memory=0.01, estimate=0), m.MCD_ERR_UNSUPPORTED, "estimate"),
        (dict(max_memory=0.01, z_threshold_search=True, report_interval=10), m.MCD_ERR_INVALID, "report_interval"),
        (dict(max_memory=0.01, report_interval=0), m.MCD_ERR_INVALID, "report_interval"),
    ],
)
def test_option_validation_before_gpu(opts, code, text, fcidumps):
    f = m.Fcidump(fcidumps["n7_5a5b"])
    with pytest.raises(m.McdError) as e:
        m.CDFCI(f, **opts)
    assert e.value.code == code and text in e.value.message


def test_run_json_missing_deck():
    assert m.run_json("/nonexistent/input.json") == 1
    assert "Can not read the input file" in m.library().mcd_last_error().decode()


def test_synth_deterministic_and_symmetric(tmp_path):
    from mcdfci_b200 import synth

    a, b = tmp_path / "a", tmp_path / "b"
    synth.write_fcidump(str(a), "n7_5a5b", seed=0)
    synth.write_fcidump(str(b), "n7_5a5b", seed=0)
    assert a.read_bytes() == b.read_bytes()
    spec, h1, eri, ecore = synth.make_integrals("n12_6a6b", seed=3)
    assert np.allclose(h1, h1.T)
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1)]:
        assert np.allclose(eri, eri.transpose(perm))
    assert synth.hf_energy(h1, eri, spec.nalpha, spec.nbeta) + ecore < 0
    # Curve endpoints differ and interpolate.
    _, h0, e0, _ = synth.make_integrals("n16_5a5b", seed=0, t=0.0)
    _, h1c, e1, _ = synth.make_integrals("n16_5a5b", seed=0, t=1.0)
    _, hm, em, _ = synth.make_integrals("n16_5a5b", seed=0, t=0.5)
    assert np.allclose(hm, 0.5 * (h0 + h1c)) and np.allclose(em, 0.5 * (e0 + e1))


def test_batch_rejects_before_gpu(fcidumps):
    """Batch limits are checked on the host, before any device work."""
    f = m.Fcidump(fcidumps["n7_5a5b"])
    with pytest.raises(m.McdError) as e:
        m.CDFCIBatch([], max_memory=0.001)
    assert e.value.code == m.MCD_ERR_INVALID
    with pytest.raises(m.McdError) as e:
        m.CDFCIBatch([f] * 65, max_memory=0.001)
    assert e.value.code == m.MCD_ERR_UNSUPPORTED
    with pytest.raises(m.McdError) as e:
        m.CDFCIBatch([f, f], max_memory=0.001, z_threshold_search=True, report_interval=1000)
    assert e.value.code == m.MCD_ERR_UNSUPPORTED
