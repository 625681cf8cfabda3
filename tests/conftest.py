import gzip
import json
import os
import shutil
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); run with -m gpu")


def load_golden(name: str):
    path = os.path.join(GOLDEN, name)
    opener = gzip.open if name.endswith(".gz") else open
    with opener(path, "rt") as f:
        return json.load(f)


@pytest.fixture(scope="session")
def fcidumps(tmp_path_factory):
    """Uncompressed copies of the FCIDUMP fixtures: name -> path."""
    d = tmp_path_factory.mktemp("fcidump")
    out = {}
    for name in ("h2o_sto3g", "n7_5a5b", "n33_2a1b"):
        src = os.path.join(GOLDEN, name + ".fcidump.gz")
        dst = os.path.join(str(d), name + ".fcidump")
        with gzip.open(src, "rb") as fi, open(dst, "wb") as fo:
            shutil.copyfileobj(fi, fo)
        out[name] = dst
    return out


@pytest.fixture(scope="session")
def synth_fcidumps(tmp_path_factory):
    """Synthetic workloads written by mcdfci_b200.synth (seed 0)."""
    from mcdfci_b200 import synth

    d = tmp_path_factory.mktemp("synth")
    out = {}
    for name in ("n7_5a5b", "n12_6a6b", "n16_5a5b", "n24_6a6b"):
        p = os.path.join(str(d), name + ".fcidump")
        synth.write_fcidump(p, name, seed=0)
        out[name] = p
    return out


# Fixture file -> (FCIDUMP fixture, hamiltonian threshold) it was produced with.
COLUMN_FIXTURES = {
    "cols_h2o.json.gz": ("h2o_sto3g", 0.0),
    "cols_h2o_thr1e-3.json.gz": ("h2o_sto3g", 1e-3),
    "cols_n7.json.gz": ("n7_5a5b", 0.0),
    "cols_n33.json.gz": ("n33_2a1b", 0.0),
}
HSUB_FIXTURES = {
    "hsub_h2o.json.gz": ("h2o_sto3g", 0.0),
    "hsub_h2o_k24.json.gz": ("h2o_sto3g", 0.0),
    "hsub_n7.json.gz": ("n7_5a5b", 0.0),
    "hsub_n33.json.gz": ("n33_2a1b", 0.0),
}
