"""bench.py's reference arm (`--impl reference`): the compiled reference,
cdfci_omp, run on this host's cores on the bench workload, parsed into the
bench's JSON line (impl, metric, unit, a positive rate, cpu_baseline and e2e
objects).  CPU only; skipped where the reference has not been compiled."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EXE = os.path.join(REPO, "oracle", "_ref", "cdfci_omp")


@pytest.mark.skipif(not os.path.exists(REF_EXE), reason="oracle/_ref/cdfci_omp not built")
def test_reference_arm_prints_one_json_line():
    res = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "3",
                          "--warmup", "3", "--max-memory", "1"], capture_output=True, text=True, timeout=600,
                         cwd=REPO)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "coord updates/s" and d["unit"] == "coordinate_updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
