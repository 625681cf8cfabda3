"""The CTAs-per-column autotuner (mcd_options.autotune): its trials are
iterations of the solve (the iteration count stays exact), it keeps the
fastest candidate, and a second solver of the same shape takes the choice
from the process's cache without trials."""
import pytest

import mcdfci_b200 as m

pytestmark = pytest.mark.gpu


def test_autotune_picks_fastest_and_caches(synth_fcidumps):
    path = synth_fcidumps["n16_5a5b"]
    kw = dict(num_of_coordinate=16, estimate=16, max_memory=1.0, threshold=0.0, z_threshold=0.0, autotune=True)
    s = m.CDFCI(m.Fcidump(path), **kw)
    s.reset()
    s.run_iterations(300)
    assert s.report()["iteration"] == 300
    info = s.autotune_info()
    assert len(info["trials"]) >= 3
    best = min(info["trials"], key=lambda t: t["column_us"])
    assert info["chosen"] == best["groups"]
    assert any(t["groups"] == info["rule"] for t in info["trials"])
    assert s.launch_info()["groups"] == info["chosen"]
    s.close()
    s2 = m.CDFCI(m.Fcidump(path), **kw)
    s2.reset()
    s2.run_iterations(200)
    i2 = s2.autotune_info()
    assert i2["trials"] == [] and i2["chosen"] == info["chosen"]
    assert s2.report()["iteration"] == 200
    s2.close()
