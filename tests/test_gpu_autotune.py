"""The autotuner picks kernel shapes by timing whole RK steps, caches them,
and a field built with the chosen shapes computes the same RK step as one
with the default shapes (to rounding: other shapes reassociate the FFT
arithmetic)."""
import json

import numpy as np
import pytest

from hos_b200 import HosField, autotune, ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [("fp32", 1e-5), ("fp64", 1e-12)])
def test_tune_caches_and_keeps_results(tmp_path, monkeypatch, prec, tol):
    monkeypatch.setenv("HOS_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    t = autotune.tune(128, 128, 3, prec, reps=1)
    assert len(t) == 12 and t[8] >= 1 and t[10] in (8, 16, 32)
    db = json.load(open(tmp_path / "tune.json"))
    (entry,) = db.values()
    assert entry["tune"] == t and "default" in entry["report"]
    assert autotune.tune(128, 128, 3, prec) == t  # from the cache
    eta, phi, info = ic.jonswap(128, 128, kp=6.0, steepness=0.1, seed=8)
    out = []
    for shapes in (None, t):
        with HosField(128, 128, order=3, precision=prec, tune=shapes) as f:
            f.set_state_physical(eta, phi)
            f.step(info["Tp"] / 50, 10)
            out.append(f.state_spectral()[0])
    assert np.max(np.abs(out[1] - out[0])) <= tol * np.max(np.abs(out[0]))
