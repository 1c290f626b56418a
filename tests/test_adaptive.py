"""Adaptive RK45 stepping, restated (oracle/hos_np.py: advance_adaptive):
the step control of hos_step_adaptive on the reference's Dormand-Prince
pair (time_schemes_par.c:183-235), whose 5th-order weights the reference
computes but never uses.  CPU tests of the controller: it lands on t_end,
its result converges to a fine fixed-step run as the tolerance tightens,
a too-large first step is rejected and shrunk, and with no error budget
pressure it keeps every step.  The GPU path is compared with this
restatement in tests/test_gpu_parity.py."""
import math

import numpy as np

from hos_b200 import ic
from oracle.hos_np import HosNumpy


def setup(n=32, M=4, seed=21):
    eta, phi, info = ic.jonswap(n, n, kp=4.0, steepness=0.1, seed=seed)
    hn = HosNumpy(n, n, 2 * math.pi, 2 * math.pi, 1.0, M)
    e, p = hn.init_state(eta, phi)
    return hn, e, p, info["Tp"]


def fine_reference(hn, e, p, t_end, nsteps=400):
    t = 0.0
    dt = t_end / nsteps
    for _ in range(nsteps):
        e, p, t, _ = hn.step(e, p, t, dt, 2)
    return e, p


def test_lands_on_t_end_and_converges_with_tolerance():
    hn, e0, p0, tp = setup()
    t_end = 2.0 * tp
    re, rp = fine_reference(hn, e0, p0, t_end)
    errs, kept = [], []
    for rtol in (1e-4, 1e-6, 1e-8):
        e, p, t, dt, H, acc, rej = hn.advance_adaptive(e0, p0, 0.0, t_end, tp / 50, rtol, 1e-14)
        assert abs(t - t_end) <= 1e-12 * t_end
        assert len(H) == acc and dt > 0
        errs.append(max(np.max(np.abs(e - re)), np.max(np.abs(p - rp))) / np.max(np.abs(re)))
        kept.append(acc)
    assert kept[0] < kept[1] < kept[2]          # tighter tolerance: more, smaller steps
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-5  # and results closer to the fine run


def test_too_large_first_step_is_rejected_and_shrunk():
    hn, e0, p0, tp = setup()
    e, p, t, dt, H, acc, rej = hn.advance_adaptive(e0, p0, 0.0, tp, 5.0 * tp, 1e-9, 1e-14)
    assert rej >= 1 and acc >= 2 and abs(t - tp) <= 1e-12 * tp


def test_loose_tolerance_keeps_every_step_and_grows_dt():
    hn, e0, p0, tp = setup()
    dt0 = tp / 200
    e, p, t, dt, H, acc, rej = hn.advance_adaptive(e0, p0, 0.0, tp / 20, dt0, 1.0, 1.0)
    assert rej == 0 and dt > dt0
