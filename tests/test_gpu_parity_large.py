"""The drop-in gate at the benchmark sizes: 100 RK4 steps of the FP64 path
against the reference's own code, and the FP32 form's accuracy over the
precision configuration's 1000 steps.

The reference results are the committed fixtures tests/golden/jonswap*_100
made by ``python tests/golden/make_golden.py large`` from the C oracle (the
reference's Csource/2dpar hot-path sources; the 2/3-rule case uses the build
whose operators_par.c:290-291 bounds read floor(N/3)).  The reference state
never leaves the dealias mask, so a fixture holds the kept modes only; the
test regenerates the seeded inputs and checks their checksum first.

Gate (SURVEY parity metric): max|d|/max|ref| and ||d||_2/||ref||_2 of the
spectra and of physical eta and phi_s <= 1e-10, the stage-0 energy series
<= 1e-10 relative, and the volume (eta-hat at k = 0) held against the
reference within 1e-10 of max|eta-hat|: the JONSWAP seas have zero mean, so
this is a conservation check of the mean level, scaled by the field."""
import math

import numpy as np
import pytest

from hos_b200 import HosField, ic
from oracle.hos_np import HosNumpy

pytestmark = pytest.mark.gpu

TOL_STEPS = 1e-10
LARGE = ["jonswap512_m4_rk4_100", "jonswap512_m4_d23_rk4_100", "jonswap1024_m5_rk4_100"]


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def inputs_of(d):
    n, _, M, _, seed, mx, my = (int(v) for v in d["meta"])
    kp, st, gamma, spread = (float(v) for v in d["ic"])
    eta, phi, info = ic.jonswap(n, n, kp=kp, steepness=st, gamma=gamma, spread_s=spread, seed=seed)
    # the fixture was made from the same seeded inputs
    assert abs(eta.sum() - float(d["eta_sum"])) <= 1e-9 * float(d["eta_l2"])
    assert abs(np.linalg.norm(eta) / float(d["eta_l2"]) - 1) < 1e-12
    assert abs(np.linalg.norm(phi) / float(d["phi_l2"]) - 1) < 1e-12
    return n, M, mx, my, eta, phi


@pytest.mark.parametrize("name", LARGE)
def test_100_rk4_steps_drop_in_gate_benchmark_sizes(golden, name):
    d = golden(name)
    n, M, mx, my, eta, phi = inputs_of(d)
    d23 = "_d23_" in name
    dt = float(d["dt"])
    with HosField(n, n, order=M, mx=mx if d23 else None, my=my if d23 else None) as f:
        assert f.bounds == (mx, my)
        f.set_state_physical(eta, phi)
        f.step(dt, 100)
        u, t = f.state_spectral()
        tt, H = f.energy_history()
        eta_g, phi_g = f.state_physical()
    ref = np.zeros_like(u)
    rows, cols = d["rows"].astype(np.int64), d["cols"].astype(np.int64)
    ref[:, rows, cols] = d["u100"]
    # nothing outside the mask, as in the reference
    mask = np.zeros(u.shape[1:], bool)
    mask[rows, cols] = True
    assert not np.any(u[:, ~mask])
    for q in range(2):
        assert rel_max(u[q], ref[q]) < TOL_STEPS
        assert rel_l2(u[q], ref[q]) < TOL_STEPS
    hn = HosNumpy(n, n, 2 * math.pi, 2 * math.pi, 1.0, M, mx=mx, my=my)
    eta_r, phi_r = hn.ifft2(ref[0]), hn.ifft2(ref[1])
    errs = {"eta_max": rel_max(eta_g, eta_r), "eta_l2": rel_l2(eta_g, eta_r),
            "phi_max": rel_max(phi_g, phi_r), "phi_l2": rel_l2(phi_g, phi_r)}
    print(name, {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) < TOL_STEPS
    assert abs(u[0][0, 0] - ref[0][0, 0]) <= TOL_STEPS * np.max(np.abs(ref[0]))
    assert abs(t - float(d["t100"])) < 1e-12
    assert len(H) == 100
    assert np.max(np.abs(H - d["ham"])) / np.max(np.abs(d["ham"])) < TOL_STEPS


def test_fp32_form_precision_configuration_1000_steps(golden):
    """1024^2, M = 5, JONSWAP kp = 24, kp*Hs/2 = 0.12, gamma = 3.3, s = 10:
    the FP32-compute form (FP64 state) against its FP64 rerun after 1000
    RK4 steps.  Target eta error <= 1e-5 Hs; the phi_s and energy errors are
    stated and held to the levels measured on B200 with a margin."""
    d = golden("jonswap1024_m5_rk4_100")
    n, M, mx, my, eta, phi = inputs_of(d)
    dt = float(d["dt"])
    hs = float(d["hs"])
    out = {}
    for prec in ("fp64", "fp32"):
        with HosField(n, n, order=M, precision=prec) as f:
            f.set_state_physical(eta, phi)
            f.step(dt, 1000)
            f.sync()
            out[prec] = (f.state_physical(), f.energy_history()[1])
    (e64, p64), H64 = out["fp64"]
    (e32, p32), H32 = out["fp32"]
    eta_err = float(np.max(np.abs(e32 - e64)) / hs)
    phi_err = rel_max(p32, p64)
    ham_err = float(np.max(np.abs(H32 - H64)) / np.max(np.abs(H64)))
    print(f"fp32 form after 1000 steps: eta err {eta_err:.2e} Hs, phi_s err {phi_err:.2e}, energy err {ham_err:.2e}")
    assert eta_err <= 1e-5
    assert phi_err <= 1e-5
    assert ham_err <= 1e-5
