"""The oracle against the golden fixtures and against itself.

The C oracle (the reference's own hot-path sources built with the shim) and
the numpy restatement must agree with each other and with the committed
fixtures, which tests/golden/make_golden.py produced from the C oracle."""
import glob
import math
import os

import numpy as np
import pytest

from oracle import ref_c
from oracle.hos_np import HosNumpy

from .conftest import GOLDEN

needs_c = pytest.mark.skipif(not ref_c.available(3), reason="C oracle not built (make -C oracle)")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_golden_files_present():
    names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    assert "stokes64_m3_rk4_100.npz" in names
    assert len(names) >= 14


def test_numpy_fft_matches_golden(golden):
    d = golden("fft_32x16")
    hn = HosNumpy(32, 16, 2 * math.pi, 2 * math.pi, 1.0, 3)
    assert rel(hn.fft2(d["x"]), d["hx"]) < 1e-14
    assert rel(hn.ifft2(d["s"]), d["xs"]) < 1e-14


@pytest.mark.parametrize("name", ["rhs_m4_32x16_d_r1", "rhs_m3_32x32_nd_r0", "rhs_m5_64x64_d_r1",
                                  "rhs_m6_32x64_d_r0", "rhs_m1_16x16_nd_r0", "rhs_m2_16x32_d_r1"])
def test_numpy_rhs_matches_golden(golden, name):
    d = golden(name)
    nx, ny, M, ramp = (int(v) for v in d["meta"])
    hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, float(d["g"]), M, rampflg=ramp, tramp=float(d["tramp"]))
    re_, rp = hn.rhs(d["u"][0], d["u"][1], float(d["t"]))
    assert rel(re_, d["rhs"][0]) < 1e-12
    assert rel(rp, d["rhs"][1]) < 1e-12


def test_numpy_stokes_100_steps_matches_golden(golden):
    d = golden("stokes64_m3_rk4_100")
    hn = HosNumpy(64, 64, 2 * math.pi, 2 * math.pi, 1.0, 3)
    e, p = hn.init_state(d["eta0"], d["phi0"])
    assert rel(e, d["u0"][0]) < 1e-14
    t = 0.0
    H = []
    for _ in range(100):
        e, p, t, h = hn.step(e, p, t, float(d["dt"]), 2)
        H.append(h)
    assert rel(e, d["u100"][0]) < 1e-11
    assert rel(p, d["u100"][1]) < 1e-11
    assert np.max(np.abs(np.array(H) - d["ham"])) / np.max(np.abs(d["ham"])) < 1e-11
    assert abs(t - float(d["t100"])) < 1e-12


@pytest.mark.parametrize("scheme", [1, 2, 3, 4, 5])
def test_numpy_schemes_match_golden(golden, scheme):
    d = golden(f"scheme{scheme}_32_m4")
    hn = HosNumpy(32, 32, 2 * math.pi, 2 * math.pi, 1.0, 4)
    e, p = d["u0"][0], d["u0"][1]
    t = 0.0
    for _ in range(5):
        e, p, t, _h = hn.step(e, p, t, float(d["dt"]), scheme)
    assert rel(e, d["u5"][0]) < 1e-12
    assert rel(p, d["u5"][1]) < 1e-12


@needs_c
def test_c_oracle_reproduces_golden(golden):
    d = golden("stokes64_m3_rk4_100")
    ref = ref_c.RefC(3, 64, 64)
    u0 = ref.init_state(d["eta0"], d["phi0"])
    assert np.array_equal(u0, d["u0"])
    u, t, ham = ref.steps(u0, 0.0, float(d["dt"]), 100)
    assert np.array_equal(u, d["u100"])
    assert np.array_equal(ham, d["ham"])


@needs_c
def test_c_oracle_matches_numpy_random():
    rng = np.random.default_rng(99)
    for M, nx, ny in [(3, 16, 16), (5, 32, 16), (7, 16, 32)]:
        hn = HosNumpy(nx, ny, 3.0, 5.0, 9.81, M, rampflg=1, tramp=1.5)
        ref = ref_c.RefC(M, nx, ny, lx=3.0, ly=5.0, g=9.81, rampflg=1, tramp=1.5)
        u = 0.01 * (rng.standard_normal((2, ny // 2 + 1, nx)) + 1j * rng.standard_normal((2, ny // 2 + 1, nx)))
        r = ref.rhs(u, 0.3)
        re_, rp = hn.rhs(u[0], u[1], 0.3)
        assert rel(re_, r[0]) < 1e-12 and rel(rp, r[1]) < 1e-12


def test_oracle_catches_planted_error(golden):
    """A mistake planted in the oracle (a wrong kx convention) must be seen by
    the golden comparison, so the comparison has teeth."""
    d = golden("rhs_m3_32x32_nd_r0")
    hn = HosNumpy(32, 32, 2 * math.pi, 2 * math.pi, 1.0, 3)
    i = np.arange(32)
    hn.kx = np.where(i <= 16, i, -(32 - i))[None, :] * np.ones((17, 1))  # textbook kx, not the reference's
    hn.kz = np.sqrt(hn.kx**2 + hn.ky**2)
    re_, _ = hn.rhs(d["u"][0], d["u"][1], float(d["t"]))
    assert rel(re_, d["rhs"][0]) > 1e-6
