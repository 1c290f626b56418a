"""Parity of the CUDA path (through the C ABI) with the oracle.

FP64 drop-in: results must match the reference CPU path to 1e-10 relative
after 100 RK4 steps; single operator evaluations to 1e-12.  The FP32-compute
form is held to the error it documents (relative to the FP64 result)."""
import math

import numpy as np
import pytest

from hos_b200 import HosField, ic
from oracle.hos_np import HosNumpy

pytestmark = pytest.mark.gpu

TOL_OP = 1e-12     # one RHS / transform, FP64
TOL_STEPS = 1e-10  # after up to 100 RK steps, FP64 (the drop-in gate)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_fft_pair_matches_golden(golden):
    d = golden("fft_32x16")
    with HosField(32, 16) as f:
        assert rel(f.fft_2d(d["x"]), d["hx"]) < 1e-14
        assert rel(f.ifft_2d(d["s"]), d["xs"]) < 1e-14


@pytest.mark.parametrize("nx,ny", [(16, 16), (64, 128), (256, 32), (1024, 1024), (2048, 512), (4096, 64)])
def test_fft_pair_random(nx, ny):
    rng = np.random.default_rng(nx + ny)
    hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, 3)
    x = rng.standard_normal((nx, ny))
    s = rng.standard_normal((ny // 2 + 1, nx)) + 1j * rng.standard_normal((ny // 2 + 1, nx))
    with HosField(nx, ny) as f:
        assert rel(f.fft_2d(x), hn.fft2(x)) < 1e-13
        assert rel(f.ifft_2d(s), hn.ifft2(s)) < 1e-13


@pytest.mark.parametrize("name", ["rhs_m4_32x16_d_r1", "rhs_m3_32x32_nd_r0", "rhs_m5_64x64_d_r1",
                                  "rhs_m6_32x64_d_r0", "rhs_m1_16x16_nd_r0", "rhs_m2_16x32_d_r1"])
def test_rhs_matches_golden(golden, name):
    d = golden(name)
    nx, ny, M, ramp = (int(v) for v in d["meta"])
    with HosField(nx, ny, order=M, g=float(d["g"]), rampflg=ramp, tramp=float(d["tramp"])) as f:
        r = f.rhs(d["u"], float(d["t"]))
    assert rel(r[0], d["rhs"][0]) < TOL_OP
    assert rel(r[1], d["rhs"][1]) < TOL_OP


def test_init_state_matches_golden(golden):
    d = golden("stokes64_m3_rk4_100")
    with HosField(64, 64, order=3) as f:
        f.set_state_physical(d["eta0"], d["phi0"])
        u, t = f.state_spectral()
    assert rel(u, d["u0"]) < 1e-14 and t == 0.0


def test_stokes_100_rk4_steps_drop_in_gate(golden):
    """First configuration: 64^2, M=3, Stokes ka=0.1, RK4 dt=T/64, 100 steps."""
    d = golden("stokes64_m3_rk4_100")
    hn = HosNumpy(64, 64, 2 * math.pi, 2 * math.pi, 1.0, 3)
    with HosField(64, 64, order=3) as f:
        f.set_state_physical(d["eta0"], d["phi0"])
        f.step(float(d["dt"]), 100)
        u, t = f.state_spectral()
        tt, H = f.energy_history()
        eta, phi = f.state_physical()
    assert rel(u[0], d["u100"][0]) < TOL_STEPS
    assert rel(u[1], d["u100"][1]) < TOL_STEPS
    # the parity metric is stated on physical eta and phi_s: max|d|/max|ref| and ||d||_2/||ref||_2
    eta_ref, phi_ref = hn.ifft2(d["u100"][0]), hn.ifft2(d["u100"][1])
    assert rel(eta, eta_ref) < TOL_STEPS and rel(phi, phi_ref) < TOL_STEPS
    assert np.linalg.norm(eta - eta_ref) / np.linalg.norm(eta_ref) < TOL_STEPS
    assert np.linalg.norm(phi - phi_ref) / np.linalg.norm(phi_ref) < TOL_STEPS
    # volume (eta-hat at k = 0) as the reference keeps it; the Stokes wave has
    # zero mean, so this is a conservation check scaled by the field (a state
    # with a non-zero mean is checked in test_volume_of_offset_sea_vs_reference)
    assert abs(u[0][0, 0] - d["u100"][0][0, 0]) <= TOL_STEPS * np.max(np.abs(d["u100"][0]))
    assert abs(t - float(d["t100"])) < 1e-12
    assert len(H) == 100
    assert np.max(np.abs(H - d["ham"])) / np.max(np.abs(d["ham"])) < TOL_STEPS
    assert abs(tt[0]) < 1e-15 and abs(tt[-1] - 99 * float(d["dt"])) < 1e-9


@pytest.mark.parametrize("scheme", [1, 2, 3, 4, 5])
def test_schemes_match_golden(golden, scheme):
    d = golden(f"scheme{scheme}_32_m4")
    with HosField(32, 32, order=4, scheme=scheme) as f:
        f.set_state_spectral(d["u0"], 0.0)
        f.step(float(d["dt"]), 5)
        u, t = f.state_spectral()
        _, H = f.energy_history()
    assert rel(u, d["u5"]) < TOL_STEPS
    assert np.max(np.abs(H - d["ham"])) / np.max(np.abs(d["ham"])) < TOL_STEPS


def test_jonswap_ramp_m5_matches_golden(golden):
    d = golden("jonswap64_m5_ramp_20")
    L = float(d["lx"])
    with HosField(64, 64, order=5, lx=L, ly=L, g=9.81, rampflg=1, tramp=200.0) as f:
        f.set_state_physical(d["eta0"], d["phi0"])
        f.step(0.2, 20)
        u, t = f.state_spectral()
        _, H = f.energy_history()
    assert rel(u, d["u20"]) < TOL_STEPS
    assert np.max(np.abs(H - d["ham"])) / np.max(np.abs(d["ham"])) < TOL_STEPS


@pytest.mark.parametrize("M,nx,ny", [(4, 512, 512), (5, 256, 128), (3, 128, 256), (6, 64, 64), (7, 32, 32)])
def test_rhs_random_sizes_vs_restatement(M, nx, ny):
    rng = np.random.default_rng(M * 1000 + nx)
    hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, M)
    u = 1e-3 * (rng.standard_normal((2, ny // 2 + 1, nx)) + 1j * rng.standard_normal((2, ny // 2 + 1, nx)))
    u[0] = hn.Dealias(u[0])
    u[1] = hn.Dealias(u[1])
    with HosField(nx, ny, order=M) as f:
        r = f.rhs(u, 0.0)
    re_, rp = hn.rhs(u[0], u[1], 0.0)
    assert rel(r[0], re_) < TOL_OP
    assert rel(r[1], rp) < TOL_OP


def test_non_dealiased_state_steps_vs_restatement():
    """A state with content beyond the dealias bounds exercises the kx quirk
    and the c2r projection on every pass."""
    rng = np.random.default_rng(5)
    nx, ny, M = 32, 32, 3
    hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, M)
    u = 1e-3 * (rng.standard_normal((2, 17, 32)) + 1j * rng.standard_normal((2, 17, 32)))
    e, p, t = u[0].copy(), u[1].copy(), 0.0
    for _ in range(3):
        e, p, t, _h = hn.step(e, p, t, 0.05, 2)
    with HosField(nx, ny, order=M) as f:
        f.set_state_spectral(u, 0.0)
        f.step(0.05, 3)
        g, _ = f.state_spectral()
    assert rel(g[0], e) < TOL_STEPS and rel(g[1], p) < TOL_STEPS


def test_finite_depth_rhs_vs_restatement():
    rng = np.random.default_rng(8)
    nx = ny = 64
    for M in (3, 5):
        hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, M, depth=0.3)
        u = 1e-3 * (rng.standard_normal((2, 33, 64)) + 1j * rng.standard_normal((2, 33, 64)))
        u[0], u[1] = hn.Dealias(u[0]), hn.Dealias(u[1])
        with HosField(nx, ny, order=M, depth=0.3) as f:
            r = f.rhs(u, 0.0)
        re_, rp = hn.rhs(u[0], u[1], 0.0)
        assert rel(r[0], re_) < TOL_OP and rel(r[1], rp) < TOL_OP


def test_dealias_override_vs_restatement():
    rng = np.random.default_rng(9)
    nx = ny = 64
    hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, 4, mx=21, my=21)
    u = 1e-3 * (rng.standard_normal((2, 33, 64)) + 1j * rng.standard_normal((2, 33, 64)))
    u[0], u[1] = hn.Dealias(u[0]), hn.Dealias(u[1])
    with HosField(nx, ny, order=4, mx=21, my=21) as f:
        assert f.bounds == (21, 21)
        r = f.rhs(u, 0.0)
    re_, rp = hn.rhs(u[0], u[1], 0.0)
    assert rel(r[0], re_) < TOL_OP and rel(r[1], rp) < TOL_OP


def test_fp32_form_error_is_small():
    """FP32 transforms/products with FP64 state: 200 RK4 steps of a JONSWAP
    sea stay within 1e-5 Hs of the FP64 run."""
    nx = ny = 128
    eta, phi, info = ic.jonswap(nx, ny, kp=12.0, steepness=0.1, seed=3)
    dt = info["Tp"] / 50
    out = {}
    for prec in ("fp64", "fp32"):
        with HosField(nx, ny, order=5, precision=prec) as f:
            f.set_state_physical(eta, phi)
            f.step(dt, 200)
            out[prec] = f.state_physical()
    err = np.max(np.abs(out["fp32"][0] - out["fp64"][0]))
    assert err < 1e-5 * info["Hs"], err


def test_deterministic_and_volume_conserved():
    eta, phi, info = ic.jonswap(64, 64, kp=8.0, steepness=0.1, seed=4)
    res = []
    for _ in range(2):
        with HosField(64, 64, order=4) as f:
            f.set_state_physical(eta, phi)
            v0 = f.volume()
            f.step(info["Tp"] / 50, 30)
            u, _ = f.state_spectral()
            assert abs(f.volume() - v0) < 1e-15
            assert f.is_finite()
            res.append(u)
    assert np.array_equal(res[0], res[1])


def test_volume_of_offset_sea_vs_reference():
    """A sea with a non-zero mean level (JONSWAP plus a constant offset of
    0.2 Hs): the volume eta-hat(0,0) after 30 RK4 steps equals the
    reference's to 1e-12 relative to the offset."""
    n, M = 64, 3
    eta, phi, info = ic.jonswap(n, n, kp=8.0, steepness=0.1, seed=12)
    off = 0.2 * info["Hs"]
    eta = eta + off
    dt = info["Tp"] / 50
    ref_u, _ = _reference_steps(M, n, eta, phi, dt, 30)
    with HosField(n, n, order=M) as f:
        f.set_state_physical(eta, phi)
        assert abs(f.volume() - off) < 1e-15
        f.step(dt, 30)
        u, _ = f.state_spectral()
        v = f.volume()
    assert abs(ref_u[0][0, 0].real - off) < 1e-3 * off  # the reference keeps the mean level
    assert abs(v - ref_u[0][0, 0].real) <= 1e-12 * off
    assert abs(u[0][0, 0] - ref_u[0][0, 0]) <= 1e-12 * off


def test_nonfinite_state_is_reported():
    with HosField(32, 32) as f:
        u = np.zeros((2, 17, 32), complex)
        u[0, 0, 1] = np.nan
        f.set_state_spectral(u)
        assert not f.is_finite()


def test_bad_arguments_raise():
    from hos_b200 import HosError

    with pytest.raises(HosError):
        HosField(48, 64)
    with pytest.raises(HosError):
        HosField(64, 64, order=9)
    with pytest.raises(HosError):
        HosField(64, 64, scheme=7)


def _reference_steps(M, n, eta, phi, dt, nsteps):
    """Spectral state after nsteps RK4 steps by the reference's own code (C
    oracle) where it is built, else by the numpy restatement."""
    from oracle import ref_c

    if ref_c.available(M):
        ref = ref_c.RefC(M, n, n, scheme=2)
        u = ref.init_state(eta, phi)
        u, _, ham = ref.steps(u, 0.0, dt, nsteps)
        return u, ham
    hn = HosNumpy(n, n, 2 * math.pi, 2 * math.pi, 1.0, M)
    e, p = hn.init_state(eta, phi)
    t, H = 0.0, []
    for _ in range(nsteps):
        e, p, t, h = hn.step(e, p, t, dt, 2)
        H.append(h)
    return np.stack([e, p]), np.array(H)


@pytest.mark.parametrize("n,M,nsteps", [(512, 3, 8), (1024, 5, 3)])
def test_multistep_large_grid_vs_reference(n, M, nsteps):
    """Multi-step runs at the grid sizes where blocks of one launch race on
    the state if the final RK update is not isolated from the stage input."""
    eta, phi, info = ic.jonswap(n, n, kp=24.0 * n / 1024, steepness=0.12, seed=7)
    dt = info["Tp"] / 50
    ref_u, ref_h = _reference_steps(M, n, eta, phi, dt, nsteps)
    with HosField(n, n, order=M) as f:
        f.set_state_physical(eta, phi)
        f.step(dt, nsteps)
        u, _ = f.state_spectral()
        _, H = f.energy_history()
    assert rel(u[0], ref_u[0]) < TOL_STEPS and rel(u[1], ref_u[1]) < TOL_STEPS
    assert np.max(np.abs(H - ref_h)) / np.max(np.abs(ref_h)) < TOL_STEPS


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_bitwise_deterministic_1024(prec):
    eta, phi, info = ic.jonswap(1024, 1024, kp=24.0, steepness=0.12, seed=2)
    out = []
    for _ in range(2):
        with HosField(1024, 1024, order=5, precision=prec) as f:
            f.set_state_physical(eta, phi)
            f.step(info["Tp"] / 50, 40)
            out.append(f.state_spectral()[0])
    assert np.array_equal(out[0], out[1])


def test_energy_conserved_1024_m5():
    eta, phi, info = ic.jonswap(1024, 1024, kp=24.0, steepness=0.12, seed=3)
    with HosField(1024, 1024, order=5) as f:
        f.set_state_physical(eta, phi)
        f.step(info["Tp"] / 50, 200)
        _, H = f.energy_history()
    assert abs(H[-1] - H[0]) / abs(H[0]) < 1e-3


def test_one_step_2048_vs_reference():
    """The largest grid of the serving mix, one RK4 step, M = 3."""
    n = 2048
    eta, phi, info = ic.jonswap(n, n, kp=128.0, steepness=0.08, seed=9)
    dt = info["Tp"] / 50
    ref_u, ref_h = _reference_steps(3, n, eta, phi, dt, 1)
    with HosField(n, n, order=3) as f:
        f.set_state_physical(eta, phi)
        f.step(dt, 1)
        u, _ = f.state_spectral()
    assert rel(u[0], ref_u[0]) < TOL_STEPS and rel(u[1], ref_u[1]) < TOL_STEPS


def test_adaptive_rk45_matches_restatement():
    """hos_step_adaptive against the restated step control (oracle/hos_np.py:
    advance_adaptive): the same kept and rejected steps, the same next dt,
    and the state and the kept steps' energies to 1e-10."""
    n, M = 64, 4
    eta, phi, info = ic.jonswap(n, n, kp=8.0, steepness=0.1, seed=31)
    tp = info["Tp"]
    hn = HosNumpy(n, n, 2 * math.pi, 2 * math.pi, 1.0, M)
    e, p = hn.init_state(eta, phi)
    # a first step far too large: the controller must reject and shrink it
    re, rp, rt, rdt, rH, racc, rrej = hn.advance_adaptive(e, p, 0.0, tp, 2.0 * tp, 1e-7, 1e-14)
    assert rrej >= 1
    with HosField(n, n, order=M, scheme="rk45") as f:
        f.set_state_physical(eta, phi)
        dt, acc, rej = f.step_adaptive(tp, 2.0 * tp, rtol=1e-7, atol=1e-14)
        u, t = f.state_spectral()
        _, H = f.energy_history()
    assert (acc, rej) == (racc, rrej)
    assert abs(dt - rdt) <= 1e-9 * rdt
    assert abs(t - rt) <= 1e-12 * tp
    assert rel(u[0], re) < TOL_STEPS and rel(u[1], rp) < TOL_STEPS
    assert len(H) == acc and np.max(np.abs(H - rH)) / np.max(np.abs(rH)) < TOL_STEPS
