"""The reference-compatible entry points (include/hos_legacy.h) driven the
way the reference's host driver drives them (main_2d_par.c:126-357):
globals set by the caller, padded physical arrays, host spectral arrays,
runtime.dat written by sol_update_RK.  Compared with the reference's own
code (the C oracle) driven identically, or with the golden fixtures."""
import ctypes
import math
import os

import numpy as np
import pytest

from hos_b200 import ic
from oracle import ref_c
from oracle.hos_np import HosNumpy

from .conftest import ROOT

pytestmark = pytest.mark.gpu
LIB = os.path.join(ROOT, "hos_b200", "libhos_gpu.so")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def lib():
    import hos_b200

    hos_b200.load()  # the package binding first: the same library object
    L = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    for name, args in {
        "Setup_TimeScheme": [ctypes.c_int], "rhs_hos_setup": [], "rhs_hos_clean": [],
        "sol_update_RK": [P, P, ctypes.c_double, P], "rhs_hos": [P, P, ctypes.c_double], "rhs_test": [P, P],
        "Zvel": [P, P, P, P, P, ctypes.c_double], "ZvelLinear": [P, P], "Hamiltonian": [P, P, P],
        "RampFun": [ctypes.c_double], "Dx": [P, P], "Dy": [P, P], "Dz": [P, P], "Mult": [P, P, P],
        "Sum": [P, P, P], "Dealias": [P], "fft_2d": [P, P, P], "ifft_2d": [P, P, P],
        "hos_legacy_set_nlevs": [ctypes.c_int], "hos_legacy_set_resident": [ctypes.c_int], "hos_legacy_sync": [],
    }.items():
        getattr(L, name).argtypes = args
    L.Hamiltonian.restype = ctypes.c_double
    L.RampFun.restype = ctypes.c_double
    return L


def set_globals(L, nx, ny, lx, ly, g, ramp, tramp, runtime):
    ctypes.c_int.in_dll(L, "Nx").value = nx
    ctypes.c_int.in_dll(L, "Ny").value = ny
    ctypes.c_double.in_dll(L, "Lx").value = lx
    ctypes.c_double.in_dll(L, "Ly").value = ly
    ctypes.c_double.in_dll(L, "Kx0").value = 2 * math.pi / lx
    ctypes.c_double.in_dll(L, "Ky0").value = 2 * math.pi / ly
    ctypes.c_double.in_dll(L, "g").value = g
    ctypes.c_int.in_dll(L, "rampflg").value = ramp
    ctypes.c_double.in_dll(L, "Tramp").value = tramp
    al = nx * (ny // 2 + 1)
    ctypes.c_ssize_t.in_dll(L, "alloc_local").value = al
    ctypes.c_ssize_t.in_dll(L, "local_N").value = al
    ctypes.c_ssize_t.in_dll(L, "local_Nyhpo").value = ny // 2 + 1
    ctypes.c_ssize_t.in_dll(L, "local_1_start").value = 0
    ctypes.c_int.in_dll(L, "mpi_rank").value = 0
    buf = (ctypes.c_char * 32).in_dll(L, "runtime_data_buff")
    buf.value = runtime.encode()


def p(a):
    return ctypes.c_void_p(a.ctypes.data)


def padded(x):
    nx, ny = x.shape
    out = np.zeros((nx, ny + 2))
    out[:, :ny] = x
    return out


def test_driver_sequence_matches_reference(lib, tmp_path, monkeypatch):
    """main_2d_par.c's sequence on a 64 x 32 JONSWAP sea, M = 4, RK4, ramp on."""
    if not ref_c.available(4):
        pytest.skip("C oracle not built")
    monkeypatch.chdir(tmp_path)  # runtime_data_buff holds 32 bytes (euler_2d_par.h:20,95)
    nx, ny, M, dt, nsteps = 64, 32, 4, 0.05, 12
    lx, ly, g, tramp = 2 * math.pi, math.pi, 9.81, 0.4
    eta, phi, _ = ic.jonswap(nx, ny, lx=lx, ly=ly, g=g, kp=6.0, steepness=0.08, seed=17)
    runtime = "runtime.dat"
    set_globals(lib, nx, ny, lx, ly, g, 1, tramp, runtime)
    lib.hos_legacy_set_nlevs(M - 1)
    lib.Setup_TimeScheme(2)
    lib.rhs_hos_setup()
    u = np.zeros((2, ny // 2 + 1, nx), complex)
    e_p, f_p = padded(eta), padded(phi)
    lib.fft_2d(p(e_p), p(u[0]), None)
    lib.fft_2d(p(f_p), p(u[1]), None)
    lib.Dealias(p(u[0]))
    lib.Dealias(p(u[1]))
    ref = ref_c.RefC(M, nx, ny, lx=lx, ly=ly, g=g, rampflg=1, tramp=tramp, scheme=2)
    u_ref = ref.init_state(eta, phi)
    assert rel(u, u_ref) < 1e-14
    # Zvel of the initial state (main_2d_par.c:264)
    outs = [np.zeros((ny // 2 + 1, nx), complex) for _ in range(4)]
    lib.Zvel(p(u), *[p(o) for o in outs], 0.0)
    want = ref.zvel(u_ref)
    for o, w in zip(outs, want):
        assert rel(o, w) < 1e-12
    t = np.zeros(1)
    for _ in range(nsteps):
        lib.sol_update_RK(p(u), p(t), dt, None)
    u_ref, t_ref, ham_ref = ref.steps(u_ref, 0.0, dt, nsteps)
    assert rel(u[0], u_ref[0]) < 1e-10 and rel(u[1], u_ref[1]) < 1e-10
    assert abs(t[0] - t_ref) < 1e-15
    lines = open(runtime).read().split("\n")[:-1]
    assert len(lines) == nsteps
    ts, hs = zip(*[(float(a), float(b)) for a, b in (ln.split("\t") for ln in lines)])
    assert np.max(np.abs(np.array(hs) - ham_ref)) / np.max(np.abs(ham_ref)) < 1e-10
    assert abs(ts[1] - dt) < 1e-9
    # output path (main_2d_par.c:310-311)
    back = np.zeros((nx, ny + 2))
    lib.ifft_2d(p(u[0]), p(back), None)
    assert rel(back[:, :ny], ref.ifft2(u_ref[0])) < 1e-10
    lib.rhs_hos_clean()


def test_resident_state_between_steps(lib, tmp_path, monkeypatch):
    """Resident mode: the state stays on the GPU across sol_update_RK calls
    (the host array is not touched), a save through ifft_2d sees the current
    state, an in-place Dealias between steps is taken up by the next step, and
    hos_legacy_sync brings the host array up to date; all as the reference's
    code computes it."""
    if not ref_c.available(3):
        pytest.skip("C oracle not built")
    monkeypatch.chdir(tmp_path)
    nx, ny, M, dt = 64, 64, 3, 0.2
    lx, g, tramp = 600.0, 9.81, 1.0
    eta, phi, _ = ic.jonswap(nx, ny, lx=lx, ly=lx, g=g, kp=2 * math.pi / lx * 6, steepness=0.08, seed=23)
    set_globals(lib, nx, ny, lx, lx, g, 1, tramp, "runtime.dat")
    lib.hos_legacy_set_nlevs(M - 1)
    lib.Setup_TimeScheme(4)
    lib.rhs_hos_setup()
    lib.hos_legacy_set_resident(1)
    try:
        u = np.zeros((2, ny // 2 + 1, nx), complex)
        e_p, f_p = padded(eta), padded(phi)  # held: the library reads them during the calls
        lib.fft_2d(p(e_p), p(u[0]), None)
        lib.fft_2d(p(f_p), p(u[1]), None)
        lib.Dealias(p(u[0]))
        lib.Dealias(p(u[1]))
        ref = ref_c.RefC(M, nx, ny, lx=lx, ly=lx, g=g, rampflg=1, tramp=tramp, scheme=4)
        u_ref = ref.init_state(eta, phi)
        u0 = u.copy()
        t = np.zeros(1)
        for _ in range(5):
            lib.sol_update_RK(p(u), p(t), dt, None)
        assert np.array_equal(u, u0)  # still on the GPU
        u_ref, t_ref, _ = ref.steps(u_ref, 0.0, dt, 5)
        back = np.zeros((nx, ny + 2))
        lib.ifft_2d(p(u[0]), p(back), None)  # the save path syncs the host copy first
        assert rel(back[:, :ny], ref.ifft2(u_ref[0])) < 1e-10
        assert rel(u[1], u_ref[1]) < 1e-10
        # a write between steps: Dealias(phi) in place (the identity on a dealiased state)
        lib.Dealias(p(u[1]))
        for _ in range(5):
            lib.sol_update_RK(p(u), p(t), dt, None)
        u_ref, t_ref, _ = ref.steps(u_ref, t_ref, dt, 5)
        lib.hos_legacy_sync()
        assert rel(u[0], u_ref[0]) < 1e-10 and rel(u[1], u_ref[1]) < 1e-10
        assert abs(t[0] - t_ref) < 1e-15
        assert len(open("runtime.dat").read().split("\n")[:-1]) == 10
    finally:
        lib.hos_legacy_set_resident(0)
        lib.rhs_hos_clean()


def test_operators_match_reference(lib, tmp_path, monkeypatch):
    if not ref_c.available(3):
        pytest.skip("C oracle not built")
    monkeypatch.chdir(tmp_path)
    nx, ny, M = 32, 32, 3
    set_globals(lib, nx, ny, 2 * math.pi, 2 * math.pi, 1.0, 1, 2.0, "runtime.dat")
    lib.hos_legacy_set_nlevs(M - 1)
    lib.Setup_TimeScheme(2)
    ref = ref_c.RefC(M, nx, ny, rampflg=1, tramp=2.0)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((17, 32)) + 1j * rng.standard_normal((17, 32))
    b = rng.standard_normal((17, 32)) + 1j * rng.standard_normal((17, 32))
    out = np.zeros_like(a)
    for name, fn in (("Dx", ref.lib.ref_dx), ("Dy", ref.lib.ref_dy), ("Dz", ref.lib.ref_dz)):
        getattr(lib, name)(p(a), p(out))
        w = np.zeros_like(a)
        fn(p(a), p(w))
        assert rel(out, w) < 1e-15, name
    lib.Mult(p(a), p(b), p(out))
    w = np.zeros_like(a)
    ref.lib.ref_mult(p(a), p(b), p(w))
    assert rel(out, w) < 1e-13
    lib.Sum(p(a), p(b), p(out))
    assert rel(out, a + b) < 1e-15
    d = a.copy()
    lib.Dealias(p(d))
    w = a.copy()
    ref.lib.ref_dealias(p(w))
    assert np.array_equal(d, w)
    u = np.stack([a, b]) * 1e-2
    r = np.zeros_like(u)
    lib.rhs_hos(p(r), p(u), 0.9)
    assert rel(r, ref.rhs(u, 0.9)) < 1e-12
    H = lib.Hamiltonian(p(u[0]), p(r[0]), p(u[1]))
    assert abs(H - ref.hamiltonian(u[0], r[0], u[1])) < 1e-13 * abs(H)
    assert abs(lib.RampFun(0.7) - ref.lib.ref_rampfun(0.7)) < 1e-16
    zl = np.zeros_like(a)
    lib.ZvelLinear(p(u), p(zl))
    w = np.zeros_like(a)
    ref.lib.ref_dz(p(u[1]), p(w))
    assert rel(zl, w) < 1e-15
    rt = np.zeros_like(u)
    lib.rhs_test(p(rt), p(u))
    wx, wy = np.zeros_like(a), np.zeros_like(a)
    ref.lib.ref_dx(p(u[0]), p(wx))
    ref.lib.ref_dy(p(u[1]), p(wy))
    assert rel(rt[0], wx) < 1e-15 and rel(rt[1], wy) < 1e-15


@pytest.mark.parametrize("name", ["zvel_m4_32x32", "zvel_m3_16x32", "zvel_m6_32x16"])
def test_zvel_matches_golden(golden, name):
    from hos_b200 import HosField

    d = golden(name)
    nx, ny, M = (int(v) for v in d["meta"])
    with HosField(nx, ny, order=M) as f:
        outs = f.zvel(d["u"])
    for o, k in zip(outs, ("wM", "wM2", "w2M", "w2M2")):
        assert rel(o, d[k]) < 1e-12, k
