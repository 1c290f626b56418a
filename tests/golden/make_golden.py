"""Generates the golden fixtures in tests/golden/ from the C oracle.

The C oracle is the reference's own hot-path sources (Csource/2dpar
hosm_2d_par.c, operators_par.c, time_schemes_par.c, fft_routines_2d_par.c)
built unchanged against the single-rank FFTW-MPI shim by oracle/Makefile.
Run from the repository root after `make -C oracle`:

    python tests/golden/make_golden.py

`python tests/golden/make_golden.py large` makes the benchmark-size cases
alone (512^2 M=4 with both dealias rules, 1024^2 M=5; about ten minutes
on eight cores).

Every case stores its inputs and the oracle's outputs in one .npz file.  The
reference ships no test vectors of its own, so these fixtures are the
pinned record of what the reference code computes on seeded inputs and on
the one input file the reference ships (`python tests/golden/make_golden.py
shipped` makes that case alone).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hos_b200 import ic  # noqa: E402
from oracle.hos_np import HosNumpy  # noqa: E402
from oracle.ref_c import RefC  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def rand_state(rng, nx, ny, scale, dealias_with=None):
    h = ny // 2
    u = scale * (rng.standard_normal((2, h + 1, nx)) + 1j * rng.standard_normal((2, h + 1, nx)))
    # a physically meaningful half spectrum: the ky = 0 and ky = Ny/2 rows of
    # a real field are Hermitian in kx; random data deliberately is not, to
    # exercise the c2r projection
    if dealias_with is not None:
        u[0] = dealias_with.Dealias(u[0])
        u[1] = dealias_with.Dealias(u[1])
    return u


def save(name, **arrays):
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


def main():
    # 1. Stokes wave, 64^2, M=3, RK4 dt=T/64, 100 steps (first configuration)
    nx = ny = 64
    eta, phi, omega = ic.stokes3(nx, ny, kmode=4, ka=0.1)
    T = 2 * math.pi / omega
    dt = T / 64
    ref = RefC(3, nx, ny, g=1.0, scheme=2)
    u0 = ref.init_state(eta, phi)
    u1, t1, ham = ref.steps(u0, 0.0, dt, 100)
    save("stokes64_m3_rk4_100", eta0=eta, phi0=phi, u0=u0, u100=u1, t100=t1, ham=ham, dt=dt,
         meta=np.array([nx, ny, 3, 2]))

    # 2. fft pair, non-square 32 x 16, including a non-Hermitian spectrum
    rng = np.random.default_rng(11)
    ref = RefC(3, 32, 16)
    x = rng.standard_normal((32, 16))
    hx = ref.fft2(x)
    s = rng.standard_normal((9, 32)) + 1j * rng.standard_normal((9, 32))
    xs = ref.ifft2(s)
    save("fft_32x16", x=x, hx=hx, s=s, xs=xs)

    # 3. RHS on random states: dealiased with ramp, and not dealiased (quirk modes live)
    for (M, nx, ny, ramp, dealias, seed) in [(4, 32, 16, 1, True, 3), (3, 32, 32, 0, False, 4), (5, 64, 64, 1, True, 5),
                                             (6, 32, 64, 0, True, 6), (1, 16, 16, 0, False, 7), (2, 16, 32, 1, True, 8)]:
        rng = np.random.default_rng(seed)
        hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, M)
        u = rand_state(rng, nx, ny, 0.01, hn if dealias else None)
        ref = RefC(M, nx, ny, g=9.81 if M == 5 else 1.0, rampflg=ramp, tramp=2.0)
        r = ref.rhs(u, 0.7)
        save(f"rhs_m{M}_{nx}x{ny}_{'d' if dealias else 'nd'}_r{ramp}", u=u, rhs=r, t=0.7,
             meta=np.array([nx, ny, M, ramp]), g=9.81 if M == 5 else 1.0, tramp=2.0)

    # 3b. Zvel outputs on random states
    for (M, nx, ny, seed) in [(4, 32, 32, 31), (3, 16, 32, 32), (6, 32, 16, 33)]:
        rng = np.random.default_rng(seed)
        hn = HosNumpy(nx, ny, 2 * math.pi, 2 * math.pi, 1.0, M)
        u = rand_state(rng, nx, ny, 0.01, hn if seed != 32 else None)
        ref = RefC(M, nx, ny)
        wM, wM2, w2M, w2M2 = ref.zvel(u)
        save(f"zvel_m{M}_{nx}x{ny}", u=u, wM=wM, wM2=wM2, w2M=w2M, w2M2=w2M2, meta=np.array([nx, ny, M]))

    # 4. each RK scheme, 5 steps on a small JONSWAP sea, M=4
    nx = ny = 32
    eta, phi, info = ic.jonswap(nx, ny, kp=4.0, steepness=0.1, seed=21)
    for scheme in (1, 2, 3, 4, 5):
        ref = RefC(4, nx, ny, scheme=scheme)
        u0 = ref.init_state(eta, phi)
        dt = info["Tp"] / 50
        u5, t5, ham = ref.steps(u0, 0.0, dt, 5)
        save(f"scheme{scheme}_32_m4", eta0=eta, phi0=phi, u0=u0, u5=u5, t5=t5, ham=ham, dt=dt,
             meta=np.array([nx, ny, 4, scheme]))

    # 5. JONSWAP 64^2 M=5 with ramp, 20 RK4 steps, domain and g of the shipped case
    nx = ny = 64
    L = 3807.99
    eta, phi, info = ic.jonswap(nx, ny, lx=L, ly=L, g=9.81, kp=2 * math.pi / L * 8, steepness=0.08, seed=5)
    ref = RefC(5, nx, ny, lx=L, ly=L, g=9.81, rampflg=1, tramp=200.0, scheme=2)
    u0 = ref.init_state(eta, phi)
    u20, t20, ham = ref.steps(u0, 0.0, 0.2, 20)
    save("jonswap64_m5_ramp_20", eta0=eta, phi0=phi, u0=u0, u20=u20, t20=t20, ham=ham, dt=0.2,
         meta=np.array([nx, ny, 5, 2]), lx=L, g=9.81, tramp=200.0)

    shipped_case()


def shipped_case():
    """The reference's shipped input (Csource/2dpar/initpars.h5 and
    initdata.1.h5, 256^2 JONSWAP, read with the library's HDF5 subset) run as
    the reference's driver runs it: M = 3 (NLevs = 2), scheme 4 (midpoint),
    dt = 0.2, ramp on with Tramp = 200, to T = 50 (250 steps).  Stored: the
    dealiased initial spectrum and the final one as (row, column, value) over
    the modes the dealias mask keeps, and the energy series."""
    from hos_b200 import h5

    from oracle import REFERENCE_SRC as src
    p = h5.read_params(os.path.join(src, "initpars.h5"))
    eta = h5.read(os.path.join(src, "initdata.1.h5"), "eta0")
    phi = h5.read(os.path.join(src, "initdata.1.h5"), "phi0")
    nx, ny = p["Nx"], p["Ny"]
    ref = RefC(3, nx, ny, lx=p["Lx"], ly=p["Ly"], g=p["g"], rampflg=p["rampflg"], tramp=p["Tramp"], scheme=4)
    u0 = ref.init_state(eta, phi)
    nsteps = int(round(p["T"] / 0.2))
    u1, t1, ham = ref.steps(u0, 0.0, 0.2, nsteps)
    keep = np.nonzero(HosNumpy(nx, ny, p["Lx"], p["Ly"], p["g"], 3).Dealias(np.ones((ny // 2 + 1, nx))))
    save("shipped256_m3_mid_250", rows=keep[0].astype(np.int16), cols=keep[1].astype(np.int16),
         u0=u0[:, keep[0], keep[1]], u250=u1[:, keep[0], keep[1]], t250=t1, ham=ham, dt=0.2,
         meta=np.array([nx, ny, 3, 4, p["rampflg"]]), lx=p["Lx"], ly=p["Ly"], g=p["g"], tramp=p["Tramp"],
         eta_l2=np.linalg.norm(eta), eta_sum=eta.sum())


LARGE_CASES = {
    # name: (n, M, kp, kp*Hs/2, gamma, s, seed, dealias variant)
    "jonswap512_m4_rk4_100": (512, 4, 16.0, 0.10, 3.3, 15.0, 2, ""),
    "jonswap512_m4_d23_rk4_100": (512, 4, 16.0, 0.10, 3.3, 15.0, 2, "d23"),
    "jonswap1024_m5_rk4_100": (1024, 5, 24.0, 0.12, 3.3, 10.0, 1000, ""),
}


def large_case(name, nsteps=100):
    """A benchmark-size JONSWAP sea run 100 RK4 steps (dt = Tp/50) by the
    reference's code.  The state of the reference stays inside the dealias
    mask (the initial state is dealiased and every stage derivative is), so
    only the kept modes are stored, as (row, column, value), together with a
    checksum of the seeded initial fields so that a test regenerating them
    can tell that it got the same inputs."""
    n, M, kp, st, gamma, spread, seed, variant = LARGE_CASES[name]
    eta, phi, info = ic.jonswap(n, n, kp=kp, steepness=st, gamma=gamma, spread_s=spread, seed=seed)
    dt = info["Tp"] / 50
    ref = RefC(M, n, n, g=1.0, scheme=2, dealias=variant)
    u0 = ref.init_state(eta, phi)
    u1, t1, ham = ref.steps(u0, 0.0, dt, nsteps)
    mx = my = n // 3 if variant == "d23" else None
    hn = HosNumpy(n, n, 2 * math.pi, 2 * math.pi, 1.0, M, mx=mx, my=my)
    mask = hn.Dealias(np.ones((n // 2 + 1, n))) != 0
    assert not np.any(u1[:, ~mask]), "state outside the dealias mask"
    keep = np.nonzero(mask)
    save(name, rows=keep[0].astype(np.int16), cols=keep[1].astype(np.int16), u100=u1[:, keep[0], keep[1]],
         t100=t1, ham=ham, dt=dt, meta=np.array([n, n, M, 2, seed, hn.mx, hn.my]),
         ic=np.array([kp, st, gamma, spread]), eta_sum=eta.sum(), eta_l2=np.linalg.norm(eta),
         phi_l2=np.linalg.norm(phi), hs=info["Hs"])


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "shipped":
        shipped_case()
    elif len(sys.argv) > 1 and sys.argv[1] == "large":
        for nm in (sys.argv[2:] or LARGE_CASES):
            large_case(nm)
    else:
        main()
