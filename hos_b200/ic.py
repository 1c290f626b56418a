"""Initial conditions for the HOS benchmarks and tests (seeded, synthetic).

The reference generates its inputs offline (python/CreateSpectra.py,
python/JONSWAP.py, python/DtoF.py, matlab/InitDataGen_PowerSpec.m) and
hands them to the solver as physical eta/phi arrays (initdata.<id>.h5,
read by get_ic_2d, hdf5_routines_2d_par.c:104-191).  The generators here
produce the same kind of input -- physical eta(x, y) and surface potential
phi_s(x, y) on an [nx, ny] grid -- from the published formulas:

* ``stokes3``: long-crested third-order deep-water Stokes wave
  (Stokes 1847; e.g. Whitham, Linear and Nonlinear Waves, sec. 13.13):
  eta = a cos q + (k a^2 / 2) cos 2q + (3 k^2 a^3 / 8) cos 3q,
  omega^2 = g k (1 + (k a)^2), and the deep-water potential, which carries
  only the first harmonic to third order, evaluated on the surface:
  phi_s = (a omega / k) exp(k eta) sin q.
* ``jonswap``: directional JONSWAP sea (Hasselmann et al. 1973) with
  Longuet-Higgins cos^(2s)(theta/2) spreading, complex-Gaussian mode
  amplitudes (Rayleigh magnitudes, uniform phases) from a seeded generator,
  rescaled to the target significant wave height Hs = 4 std(eta), and the
  linear surface potential phi_hat = -i (g / omega) eta_hat of each
  wave component (omega^2 = g k tanh(k h)); the mean and Nyquist modes are
  zero (as InitDataGen_PowerSpec.m:55-60 does).
"""
from __future__ import annotations

import math

import numpy as np


def stokes3(nx, ny, lx=2 * math.pi, ly=2 * math.pi, g=1.0, kmode=4, ka=0.1):
    """Third-order Stokes wave travelling in +x.  Returns (eta, phi, omega)
    with eta, phi of shape [nx, ny] (x major)."""
    k = 2 * math.pi * kmode / lx
    a = ka / k
    x = np.arange(nx) * (lx / nx)
    q = k * x
    eta1 = a * np.cos(q) + 0.5 * k * a * a * np.cos(2 * q) + 3.0 / 8.0 * k * k * a**3 * np.cos(3 * q)
    omega = math.sqrt(g * k * (1 + (k * a) ** 2))
    phi1 = (a * omega / k) * np.exp(k * eta1) * np.sin(q)
    eta = np.repeat(eta1[:, None], ny, axis=1)
    phi = np.repeat(phi1[:, None], ny, axis=1)
    return np.ascontiguousarray(eta), np.ascontiguousarray(phi), omega


def jonswap(
    nx,
    ny,
    lx=2 * math.pi,
    ly=2 * math.pi,
    g=1.0,
    kp=16.0,
    steepness=0.1,
    gamma=3.3,
    spread_s=15.0,
    seed=0,
    depth=None,
    theta0=0.0,
):
    """Directional JONSWAP sea.  ``kp`` is the peak wavenumber, ``steepness``
    is kp*Hs/2.  Returns (eta, phi, info) with eta, phi [nx, ny] and info a
    dict holding Hs, Tp (peak period), omega_p and the seed."""
    rng = np.random.default_rng(seed)
    kx = 2 * math.pi / lx * np.fft.fftfreq(nx, d=1.0 / nx)
    ky = 2 * math.pi / ly * np.fft.fftfreq(ny, d=1.0 / ny)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")  # [nx, ny]
    K = np.hypot(KX, KY)

    def omega_of(k):
        kk = np.maximum(k, 1e-300)
        return np.sqrt(g * kk * (np.tanh(kk * depth) if depth else 1.0))

    wp = float(omega_of(np.array(kp)))
    W = omega_of(K)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        sigma = np.where(W <= wp, 0.07, 0.09)
        r = np.exp(-((W - wp) ** 2) / (2 * sigma**2 * wp**2))
        Sw = g * g * W**-5 * np.exp(-1.25 * (wp / W) ** 4) * gamma**r
        # dω/dk for the dispersion relation in use (numerical derivative-free form)
        if depth:
            th = np.tanh(K * depth)
            dwdk = g * (th + K * depth * (1 - th * th)) / (2 * W)
        else:
            dwdk = 0.5 * np.sqrt(g / np.maximum(K, 1e-300))
        Sk = Sw * dwdk
        theta = np.arctan2(KY, KX) - theta0
        D = np.cos(0.5 * theta) ** (2 * spread_s)
        F = Sk * D / K
    F = np.where(np.isfinite(F) & (K > 0), F, 0.0)
    # zero the Nyquist rows/columns
    F[nx // 2, :] = 0.0
    F[:, ny // 2] = 0.0
    dkx = 2 * math.pi / lx
    dky = 2 * math.pi / ly
    amp = np.sqrt(2 * F * dkx * dky)
    xi = (rng.standard_normal(F.shape) + 1j * rng.standard_normal(F.shape)) / math.sqrt(2.0)
    A = amp * xi
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(K > 0, -1j * g / np.maximum(W, 1e-300) * A, 0.0)
    eta = np.real(np.fft.ifft2(A) * (nx * ny))
    phi = np.real(np.fft.ifft2(P) * (nx * ny))
    hs_target = 2.0 * steepness / kp
    std = float(np.std(eta))
    scale = hs_target / (4.0 * std) if std > 0 else 0.0
    eta *= scale
    phi *= scale
    info = {"Hs": hs_target, "Tp": 2 * math.pi / wp, "omega_p": wp, "seed": seed, "kp": kp}
    return np.ascontiguousarray(eta), np.ascontiguousarray(phi), info
