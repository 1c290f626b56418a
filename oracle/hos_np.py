"""Numpy FP64 restatement of the reference HOS hot path.

TEST INFRASTRUCTURE ONLY.  This module is an independent second oracle: it
restates, operator by operator, the reference code in Csource/2dpar so that
the C oracle (the reference's own sources compiled against the shim in
oracle/shim, see oracle/Makefile) can be cross-checked, and so that variants
the C sources cannot express without editing them (a dealias bound other than
the reference's, finite depth) have a CPU reference too.  Only tests/, the
smoke check and the bench's CPU baseline leg import it.

Layouts follow the reference's single-rank TRANSPOSED_OUT convention:
physical fields are [Nx, Ny] (x major), spectral fields are complex
[Ny//2+1, Nx] (ky major, kx contiguous), normalised by 1/(Nx*Ny) on the
forward transform (fft_routines_2d_par.c:53-55) and unnormalised on the
inverse.

Parity status: pinned.  At every size the tests use this restatement agrees
with the C oracle built from the reference's own sources (tests/test_oracle.py).
The finite-depth operator and the dealias override have no counterpart in the
reference (parity unpinned for those two variants only).
"""
from __future__ import annotations

import math

import numpy as np

# Butcher tables of Setup_TimeScheme (time_schemes_par.c:127-314).
# scheme id -> (b lower-triangular stage matrix, c final weights)
_SCHEMES = {
    1: (  # Dormand-Prince RK45, 4th-order weights used (time_schemes_par.c:183-235)
        [
            [],
            [1.0 / 5.0],
            [3.0 / 40.0, 9.0 / 40.0],
            [44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0],
            [19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0],
            [9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0],
            [35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0],
        ],
        [1951.0 / 21600.0, 0.0, 22642.0 / 50085.0, 451.0 / 720.0, -12231.0 / 42400.0, 649.0 / 6300.0, 1.0 / 60.0],
    ),
    2: (  # classical RK4 (time_schemes_par.c:243-261)
        [[], [0.5], [0.0, 0.5], [0.0, 0.0, 1.0]],
        [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0],
    ),
    3: ([[]], [1.0]),  # Euler (time_schemes_par.c:270-274)
    4: ([[], [0.5]], [0.0, 1.0]),  # midpoint (time_schemes_par.c:280-288)
    5: ([[], [1.0]], [0.5, 0.5]),  # Heun (time_schemes_par.c:294-302)
}


# 5th-order weights of the RK45 pair (time_schemes_par.c:225-231); the
# reference computes them and never uses them.
RK45_CS = [35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0]


def butcher(scheme: int):
    """Return (b, c) for a reference scheme id; b[s][p] for p < s."""
    if scheme not in _SCHEMES:
        raise ValueError(f"unknown time scheme {scheme}")
    b, c = _SCHEMES[scheme]
    return [list(row) for row in b], list(c)


class HosNumpy:
    """FP64 restatement of operators_par.c, hosm_2d_par.c and time_schemes_par.c.

    M is the HOS order (NLevs = M - 1, euler_2d_par.h:24).  ``mx``/``my``
    override the dealias bounds of operators_par.c:290-291; ``depth`` (None
    for deep water) selects the finite-depth z-derivative, which the
    reference does not implement (operators_par.c:140-166 is dead code).
    """

    def __init__(self, nx, ny, lx, ly, g, M, rampflg=0, tramp=1.0, mx=None, my=None, depth=None):
        self.nx, self.ny = int(nx), int(ny)
        self.lx, self.ly, self.g = float(lx), float(ly), float(g)
        self.M = int(M)
        self.L = self.M - 1
        self.rampflg = int(rampflg)
        self.tramp = float(tramp)
        self.depth = depth
        kx0 = 2 * math.pi / self.lx  # hdf5_routines_2d_par.c:98
        ky0 = 2 * math.pi / self.ly
        i = np.arange(self.nx)
        # operators_par.c:55-63 -- note i <= Nx/2+1 counts as positive
        kx = np.where(i <= self.nx // 2 + 1, i * kx0, -(self.nx - i) * kx0)
        ky = np.arange(self.ny // 2 + 1) * ky0  # operators_par.c:110
        self.kx = kx[None, :] * np.ones((self.ny // 2 + 1, 1))
        self.ky = ky[:, None] * np.ones((1, self.nx))
        self.kz = np.sqrt(self.kx * self.kx + self.ky * self.ky)  # operators_par.c:173-176
        if mx is None:
            mx = math.floor(0.5 * self.nx / (1 + 0.5 * self.L))  # operators_par.c:290
        if my is None:
            my = math.floor(0.5 * self.ny / (1 + 0.5 * self.L))  # operators_par.c:291
        self.mx, self.my = int(mx), int(my)
        ii = np.arange(self.nx)[None, :]
        jj = np.arange(self.ny // 2 + 1)[:, None]
        zero = ((ii >= self.mx) & (ii < self.nx - self.mx + 1)) | (jj >= self.my)  # operators_par.c:314
        self.keep = ~zero
        self.coeff = [float(math.factorial(n)) for n in range(self.L + 1)]  # hosm_2d_par.c:89-95

    # ---- transforms (fft_routines_2d_par.c) ----
    def fft2(self, u):
        """Normalised r2c, output [Ny/2+1, Nx] (fft_2d, fft_routines_2d_par.c:21-58)."""
        s = np.fft.rfft2(np.asarray(u, dtype=np.float64))  # [Nx, Ny/2+1]
        return np.ascontiguousarray(s.T) / self.nx / self.ny

    def ifft2(self, hu):
        """Unnormalised c2r (ifft_2d, fft_routines_2d_par.c:68-103).

        Complex inverse along x for every ky, then a real inverse along y that
        ignores the imaginary parts of the ky=0 and ky=Ny/2 bins.
        """
        z = np.fft.ifft(np.asarray(hu, dtype=np.complex128), axis=1) * self.nx  # [ky, ix]
        zt = np.ascontiguousarray(z.T)  # [ix, ky]
        zt[:, 0] = zt[:, 0].real
        zt[:, -1] = zt[:, -1].real
        return np.fft.irfft(zt, n=self.ny, axis=1) * self.ny

    # ---- operators (operators_par.c) ----
    def Dx(self, hu):
        return 1j * self.kx * hu

    def Dy(self, hu):
        return 1j * self.ky * hu

    def dz_mult(self, order):
        """Multiplier of the order-th z-derivative.  Deep water: kz**order.
        Finite depth (no reference counterpart): odd orders carry one
        tanh(kz h) factor, even orders none."""
        m = self.kz**order
        if self.depth is not None and order % 2 == 1:
            m = m * np.tanh(self.kz * self.depth)
        return m

    def Dz(self, hu):
        return self.kz * hu if self.depth is None else self.kz * np.tanh(self.kz * self.depth) * hu

    def Mult(self, a, b):
        return self.fft2(self.ifft2(a) * self.ifft2(b))

    def Dealias(self, hu):
        return np.where(self.keep, hu, 0.0)

    @staticmethod
    def RampFun(t, tramp):
        return 1 - math.exp(-t * t / tramp / tramp)  # hosm_2d_par.c:526-530

    # ---- model (hosm_2d_par.c) ----
    def Zvel(self, heta, hphi):
        """Zvel (hosm_2d_par.c:240-445); returns (hwM, hwM2, hw2M, hw2M2).

        For finite depth the in-place repeated Dz of hosm_2d_par.c:326 is
        replaced by tracking each level's derivative count, so that every
        derivative order gets its even/odd tanh factor exactly once.
        """
        L = self.L
        C = self.coeff
        shape = heta.shape
        hetan = [np.zeros(shape, complex) for _ in range(L + 1)]
        hetan[0][0, 0] = 1.0  # hosm_2d_par.c:276-278
        phin = [np.zeros(shape, complex) for _ in range(L + 1)]  # underived phi^(m+1)
        order = [0] * (L + 1)  # derivative count currently applied to level m
        hwn = [np.zeros(shape, complex) for _ in range(L + 1)]
        phin[0] = hphi.copy()
        order[0] = 1
        hwn[0] = self.dz_mult(1) * phin[0]  # hosm_2d_par.c:280-288

        def derived(m):
            return self.dz_mult(order[m]) * phin[m]

        for n in range(1, L + 1):
            hetan[n] = self.Mult(heta, hetan[n - 1])  # :297
            for m in range(n):  # :302-317
                phin[n] = phin[n] - self.Mult(derived(m), hetan[n - m]) / C[n - m]
            for m in range(n + 1):  # :322-357
                order[m] += 1
                hwn[n] = hwn[n] + self.Mult(derived(m), hetan[n - m]) / C[n - m]
        zero = np.zeros(shape, complex)
        hwM2 = zero.copy()
        for n in range(0, L - 1):  # :362-370
            hwM2 = hwM2 + hwn[n]
        hwM = hwM2.copy()
        for n in range(L - 1, L + 1):  # :373-394
            if n >= 0:
                hwM = hwM + hwn[n]
        hw2M2 = zero.copy()
        for n in range(0, L - 2):  # :397-416
            for m in range(n + 1):
                hw2M2 = hw2M2 + self.Mult(hwn[m], hwn[n - m])
        hw2M = hw2M2.copy()
        for n in range(L - 2, L):  # :420-442
            for m in range(n + 1):
                hw2M = hw2M + self.Mult(hwn[m], hwn[n - m])
        return hwM, hwM2, hw2M, hw2M2

    def rhs(self, heta, hphi, t):
        """rhs_hos (hosm_2d_par.c:138-235); returns (heta_t, hphi_t)."""
        g = self.g
        r_eta = -self.Mult(self.Dx(heta), self.Dx(hphi)) - self.Mult(self.Dy(heta), self.Dy(hphi))
        hwM, hwM2, hw2M, hw2M2 = self.Zvel(heta, hphi)
        grad2 = self.Mult(self.Dx(heta), self.Dx(heta)) + self.Mult(self.Dy(heta), self.Dy(heta))
        r_eta = r_eta + (hwM + self.Mult(grad2, hwM2))
        t2 = hw2M + self.Mult(grad2, hw2M2)
        r_phi = -g * heta + 0.5 * t2
        gphi = self.Mult(self.Dx(hphi), self.Dx(hphi)) + self.Mult(self.Dy(hphi), self.Dy(hphi))
        r_phi = r_phi - 0.5 * gphi
        if self.rampflg == 1:  # :211-229
            lin = self.Dz(hphi)
            R = self.RampFun(t, self.tramp)
            r_eta = (r_eta - lin) * R + lin
            r_phi = (r_phi + g * heta) * R - g * heta
        return self.Dealias(r_eta), self.Dealias(r_phi)

    def hamiltonian(self, heta, heta_t, hphi):
        """Hamiltonian (hosm_2d_par.c:462-523); row ky=0 weight 1, others 2."""
        w = np.full((heta.shape[0], 1), 2.0)
        w[0] = 1.0
        term = self.g * (heta.real**2 + heta.imag**2) + hphi.real * heta_t.real + hphi.imag * heta_t.imag
        return float(np.sum(w * term))

    def init_state(self, eta, phi):
        """main_2d_par.c:258-262: transform and dealias both fields."""
        return self.Dealias(self.fft2(eta)), self.Dealias(self.fft2(phi))

    def step(self, heta, hphi, t, dt, scheme=2):
        """One call of sol_update_RK (time_schemes_par.c:28-121).

        Every stage is evaluated at the step-start time t (:70).  Returns
        (heta, hphi, t + dt, H) with H the stage-0 Hamiltonian (:73-74).
        """
        b, c = butcher(scheme)
        ks = []
        H = None
        for s in range(len(c)):
            ue, up = heta.copy(), hphi.copy()
            for p in range(s):
                ue = ue + dt * b[s][p] * ks[p][0]
                up = up + dt * b[s][p] * ks[p][1]
            k = self.rhs(ue, up, t)
            if s == 0:
                H = self.hamiltonian(heta, k[0], hphi)
            ks.append(k)
        ne, npf = heta.copy(), hphi.copy()
        for s in range(len(c)):
            ne = ne + dt * c[s] * ks[s][0]
            npf = npf + dt * c[s] * ks[s][1]
        self.last_stages = ks
        return ne, npf, t + dt, H

    def advance_adaptive(self, heta, hphi, t, t_end, dt, rtol, atol, max_steps=100000):
        """Adaptive steps with the RK45 pair, the step control of the
        library's hos_step_adaptive restated: update with the 4th-order
        weights c (as scheme 1 of the reference), error e = dt sum (c - cs) k,
        keep the step when max|e| <= atol + rtol max|u_new|, next step
        dt * min(5, max(0.2, 0.9 (max|e|/tol)^(-1/5))), the last one shortened
        to land on t_end.  Returns (heta, hphi, t, next dt, kept energies,
        kept, rejected)."""
        _, c = butcher(1)
        span = max(abs(t_end), abs(t))
        acc = rej = 0
        H = []
        while t_end - t > 1e-12 * span and acc + rej < max_steps:
            dts = min(dt, t_end - t)
            ne, npf, _, h = self.step(heta, hphi, t, dts, 1)
            ks = self.last_stages
            ee = sum(dts * (c[s] - RK45_CS[s]) * ks[s][0] for s in range(7))
            ep = sum(dts * (c[s] - RK45_CS[s]) * ks[s][1] for s in range(7))
            me = max(np.max(np.abs(ee)), np.max(np.abs(ep)))
            mu = max(np.max(np.abs(ne)), np.max(np.abs(npf)))
            err = me / (atol + rtol * mu)
            if err <= 1.0:
                acc += 1
                heta, hphi, t = ne, npf, t + dts
                H.append(h)
            else:
                rej += 1
            fac = 5.0 if err == 0.0 else min(5.0, max(0.2, 0.9 * err ** -0.2))
            dt = dts * fac
        return heta, hphi, t, dt, np.array(H), acc, rej
