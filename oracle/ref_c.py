"""ctypes driver of the C oracle oracle/_ref/libhosref_M<M>.so.

TEST INFRASTRUCTURE ONLY.  The shared object is the reference's own
hosm_2d_par.c, operators_par.c, time_schemes_par.c and fft_routines_2d_par.c
(Csource/2dpar) compiled unchanged with NLevs = M-1, linked with the
single-rank FFTW-MPI shim and oracle/ref_harness.c (see oracle/Makefile).
Each library keeps the reference's process-global state, so one RefC object
per order is live at a time; ``setup`` is re-run when the grid changes.

``dealias="d23"`` selects the build whose operators_par.c has the two
dealias bounds (operators_par.c:290-291) replaced by floor(Nx/3),
floor(Ny/3) (the "2/3 rule"; oracle/Makefile makes it for M = 4).
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.c_double
_P = ctypes.c_void_p
_libs = {}


def lib_path(M, dealias=""):
    suffix = f"_{dealias}" if dealias else ""
    return os.path.join(_HERE, "_ref", f"libhosref_M{int(M)}{suffix}.so")


def available(M=3, dealias=""):
    return os.path.exists(lib_path(M, dealias))


def _load(M, dealias=""):
    key = (M, dealias)
    if key in _libs:
        return _libs[key]
    path = lib_path(M, dealias)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference sources are present")
    lib = ctypes.CDLL(path)
    lib.ref_setup.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, ctypes.c_int, _D, ctypes.c_int]
    lib.ref_setup.restype = ctypes.c_int
    for fn in ["ref_fft_2d", "ref_ifft_2d", "ref_dx", "ref_dy", "ref_dz", "ref_dealias"]:
        getattr(lib, fn).argtypes = [_P, _P] if fn != "ref_dealias" else [_P]
    lib.ref_init_state.argtypes = [_P, _P, _P]
    lib.ref_rhs.argtypes = [_P, _P, _D]
    lib.ref_zvel.argtypes = [_P, _P, _P, _P, _P, _D]
    lib.ref_steps.argtypes = [_P, _P, _D, ctypes.c_int, _P]
    lib.ref_mult.argtypes = [_P, _P, _P]
    lib.ref_hamiltonian.argtypes = [_P, _P, _P]
    lib.ref_hamiltonian.restype = _D
    lib.ref_rampfun.argtypes = [_D]
    lib.ref_rampfun.restype = _D
    lib.ref_nlevs.restype = ctypes.c_int
    _libs[key] = lib
    return lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class RefC:
    def __init__(self, M, nx, ny, lx=2 * math.pi, ly=2 * math.pi, g=1.0, rampflg=0, tramp=1.0, scheme=2,
                 dealias=""):
        self.M = int(M)
        self.lib = _load(self.M, dealias)
        assert self.lib.ref_nlevs() == self.M - 1
        self.nx, self.ny, self.h = int(nx), int(ny), int(ny) // 2
        self.args = (self.nx, self.ny, float(lx), float(ly), float(g), int(rampflg), float(tramp), int(scheme))
        self.setup()

    def setup(self):
        rc = self.lib.ref_setup(*self.args)
        if rc != 0:
            raise ValueError(f"ref_setup failed ({rc})")

    def _spec(self, n):
        return np.zeros((n, self.h + 1, self.nx) if n > 1 else (self.h + 1, self.nx), np.complex128)

    def fft2(self, x):
        x = np.ascontiguousarray(x, np.float64)
        out = self._spec(1)
        self.lib.ref_fft_2d(_p(x), _p(out))
        return out

    def ifft2(self, hu):
        hu = np.ascontiguousarray(hu, np.complex128)
        out = np.zeros((self.nx, self.ny))
        self.lib.ref_ifft_2d(_p(hu), _p(out))
        return out

    def init_state(self, eta, phi):
        e = np.ascontiguousarray(eta, np.float64)
        f = np.ascontiguousarray(phi, np.float64)
        u = self._spec(2)
        self.lib.ref_init_state(_p(e), _p(f), _p(u))
        return u

    def rhs(self, u, t):
        u = np.ascontiguousarray(u, np.complex128)
        out = self._spec(2)
        self.lib.ref_rhs(_p(u), _p(out), float(t))
        return out

    def zvel(self, u, t=0.0):
        u = np.ascontiguousarray(u, np.complex128)
        outs = [self._spec(1) for _ in range(4)]
        self.lib.ref_zvel(_p(u), *[_p(o) for o in outs], float(t))
        return outs

    def steps(self, u, t, dt, n):
        """n calls of sol_update_RK; returns (u, t, ham[n])."""
        u = np.array(u, np.complex128, copy=True, order="C")
        tt = np.array([float(t)])
        ham = np.zeros(max(int(n), 1))
        self.lib.ref_steps(_p(u), _p(tt), float(dt), int(n), _p(ham))
        return u, float(tt[0]), ham[: int(n)]

    def hamiltonian(self, heta, heta_t, hphi):
        a = np.ascontiguousarray(heta, np.complex128)
        b = np.ascontiguousarray(heta_t, np.complex128)
        c = np.ascontiguousarray(hphi, np.complex128)
        return float(self.lib.ref_hamiltonian(_p(a), _p(b), _p(c)))
