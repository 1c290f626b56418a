"""Python mirror of the HOS hot-path interface over libhos_gpu.so.

``HosField`` owns one handle of the C ABI (include/hos_gpu.h): one wave
field whose FP64 spectral state stays resident on the GPU.  Its methods map
onto the reference's routines:

=====================  ====================================================
HosField method        reference routine
=====================  ====================================================
``set_state_physical`` fft_2d x2 + Dealias x2 (main_2d_par.c:258-262)
``state_physical``     ifft_2d x2 (main_2d_par.c:310-311)
``step``               sol_update_RK (time_schemes_par.c:28-121), n times
``step_adaptive``      RK45 pair of Setup_TimeScheme(1) with step control
``rhs``                rhs_hos (hosm_2d_par.c:138-235)
``fft_2d``/``ifft_2d`` fft_routines_2d_par.c:21-103
``energy_history``     Hamiltonian at stage 0 (hosm_2d_par.c:462-523),
                       the record the reference appends to runtime.dat
                       (time_schemes_par.c:73-93)
=====================  ====================================================

Spectral arrays are complex128 of shape [2, ny//2+1, nx] (packed state) or
[ny//2+1, nx] (one field), i.e. the reference's TRANSPOSED_OUT layout;
physical arrays are float64 [nx, ny].
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib

_SCHEMES = {"rk45": 1, "rk4": 2, "euler": 3, "midpoint": 4, "heun": 5}
_PREC = {"fp64": 0, "fp32": 1}


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class HosField:
    def __init__(
        self,
        nx,
        ny,
        order=3,
        lx=2 * math.pi,
        ly=2 * math.pi,
        g=1.0,
        precision="fp64",
        depth=None,
        rampflg=0,
        tramp=1.0,
        scheme="rk4",
        mx=None,
        my=None,
        tune=None,
    ):
        self._lib = _lib.load()
        p = _lib.HosParams()
        self._lib.hos_default_params(ctypes.byref(p), int(nx), int(ny))
        p.lx, p.ly, p.g = float(lx), float(ly), float(g)
        p.order = int(order)
        p.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
        p.depth = float(depth) if depth else 0.0
        p.rampflg = int(rampflg)
        p.tramp = float(tramp)
        p.scheme = _SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)
        p.mx = int(mx or 0)
        p.my = int(my or 0)
        if isinstance(tune, str) and tune == "auto":
            from .autotune import tune as _autotune

            tune = _autotune(int(nx), int(ny), int(order), precision if isinstance(precision, str) else
                             ("fp32" if int(precision) else "fp64"))
        if tune is not None:
            tv = list(tune)
            for i, v in enumerate(tv[:8]):
                p.tune[i] = int(v)
            if len(tv) > 8:
                p.tune_opb = int(tv[8])
            if len(tv) > 9:
                p.tune_nofuse = int(tv[9])
            if len(tv) > 11:
                p.tune_ys, p.tune_sys = int(tv[10]), int(tv[11])
        self.params = p
        self.nx, self.ny, self.h = int(nx), int(ny), int(ny) // 2
        h = ctypes.c_void_p()
        _lib.check(self._lib.hos_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._lib.hos_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def footprint_bytes(nx, ny, order=3, precision="fp64", scheme="rk4"):
        lib = _lib.load()
        p = _lib.HosParams()
        lib.hos_default_params(ctypes.byref(p), int(nx), int(ny))
        p.order = int(order)
        p.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
        p.scheme = _SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)
        return int(lib.hos_footprint_bytes(ctypes.byref(p)))

    @property
    def bounds(self):
        mx, my = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.hos_get_bounds(self._h, ctypes.byref(mx), ctypes.byref(my)))
        return mx.value, my.value

    @property
    def stream(self):
        return self._lib.hos_stream(self._h)

    # ------------------------------------------------------------ shapes
    def _spec(self, nfields):
        return np.zeros((nfields, self.h + 1, self.nx) if nfields > 1 else (self.h + 1, self.nx), np.complex128)

    def _as_spec(self, u, nfields):
        a = np.ascontiguousarray(u, dtype=np.complex128)
        want = (nfields, self.h + 1, self.nx) if nfields > 1 else (self.h + 1, self.nx)
        if a.shape != want:
            raise ValueError(f"spectral array of shape {a.shape}, expected {want}")
        return a

    def _as_phys(self, x):
        a = np.ascontiguousarray(x, dtype=np.float64)
        if a.shape != (self.nx, self.ny):
            raise ValueError(f"physical array of shape {a.shape}, expected {(self.nx, self.ny)}")
        return a

    # ------------------------------------------------------------ state
    def set_state_physical(self, eta, phi, t=0.0):
        e, f = self._as_phys(eta), self._as_phys(phi)
        _lib.check(self._lib.hos_set_state_physical(self._h, _ptr(e), _ptr(f), float(t)))

    def set_state_spectral(self, u, t=0.0):
        a = self._as_spec(u, 2)
        _lib.check(self._lib.hos_set_state_spectral(self._h, _ptr(a), float(t)))

    def state_spectral(self):
        out = self._spec(2)
        t = ctypes.c_double()
        _lib.check(self._lib.hos_get_state_spectral(self._h, _ptr(out), ctypes.byref(t)))
        return out, t.value

    def state_physical(self):
        e = np.zeros((self.nx, self.ny))
        f = np.zeros((self.nx, self.ny))
        _lib.check(self._lib.hos_get_state_physical(self._h, _ptr(e), _ptr(f)))
        return e, f

    # ------------------------------------------------------------ time stepping
    def step(self, dt, nsteps=1):
        _lib.check(self._lib.hos_step(self._h, float(dt), int(nsteps)))

    def step_adaptive(self, t_end, dt, rtol=1e-8, atol=1e-12, max_steps=100000):
        """Adaptive RK45 steps (scheme "rk45") from the field's time to t_end;
        returns (next proposed dt, kept steps, rejected steps)."""
        d = ctypes.c_double(float(dt))
        acc, rej = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.hos_step_adaptive(self._h, float(t_end), ctypes.byref(d), float(rtol), float(atol),
                                               int(max_steps), ctypes.byref(acc), ctypes.byref(rej)))
        return d.value, acc.value, rej.value

    def sync(self):
        """Waits for queued steps; raises HosError (code HOS_ERR_NONFINITE)
        when a step's energy was NaN or Inf."""
        _lib.check(self._lib.hos_sync(self._h))

    def health(self):
        """First step whose energy was not finite, or None."""
        s = ctypes.c_longlong()
        _lib.check(self._lib.hos_health(self._h, ctypes.byref(s)))
        return None if s.value < 0 else s.value

    def energy_history(self, max_records=1 << 16):
        t = np.zeros(max_records)
        H = np.zeros(max_records)
        n = ctypes.c_int()
        _lib.check(self._lib.hos_energy_history(self._h, _ptr(t), _ptr(H), int(max_records), ctypes.byref(n)))
        return t[: n.value].copy(), H[: n.value].copy()

    def clear_history(self):
        _lib.check(self._lib.hos_clear_history(self._h))

    # ------------------------------------------------------------ operators
    def rhs(self, u, t=0.0):
        a = self._as_spec(u, 2)
        out = self._spec(2)
        _lib.check(self._lib.hos_rhs(self._h, _ptr(a), _ptr(out), float(t)))
        return out

    def zvel(self, u):
        """Zvel (hosm_2d_par.c:240-445): spectral W^(M), W^(M-2), (W^2)^(M), (W^2)^(M-2)."""
        a = self._as_spec(u, 2)
        outs = [self._spec(1) for _ in range(4)]
        _lib.check(self._lib.hos_zvel(self._h, _ptr(a), *[_ptr(o) for o in outs]))
        return outs

    def spectral_op(self, op, a, b=None):
        """Dx, Dy, Dz, Dealias, Sum, Mult of operators_par.c on one field."""
        codes = {"Dx": 0, "Dy": 1, "Dz": 2, "Dealias": 3, "Sum": 4, "Mult": 5}
        x = self._as_spec(a, 1)
        y = self._as_spec(b, 1) if b is not None else None
        out = self._spec(1)
        _lib.check(self._lib.hos_spectral_op(self._h, codes[op], _ptr(x), _ptr(y) if y is not None else None, _ptr(out)))
        return out

    def hamiltonian(self, heta, heta_t, hphi):
        a, b, c = (self._as_spec(x, 1) for x in (heta, heta_t, hphi))
        H = ctypes.c_double()
        _lib.check(self._lib.hos_hamiltonian(self._h, _ptr(a), _ptr(b), _ptr(c), ctypes.byref(H)))
        return H.value

    def fft_2d(self, x):
        a = self._as_phys(x)
        out = self._spec(1)
        _lib.check(self._lib.hos_fft_2d(self._h, _ptr(a), _ptr(out)))
        return out

    def ifft_2d(self, hu):
        a = self._as_spec(hu, 1)
        out = np.zeros((self.nx, self.ny))
        _lib.check(self._lib.hos_ifft_2d(self._h, _ptr(a), _ptr(out)))
        return out

    def is_finite(self):
        f = ctypes.c_int()
        _lib.check(self._lib.hos_check_finite(self._h, ctypes.byref(f)))
        return bool(f.value)

    def profile_stage(self, dt, reps=5):
        """Per-pass timing of one RK stage: list of dicts with name,
        launches_per_stage, ms_per_launch, bytes_per_launch."""
        arr = (_lib.HosPassStat * 16)()
        n = ctypes.c_int()
        _lib.check(self._lib.hos_profile_stage(self._h, float(dt), int(reps), arr, 16, ctypes.byref(n)))
        return [
            {
                "name": arr[i].name.decode(),
                "launches_per_stage": arr[i].launches_per_stage,
                "ms_per_launch": arr[i].ms_per_launch,
                "bytes_per_launch": arr[i].bytes_per_launch,
            }
            for i in range(n.value)
        ]

    @property
    def launches_per_step(self):
        return int(self._lib.hos_launches_per_step(self._h))

    def volume(self):
        v = ctypes.c_double()
        _lib.check(self._lib.hos_volume(self._h, ctypes.byref(v)))
        return v.value
