"""Ensembles: many independent wave fields advanced together on one GPU.

``HosEnsemble`` groups existing ``HosField`` handles (any grid, order,
precision, depth and time step).  Members that share grid, precision and
scheme form a size class: every pass of the RK step is one kernel launch
over all members of the class, and a whole step of all classes is one CUDA
graph with the classes on parallel streams (hos_ensemble_* in
include/hos_gpu.h).  Each member advances exactly as ``field.step(dt)``
would; the reference advances one field per process and has no
counterpart.
"""
from __future__ import annotations

import ctypes

from . import _lib


class HosEnsemble:
    def __init__(self, fields, dts):
        if len(fields) != len(dts) or not fields:
            raise ValueError("one dt per field")
        self._lib = _lib.load()
        self.fields = list(fields)
        hs = (ctypes.c_void_p * len(fields))(*[f._h.value for f in fields])
        ds = (ctypes.c_double * len(fields))(*[float(d) for d in dts])
        h = ctypes.c_void_p()
        _lib.check(self._lib.hos_ensemble_create(hs, ds, len(fields), ctypes.byref(h)))
        self._h = h

    def step(self, nsteps=1):
        _lib.check(self._lib.hos_ensemble_step(self._h, int(nsteps)))

    def sync(self):
        _lib.check(self._lib.hos_ensemble_sync(self._h))

    @property
    def stream(self):
        """cudaStream_t (as an int) the step graphs run on."""
        return self._lib.hos_ensemble_stream(self._h)

    @property
    def info(self):
        nc, nl = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.hos_ensemble_info(self._h, ctypes.byref(nc), ctypes.byref(nl)))
        return {"classes": nc.value, "launches_per_step": nl.value}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hos_ensemble_destroy(self._h)
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
