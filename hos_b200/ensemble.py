"""Ensembles: many independent wave fields advanced together on one GPU.

``HosEnsemble`` groups existing ``HosField`` handles (any grid, order,
precision, depth and time step).  Two modes (hos_ensemble_* in
include/hos_gpu.h):

* ``"persistent"``: one RK step of all members is one launch of a
  persistent kernel; its resident blocks take work items (blocks of one pass
  of one member) from a device list in order and wait, with a bounded wait,
  for the member's earlier passes.  Grids of 64..2048 points per direction,
  default kernel shapes.
* ``"classes"``: members that share grid, precision and scheme form a size
  class; every pass of the RK step is one kernel launch over all members of
  the class, and a whole step of all classes is one CUDA graph with the
  classes on parallel streams.

In both modes members can be given step budgets: a member stops after its
own number of steps while the others go on.  Either way each member
advances exactly as ``field.step(dt)`` would; the
reference advances one field per process and has no counterpart.
"""
from __future__ import annotations

import ctypes

from . import _lib


_MODES = {"classes": 0, "persistent": 1}


class HosEnsemble:
    def __init__(self, fields, dts, mode="classes"):
        if len(fields) != len(dts) or not fields:
            raise ValueError("one dt per field")
        self._lib = _lib.load()
        self.fields = list(fields)
        self.mode = mode
        hs = (ctypes.c_void_p * len(fields))(*[f._h.value for f in fields])
        ds = (ctypes.c_double * len(fields))(*[float(d) for d in dts])
        h = ctypes.c_void_p()
        _lib.check(self._lib.hos_ensemble_create_ex(hs, ds, len(fields), _MODES[mode], ctypes.byref(h)))
        self._h = h

    def set_steps(self, steps):
        """Each member takes steps[i] more steps and then stops (-1: no
        limit), whatever number of steps is launched (either mode)."""
        arr = (ctypes.c_int * len(self.fields))(*[int(s) for s in steps])
        _lib.check(self._lib.hos_ensemble_set_steps(self._h, arr))

    def remaining(self):
        arr = (ctypes.c_int * len(self.fields))()
        _lib.check(self._lib.hos_ensemble_get_remaining(self._h, arr))
        return list(arr)

    def set_wait_limit(self, seconds):
        """Bound of one wait of the persistent kernel."""
        _lib.check(self._lib.hos_ensemble_set_wait_limit(self._h, int(seconds * 1e9)))

    def withhold_dependency(self, on=True):
        """Failure injection: one task waits for an item that never completes,
        so the next step's wait runs out (sync raises HOS_ERR_TIMEOUT)."""
        _lib.check(self._lib.hos_ensemble_withhold_dependency(self._h, 1 if on else 0))

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
