"""ctypes binding of libhos_gpu.so (declared in include/hos_gpu.h).

The library is loaded from the package directory, where `make -C
hos_b200/csrc` (or ``__graft_entry__.build()``) puts it.  There is no
fallback: if the shared object is missing or fails to load, importing the
package's compute API raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhos_gpu.so")

HOS_OK = 0
HOS_ERR_ARG = 1
HOS_ERR_CUDA = 2
HOS_ERR_NOMEM = 3
HOS_ERR_NONFINITE = 4
HOS_ERR_STATE = 5
HOS_ERR_TIMEOUT = 6
HOS_ERR_BUSY = 7

HOS_PREC_FP64 = 0
HOS_PREC_FP32 = 1

HOS_RK45DP, HOS_RK4, HOS_EULER, HOS_MIDPOINT, HOS_HEUN = 1, 2, 3, 4, 5


class HosParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("lx", ctypes.c_double),
        ("ly", ctypes.c_double),
        ("g", ctypes.c_double),
        ("order", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("depth", ctypes.c_double),
        ("rampflg", ctypes.c_int),
        ("tramp", ctypes.c_double),
        ("scheme", ctypes.c_int),
        ("mx", ctypes.c_int),
        ("my", ctypes.c_int),
        ("tune", ctypes.c_int * 8),
        ("tune_opb", ctypes.c_int),
        ("tune_nofuse", ctypes.c_int),
        ("tune_ys", ctypes.c_int),
        ("tune_sys", ctypes.c_int),
    ]


class HosPassStat(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches_per_stage", ctypes.c_int),
        ("ms_per_launch", ctypes.c_double),
        ("bytes_per_launch", ctypes.c_double),
    ]


class HosError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hos error {code}: {msg}")
        self.code = code


_lock = threading.Lock()
_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_H = ctypes.c_void_p

_SIGNATURES = {
    "hos_default_params": (None, [ctypes.POINTER(HosParams), _I, _I]),
    "hos_create": (_I, [ctypes.POINTER(HosParams), ctypes.POINTER(_H)]),
    "hos_destroy": (_I, [_H]),
    "hos_footprint_bytes": (ctypes.c_size_t, [ctypes.POINTER(HosParams)]),
    "hos_device_free_bytes": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t)]),
    "hos_get_bounds": (_I, [_H, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "hos_set_state_spectral": (_I, [_H, _P, _D]),
    "hos_get_state_spectral": (_I, [_H, _P, _DP]),
    "hos_set_state_physical": (_I, [_H, _P, _P, _D]),
    "hos_get_state_physical": (_I, [_H, _P, _P]),
    "hos_step": (_I, [_H, _D, _I]),
    "hos_step_adaptive": (_I, [_H, _D, ctypes.POINTER(_D), _D, _D, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "hos_sync": (_I, [_H]),
    "hos_health": (_I, [_H, ctypes.POINTER(ctypes.c_longlong)]),
    "hos_inject_alloc_failure": (None, [ctypes.c_long]),
    "hos_energy_history": (_I, [_H, _P, _P, _I, ctypes.POINTER(_I)]),
    "hos_clear_history": (_I, [_H]),
    "hos_rhs": (_I, [_H, _P, _P, _D]),
    "hos_fft_2d": (_I, [_H, _P, _P]),
    "hos_fft_2d_ld": (_I, [_H, _P, _I, _P]),
    "hos_ifft_2d_ld": (_I, [_H, _P, _P, _I]),
    "hos_zvel": (_I, [_H, _P, _P, _P, _P, _P]),
    "hos_spectral_op": (_I, [_H, _I, _P, _P, _P]),
    "hos_hamiltonian": (_I, [_H, _P, _P, _P, _DP]),
    "hos_ifft_2d": (_I, [_H, _P, _P]),
    "hos_check_finite": (_I, [_H, ctypes.POINTER(_I)]),
    "hos_volume": (_I, [_H, _DP]),
    "hos_stream": (_P, [_H]),
    "hos_profile_stage": (_I, [_H, _D, _I, ctypes.POINTER(HosPassStat), _I, ctypes.POINTER(_I)]),
    "hos_launches_per_step": (_I, [_H]),
    "hos_ensemble_create": (_I, [ctypes.POINTER(_H), ctypes.POINTER(_D), _I, ctypes.POINTER(_H)]),
    "hos_ensemble_create_ex": (_I, [ctypes.POINTER(_H), ctypes.POINTER(_D), _I, _I, ctypes.POINTER(_H)]),
    "hos_ensemble_set_wait_limit": (_I, [_H, ctypes.c_longlong]),
    "hos_ensemble_set_steps": (_I, [_H, ctypes.POINTER(_I)]),
    "hos_ensemble_get_remaining": (_I, [_H, ctypes.POINTER(_I)]),
    "hos_ensemble_withhold_dependency": (_I, [_H, _I]),
    "hos_ensemble_step": (_I, [_H, _I]),
    "hos_ensemble_sync": (_I, [_H]),
    "hos_ensemble_info": (_I, [_H, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "hos_ensemble_stream": (_P, [_H]),
    "hos_ensemble_destroy": (_I, [_H]),
    "hos_last_error": (ctypes.c_char_p, []),
    "hos_version": (ctypes.c_char_p, []),
}


def load():
    """Load libhos_gpu.so (once).  Raises if it is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C hos_b200/csrc` "
                "(the HOS library has no CPU fallback)"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc):
    if rc != HOS_OK:
        msg = load().hos_last_error()
        raise HosError(rc, msg.decode() if msg else "")
    return rc
