"""hos_b200: B200-native (sm_100a) time-advance hot path of the HOS water-wave
solver (reference: EsterDoesProgramming/hos, Csource/2dpar).

The compute lives in libhos_gpu.so (C ABI, include/hos_gpu.h); this package
is the Python host side: a ctypes binding (``_lib``), the field handle
(``HosField``) and the seeded initial-condition generators (``ic``).
"""
from . import ic
from ._lib import HosError, load
from .ensemble import HosEnsemble
from .field import HosField

__all__ = ["HosField", "HosEnsemble", "HosError", "ic", "load"]
