"""HDF5 files of the HOS driver, read and written by the library's own
subset of the format (hos_h5_* in include/hos_gpu.h; no libhdf5 or h5py).

* ``read(path, name)``: one dataset as a float64 array, converted from its
  stored type as the reference's H5Dread with a H5T_IEEE_F64LE memory type
  does (hdf5_routines_2d_par.c:13-101, :104-188);
* ``write(path, datasets)``: a new file of root-group datasets, each float64,
  float32 or int64, rank 0 to 2;
* ``read_params`` / ``write_inputs``: the parameter and initial-condition
  files of a run (``initpars.h5``, ``initdata.<runsubid>.h5``), with the
  datasets and stored types of the reference's python/write_hdf5.py:5-40;
* ``write_snapshot``: a snapshot file as write_header_2d + write_field_2d
  produce it (hdf5_routines_2d_par.c:227-392).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

F64, F32, I64, I32 = 0, 1, 2, 3

# initpars.h5: every name get_params reads (hdf5_routines_2d_par.c:13-101)
# plus KP and h, which write_hdf5.py stores and the C code does not read.
# Counts and flags are stored as int64; the other values as h5py stores the
# Python value given (int64 for an int, float64 for a float).
INT_PARAMS = ("Nx", "Ny", "KP", "saveflg", "runsubid", "rampflg", "M", "scheme")
REQUIRED_PARAMS = ("Nx", "Ny", "Lx", "Ly", "g", "runsubid", "T", "dtsave", "saveflg", "rampflg", "Tramp")


def _lib_h5():
    lib = _lib.load()
    if not getattr(lib, "_h5_bound", False):
        c = ctypes
        lib.hos_h5_list.argtypes = [c.c_char_p, c.c_char_p, c.c_int, c.POINTER(c.c_int)]
        lib.hos_h5_info.argtypes = [c.c_char_p, c.c_char_p, c.POINTER(c.c_int), c.POINTER(c.c_longlong),
                                    c.POINTER(c.c_int)]
        lib.hos_h5_read_f64.argtypes = [c.c_char_p, c.c_char_p, c.c_void_p, c.c_longlong]
        lib.hos_h5_write.argtypes = [c.c_char_p, c.c_int, c.POINTER(c.c_char_p), c.POINTER(c.c_void_p),
                                     c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_longlong)]
        for f in (lib.hos_h5_list, lib.hos_h5_info, lib.hos_h5_read_f64, lib.hos_h5_write):
            f.restype = c.c_int
        lib._h5_bound = True
    return lib


def _b(s):
    return os.fsencode(s)


def names(path):
    lib = _lib_h5()
    buf = ctypes.create_string_buffer(1 << 16)
    n = ctypes.c_int()
    _lib.check(lib.hos_h5_list(_b(path), buf, len(buf), ctypes.byref(n)))
    return [s for s in buf.value.decode().split("\n") if s]


def info(path, name):
    """(shape, stored type code)."""
    lib = _lib_h5()
    rank, typ = ctypes.c_int(), ctypes.c_int()
    dims = (ctypes.c_longlong * 4)()
    _lib.check(lib.hos_h5_info(_b(path), _b(name), ctypes.byref(rank), dims, ctypes.byref(typ)))
    return tuple(int(dims[i]) for i in range(rank.value)), typ.value


def read(path, name):
    shape, _ = info(path, name)
    out = np.empty(shape, dtype=np.float64)
    lib = _lib_h5()
    _lib.check(lib.hos_h5_read_f64(_b(path), _b(name), out.ctypes.data_as(ctypes.c_void_p), out.size))
    return out


def write(path, datasets, types=None):
    """datasets: {name: array or scalar}; types: {name: F64|F32|I64}
    (default F64 for floats, I64 for integers)."""
    types = dict(types or {})
    keep, nm, ptrs, ty, rk, dm = [], [], [], [], [], []
    for name, v in datasets.items():
        a = np.asarray(v)
        t = types.get(name, I64 if np.issubdtype(a.dtype, np.integer) else F64)
        a = np.array(a, dtype={F64: "<f8", F32: "<f4", I64: "<i8"}[t], order="C")  # keeps rank 0
        if a.ndim > 2:
            raise ValueError(f"{name}: rank {a.ndim} (0..2 supported)")
        keep.append(a)
        nm.append(_b(name))
        ptrs.append(a.ctypes.data if a.size else None)
        ty.append(t)
        rk.append(a.ndim)
        dm.extend(list(a.shape) + [0] * (2 - a.ndim))
    n = len(nm)
    lib = _lib_h5()
    _lib.check(lib.hos_h5_write(_b(path), n, (ctypes.c_char_p * n)(*nm), (ctypes.c_void_p * n)(*ptrs),
                                (ctypes.c_int * n)(*ty), (ctypes.c_int * n)(*rk), (ctypes.c_longlong * (2 * n))(*dm)))


def read_params(path):
    """The run parameters as get_params reads them (all as float), with the
    reference's rule for rampflg (a value other than 0 or 1 becomes 0,
    hdf5_routines_2d_par.c:81-86) and Kx0 = 2 pi/Lx, Ky0 = 2 pi/Ly (:98-99)."""
    p = {}
    present = set(names(path))
    for k in REQUIRED_PARAMS:
        if k not in present:
            raise KeyError(f"{path}: parameter dataset /{k} missing")
        p[k] = float(read(path, k).reshape(-1)[0])
    for k in ("KP", "h", "M", "scheme", "dt"):  # the last three: hos_run's optional run settings
        if k in present:
            p[k] = float(read(path, k).reshape(-1)[0])
    for k in ("Nx", "Ny", "runsubid", "saveflg", "rampflg"):
        p[k] = int(p[k])
    if p["rampflg"] not in (0, 1):
        p["rampflg"] = 0
    p["Kx0"] = 2 * np.pi / p["Lx"]
    p["Ky0"] = 2 * np.pi / p["Ly"]
    return p


def write_inputs(folder, eta, phi, lx, ly, g, T, dtsave, runsubid=1, saveflg=1, rampflg=1, tramp=200, h=1000.0,
                 kp=10000, bathy=None, order=None, scheme=None, dt=None):
    """initpars.h5 and initdata.<runsubid>.h5 in `folder`, holding what the
    reference's python/write_hdf5.py:5-40 writes (the file names are the
    ones main_2d_par.c:80-100 opens).  order, scheme and dt, when given, are
    stored as /M, /scheme and /dt, which hos_run reads in place of the
    values the reference compiles in (M = 3, scheme 4, dt = 0.2)."""
    eta = np.asarray(eta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    nx, ny = eta.shape
    bathy = np.zeros_like(eta) if bathy is None else np.asarray(bathy, dtype=np.float64)
    vals = {"Nx": nx, "Ny": ny, "Lx": lx, "Ly": ly, "g": g, "KP": kp, "h": h, "T": T, "dtsave": dtsave,
            "saveflg": saveflg, "runsubid": runsubid, "rampflg": rampflg, "Tramp": tramp}
    for k, v in (("M", order), ("scheme", scheme), ("dt", dt)):
        if v is not None:
            vals[k] = v
    types = {k: I64 if k in INT_PARAMS or isinstance(v, (int, np.integer)) else F64 for k, v in vals.items()}
    os.makedirs(folder, exist_ok=True)
    write(os.path.join(folder, "initpars.h5"), vals, types)
    write(os.path.join(folder, f"initdata.{int(runsubid)}.h5"), {"eta0": eta, "phi0": phi, "bat0": bathy})


def write_snapshot(path, t, g, lx, ly, eta, phi, bat):
    """One output file as main_2d_par.c:271-273 / :323-325 write it: the
    header (time, g, Nx, Ny, Lx, Ly as 1x1 float64) and eta, phi, bat."""
    nx, ny = np.shape(eta)
    one = lambda v: np.full((1, 1), float(v))  # noqa: E731
    write(path, {"time": one(t), "g": one(g), "Nx": one(nx), "Ny": one(ny), "Lx": one(lx), "Ly": one(ly),
                 "eta": eta, "phi": phi, "bat": bat})
