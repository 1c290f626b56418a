"""CPU tests of libhos_hostshim.so: the single-rank MPI, FFTW-MPI set-up and
HDF5 calls that let the reference's own driver (main_2d_par.c,
hdf5_routines_2d_par.c) run against libhos_gpu.so without MPI, FFTW or
libhdf5.  The HDF5 calls are exercised the way hdf5_routines_2d_par.c makes
them (1x1 headers written with H5S_ALL, [Nx][Ny] fields through a hyperslab
of the file space, reads converted to F64) and the files are read back with
the library's own reader."""
import ctypes
import os

import numpy as np
import pytest

from hos_b200 import h5

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "hos_b200", "libhos_hostshim.so")

H5F_ACC_RDONLY, H5F_ACC_TRUNC = 0, 2
H5P_FILE_ACCESS, H5P_DATASET_XFER = 0x1000000001, 0x1000000002
F64, F32 = 0x2000000001, 0x2000000002


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(SHIM):
        pytest.skip("libhos_hostshim.so not built (make -C hos_b200/csrc)")
    L = ctypes.CDLL(SHIM)
    I64, U64P, VP = ctypes.c_longlong, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_void_p
    sig = {
        "H5Fcreate": ([ctypes.c_char_p, ctypes.c_uint, I64, I64], I64),
        "H5Fopen": ([ctypes.c_char_p, ctypes.c_uint, I64], I64),
        "H5Fclose": ([I64], ctypes.c_int),
        "H5Dcreate": ([I64, ctypes.c_char_p, I64, I64, I64, I64, I64], I64),
        "H5Dopen": ([I64, ctypes.c_char_p, I64], I64),
        "H5Dwrite": ([I64, I64, I64, I64, I64, VP], ctypes.c_int),
        "H5Dread": ([I64, I64, I64, I64, I64, VP], ctypes.c_int),
        "H5Dget_space": ([I64], I64),
        "H5Dclose": ([I64], ctypes.c_int),
        "H5Screate_simple": ([ctypes.c_int, U64P, U64P], I64),
        "H5Sselect_hyperslab": ([I64, ctypes.c_int, U64P, U64P, U64P, U64P], ctypes.c_int),
        "H5Sclose": ([I64], ctypes.c_int),
        "H5Pcreate": ([I64], I64),
        "H5Pclose": ([I64], ctypes.c_int),
        "H5Pset_fapl_mpio": ([I64, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "H5Tcopy": ([I64], I64),
        "fftw_mpi_local_size_2d_transposed": ([ctypes.c_ssize_t, ctypes.c_ssize_t, ctypes.c_int] +
                                              [ctypes.POINTER(ctypes.c_ssize_t)] * 4, ctypes.c_ssize_t),
        "fftw_alloc_real": ([ctypes.c_size_t], VP),
        "fftw_free": ([VP], None),
        "MPI_Comm_size": ([ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "MPI_Comm_rank": ([ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "MPI_Reduce": ([VP, VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


def dims(*v):
    return (ctypes.c_ulonglong * len(v))(*v)


def test_single_rank_mpi_and_fftw_sizes(lib):
    n = ctypes.c_int()
    assert lib.MPI_Comm_size(0, ctypes.byref(n)) == 0 and n.value == 1
    assert lib.MPI_Comm_rank(0, ctypes.byref(n)) == 0 and n.value == 0
    a = np.array([1.5, 2.5])
    b = np.zeros(2)
    lib.MPI_Reduce(a.ctypes.data, b.ctypes.data, 2, 2, 1, 0, 0)
    assert np.array_equal(a, b)
    l0, s0, l1, s1 = (ctypes.c_ssize_t() for _ in range(4))
    tot = lib.fftw_mpi_local_size_2d_transposed(64, 33, 0, ctypes.byref(l0), ctypes.byref(s0), ctypes.byref(l1),
                                                ctypes.byref(s1))
    assert (tot, l0.value, s0.value, l1.value, s1.value) == (64 * 33, 64, 0, 33, 0)
    p = lib.fftw_alloc_real(1000)
    assert p and p % 64 == 0
    lib.fftw_free(p)


def test_hdf5_calls_of_the_driver_round_trip(lib, tmp_path):
    nx, ny = 16, 8
    rng = np.random.default_rng(1)
    field = rng.standard_normal((nx, ny))
    path = str(tmp_path / "data1.1.h5").encode()
    fapl = lib.H5Pcreate(H5P_FILE_ACCESS)
    assert lib.H5Pset_fapl_mpio(fapl, 0, 0) == 0
    f = lib.H5Fcreate(path, H5F_ACC_TRUNC, 0, fapl)
    assert f > 0
    lib.H5Pclose(fapl)
    t = lib.H5Tcopy(F64)
    one = lib.H5Screate_simple(2, dims(1, 1), None)
    v = np.array([2.75])
    d = lib.H5Dcreate(f, b"time", t, one, 0, 0, 0)
    assert lib.H5Dwrite(d, t, 0, 0, 0, v.ctypes.data) == 0
    lib.H5Dclose(d)
    lib.H5Sclose(one)
    # write_field_2d: file space [Nx][Ny], memory space = the local block, hyperslab at offset 0
    fs = lib.H5Screate_simple(2, dims(nx, ny), None)
    d = lib.H5Dcreate(f, b"eta", t, fs, 0, 0, 0)
    lib.H5Sclose(fs)
    ms = lib.H5Screate_simple(2, dims(nx, ny), None)
    fs = lib.H5Dget_space(d)
    assert lib.H5Sselect_hyperslab(fs, 0, dims(0, 0), None, dims(nx, ny), None) == 0
    xf = lib.H5Pcreate(H5P_DATASET_XFER)
    assert lib.H5Dwrite(d, t, ms, fs, xf, field.ctypes.data) == 0
    lib.H5Dclose(d)
    lib.H5Sclose(fs)
    lib.H5Sclose(ms)
    # a single-precision dataset keeps its stored type
    d = lib.H5Dcreate(f, b"single", lib.H5Tcopy(F32), lib.H5Screate_simple(2, dims(nx, ny), None), 0, 0, 0)
    assert lib.H5Dwrite(d, F64, 0, 0, 0, field.ctypes.data) == 0
    assert lib.H5Fclose(f) == 0

    assert h5.read(tmp_path / "data1.1.h5", "time")[0, 0] == 2.75
    assert np.array_equal(h5.read(tmp_path / "data1.1.h5", "eta"), field)
    assert np.array_equal(h5.read(tmp_path / "data1.1.h5", "single"), field.astype(np.float32).astype(np.float64))

    # get_ic_2d: read through a hyperslab of the file space into F64 and F32 buffers
    f = lib.H5Fopen(path, H5F_ACC_RDONLY, 0)
    d = lib.H5Dopen(f, b"/eta", 0)
    fs = lib.H5Dget_space(d)
    lib.H5Sselect_hyperslab(fs, 0, dims(4, 0), None, dims(8, ny), None)
    ms = lib.H5Screate_simple(2, dims(8, ny), None)
    got = np.zeros((8, ny))
    assert lib.H5Dread(d, F64, ms, fs, 0, got.ctypes.data) == 0
    assert np.array_equal(got, field[4:12])
    got32 = np.zeros((nx, ny), np.float32)
    assert lib.H5Dread(d, F32, 0, 0, 0, got32.ctypes.data) == 0
    assert np.array_equal(got32, field.astype(np.float32))
    # errors are reported, not guessed
    assert lib.H5Dopen(f, b"/missing", 0) < 0
    assert lib.H5Sselect_hyperslab(fs, 0, dims(0, 0), dims(2, 1), dims(4, ny), None) < 0
    lib.H5Fclose(f)
    assert lib.H5Fopen(str(tmp_path / "nope.h5").encode(), H5F_ACC_RDONLY, 0) < 0
