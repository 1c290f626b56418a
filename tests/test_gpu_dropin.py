"""The literal drop-in: the reference's own host driver, unchanged, on the GPU.

oracle/_ref/euler_2d_par_gpu is Csource/2dpar/main_2d_par.c with
hdf5_routines_2d_par.c and xdmf_routines_2d_par.c, compiled unchanged
(-fcommon -DUSE_DOUBLES) against the single-rank MPI / FFTW-MPI / HDF5
headers of hos_b200/hostshim and linked with libhos_gpu.so in place of the
reference's four hot-path objects (`make -C oracle dropin`).  Its globals
(euler_2d_par.h:40-98, fft_routines_2d_par.h:17-38) are the ones the
library's reference-named functions read, through the dynamic link.

The run is the reference's shipped configuration (256^2 JONSWAP,
Lx = 3807.99, g = 9.81, ramp Tramp = 200, T = 50, dtsave = 1, and the
driver's compiled-in M = 3, midpoint RK2, dt = 0.2): its input files are
written from the dealiased initial spectrum of the shipped case (the golden
fixture shipped256_m3_mid_250), so that the run reproduces the reference's
own 250 steps.  Every snapshot, runtime.dat and the driver's messages are
checked; the last snapshot and the energy series against the reference's
code to 1e-10."""
import math
import os
import subprocess

import numpy as np
import pytest

from hos_b200 import h5
from oracle.hos_np import HosNumpy

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "euler_2d_par_gpu")
TOL = 1e-10


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _shipped_inputs(d, folder, dtsave, saveflg):
    nx, ny, M, scheme, ramp = (int(v) for v in d["meta"])
    lx, ly, g = float(d["lx"]), float(d["ly"]), float(d["g"])
    rows, cols = d["rows"].astype(int), d["cols"].astype(int)
    u0 = np.zeros((2, ny // 2 + 1, nx), complex)
    u0[:, rows, cols] = d["u0"]
    hn = HosNumpy(nx, ny, lx, ly, g, M, rampflg=ramp, tramp=float(d["tramp"]))
    eta, phi = hn.ifft2(u0[0]), hn.ifft2(u0[1])
    h5.write_inputs(folder, eta, phi, lx, ly, g, T=50.0, dtsave=dtsave, runsubid=1, saveflg=saveflg, rampflg=ramp,
                    tramp=float(d["tramp"]), kp=10000, h=1000.0)
    return hn, eta, phi, rows, cols


def _run(folder, resident):
    env = dict(os.environ)
    env.pop("HOS_NLEVS", None)  # the driver's own NLevs = 2 (M = 3), the library's default
    env["HOS_LEGACY_RESIDENT"] = "1" if resident else "0"
    r = subprocess.run([DROPIN], cwd=folder, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


@pytest.mark.parametrize("resident", [False, True])
def test_reference_driver_runs_the_shipped_case_on_the_gpu(golden, tmp_path, resident):
    assert os.path.exists(DROPIN), "built by `make -C oracle dropin` where the reference sources are present"
    d = golden("shipped256_m3_mid_250")
    # resident mode: extended output (saveflg 2) every 10 time units
    dtsave, saveflg = (10.0, 2) if resident else (1.0, 1)
    hn, eta, phi, rows, cols = _shipped_inputs(d, tmp_path, dtsave, saveflg)
    out = _run(tmp_path, resident)
    nsave = int(round(50.0 / dtsave))
    assert "Reading initial data from:\tinitdata.1.h5" in out
    assert "Datafile 'data0.1.h5' written at t=0.000000" in out
    assert f"Datafile 'data{nsave}.1.h5' written at t=50.000000" in out
    assert "Total computational time:" in out

    # the initial snapshot is the input as read (padded copy, main_2d_par.c:270-273)
    d0 = tmp_path / "data0.1.h5"
    assert np.array_equal(h5.read(d0, "eta"), eta) and np.array_equal(h5.read(d0, "phi"), phi)
    assert h5.read(d0, "Nx")[0, 0] == 256 and h5.read(d0, "g")[0, 0] == 9.81
    # every save time has its file, and no more
    for k in range(1, nsave + 1):
        f = tmp_path / f"data{k}.1.h5"
        assert abs(h5.read(f, "time")[0, 0] - k * dtsave) < 1e-9
    assert not (tmp_path / f"data{nsave + 1}.1.h5").exists()

    # the final state against the reference's own 250 steps
    u250 = np.zeros((2, 129, 256), complex)
    u250[:, rows, cols] = d["u250"]
    last = tmp_path / f"data{nsave}.1.h5"
    assert rel(h5.read(last, "eta"), hn.ifft2(u250[0])) < TOL
    assert rel(h5.read(last, "phi"), hn.ifft2(u250[1])) < TOL

    # runtime.dat: "%14.10f\t%.16g" per step, the stage-0 Hamiltonian at the step-start time
    lines = (tmp_path / "runtime.dat").read_text().splitlines()
    assert len(lines) == 250
    t = np.array([float(x.split("\t")[0]) for x in lines])
    H = np.array([float(x.split("\t")[1]) for x in lines])
    assert np.allclose(t, 0.2 * np.arange(250), atol=1e-9)
    assert rel(H, d["ham"]) < TOL

    if saveflg > 1:
        # data_extra: the initial W^(M), W^(M-2) in every file (main_2d_par.c:264-265,276-285,335-351)
        u0 = np.zeros((2, 129, 256), complex)
        u0[:, rows, cols] = d["u0"]
        wM, wM2, _, _ = hn.Zvel(u0[0], u0[1])
        for k in range(nsave + 1):
            f = tmp_path / f"data_extra{k}.1.h5"
            assert rel(h5.read(f, "Array1"), hn.ifft2(wM)) < 1e-12
            assert rel(h5.read(f, "Array2"), hn.ifft2(wM2)) < 1e-12
    xmf = (tmp_path / "HOS_data.xmf").read_text()
    assert xmf.startswith("<Xdmf>") and xmf.count("<Grid Name=\"Cells\"") == nsave + 1
    assert math.isfinite(H[-1])
