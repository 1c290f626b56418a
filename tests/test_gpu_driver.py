"""The reference's driver configuration end to end on the GPU.

* The reference's only shipped input (256^2 JONSWAP, Lx = 3807.99, g = 9.81,
  ramp with Tramp = 200) advanced as its driver does (M = 3, midpoint RK2,
  dt = 0.2, 250 steps to T = 50) matches the reference's own code (golden
  fixture from the C oracle) to 1e-10.
* hos_run, the driver program on the library, reads the run's HDF5 inputs
  and writes the snapshots, the extra fields, runtime.dat and the ParaView
  index as main_2d_par.c does; every snapshot and energy record matches the
  reference's code run on the same input.
"""
import math
import os
import re
import subprocess

import numpy as np
import pytest

from hos_b200 import HosField, h5, ic

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOS_RUN = os.path.join(ROOT, "hos_b200", "hos_run")
TOL = 1e-10


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_shipped_input_matches_reference(golden):
    d = golden("shipped256_m3_mid_250")
    nx, ny, M, scheme, ramp = (int(v) for v in d["meta"])
    rows, cols = d["rows"].astype(int), d["cols"].astype(int)
    u0 = np.zeros((2, ny // 2 + 1, nx), complex)
    u0[:, rows, cols] = d["u0"]
    with HosField(nx, ny, order=M, lx=float(d["lx"]), ly=float(d["ly"]), g=float(d["g"]), rampflg=ramp,
                  tramp=float(d["tramp"]), scheme=scheme) as f:
        f.set_state_spectral(u0, 0.0)
        f.step(float(d["dt"]), len(d["ham"]))
        u, t = f.state_spectral()
        _, H = f.energy_history()
    assert abs(t - float(d["t250"])) < 1e-12
    assert rel(u[0][rows, cols], d["u250"][0]) < TOL and rel(u[1][rows, cols], d["u250"][1]) < TOL
    outside = np.ones(u.shape[1:], bool)
    outside[rows, cols] = False
    assert not u[:, outside].any()  # dealiased
    assert rel(H, d["ham"]) < TOL


class _Oracle:
    """The reference's own code (C oracle) where it is built, else the numpy
    restatement, behind one interface."""

    def __init__(self, M, n, lx, g, ramp, tramp, scheme):
        from oracle import ref_c
        from oracle.hos_np import HosNumpy

        self.c = ref_c.RefC(M, n, n, lx=lx, ly=lx, g=g, rampflg=ramp, tramp=tramp, scheme=scheme) \
            if ref_c.available(M) else None
        self.np = HosNumpy(n, n, lx, lx, g, M, rampflg=ramp, tramp=tramp)
        self.scheme = scheme

    def init(self, eta, phi):
        return self.c.init_state(eta, phi) if self.c else np.stack(self.np.init_state(eta, phi))

    def steps(self, u, t, dt, n):
        if self.c:
            return self.c.steps(u, t, dt, n)
        e, p, H = u[0], u[1], []
        for _ in range(n):
            e, p, t, h = self.np.step(e, p, t, dt, self.scheme)
            H.append(h)
        return np.stack([e, p]), t, np.array(H)

    def ifft2(self, hu):
        return self.c.ifft2(hu) if self.c else self.np.ifft2(hu)

    def zvel(self, u):
        return self.c.zvel(u) if self.c else self.np.Zvel(u[0], u[1])


def test_hos_run_driver_matches_reference(tmp_path):
    assert os.path.exists(HOS_RUN), "hos_run is built by make -C hos_b200/csrc"
    n, M, lx, g = 64, 3, 1000.0, 9.81
    eta, phi, info = ic.jonswap(n, n, lx=lx, ly=lx, g=g, kp=2 * math.pi / lx * 6, steepness=0.08, seed=9)
    bat = np.zeros_like(eta)
    h5.write_inputs(tmp_path, eta, phi, lx, lx, g, T=3, dtsave=1.0, runsubid=3, saveflg=2, rampflg=1, tramp=2,
                    bathy=bat)
    r = subprocess.run([HOS_RUN, "-C", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Reading initial data from:\tinitdata.3.h5" in r.stdout
    assert "Datafile 'data3.3.h5' written at t=3.000000" in r.stdout

    ora = _Oracle(M, n, lx, g, 1, 2.0, 4)
    u = ora.init(eta, phi)
    # data0: the input as read; then one snapshot per unit of time (5 steps of 0.2)
    d0 = tmp_path / "data0.3.h5"
    assert np.array_equal(h5.read(d0, "eta"), eta) and np.array_equal(h5.read(d0, "phi"), phi)
    t, hams, times = 0.0, [], []
    for k in (1, 2, 3):
        t0 = t
        u, t, H = ora.steps(u, t, 0.2, 5)
        hams.extend(H)
        times.extend(t0 + 0.2 * i for i in range(5))
        f = tmp_path / f"data{k}.3.h5"
        assert h5.read(f, "time")[0, 0] == t
        assert (h5.read(f, "Nx")[0, 0], h5.read(f, "g")[0, 0], h5.read(f, "Lx")[0, 0]) == (n, g, lx)
        assert rel(h5.read(f, "eta"), ora.ifft2(u[0])) < TOL
        assert rel(h5.read(f, "phi"), ora.ifft2(u[1])) < TOL
        assert not h5.read(f, "bat").any()
    assert not (tmp_path / "data4.3.h5").exists()

    # runtime.dat: one "%14.10f\t%.16g" line per step, step-start time
    lines = (tmp_path / "runtime.dat").read_text().splitlines()
    assert len(lines) == 15
    for line, tt, hh in zip(lines, times, hams):
        assert re.fullmatch(r" *-?\d+\.\d{10}\t\S+", line), line
        a, b = line.split("\t")
        assert abs(float(a) - tt) < 1e-9
        assert abs(float(b) - hh) <= TOL * abs(hh)

    # data_extra: W^(M), W^(M-2) of the initial state, the same in every file
    w = ora.zvel(ora.init(eta, phi))
    for k in range(4):
        f = tmp_path / f"data_extra{k}.3.h5"
        assert rel(h5.read(f, "Array1"), ora.ifft2(w[0])) < 1e-12
        assert rel(h5.read(f, "Array2"), ora.ifft2(w[1])) < 1e-12

    xmf = (tmp_path / "HOS_data.xmf").read_text()
    assert xmf.startswith("<Xdmf>") and xmf.rstrip().endswith("</Xdmf>")
    assert xmf.count("<Grid Name=\"Cells\"") == 4 and "data0.1.h5:/eta" in xmf and "data3.3.h5:/phi" in xmf
    assert h5.read(tmp_path / "data_coordinates.h5", "xy").shape == (n * n, 2)


def test_hos_run_takes_order_scheme_dt_from_the_parameter_file(tmp_path):
    n, lx, g = 64, 1000.0, 9.81
    eta, phi, info = ic.jonswap(n, n, lx=lx, ly=lx, g=g, kp=2 * math.pi / lx * 6, steepness=0.08, seed=10)
    h5.write_inputs(tmp_path, eta, phi, lx, lx, g, T=1, dtsave=1.0, runsubid=1, saveflg=1, rampflg=0, tramp=1,
                    order=4, scheme=2, dt=0.1)
    assert h5.read_params(tmp_path / "initpars.h5")["M"] == 4.0
    r = subprocess.run([HOS_RUN, "-C", str(tmp_path), "-q"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ora = _Oracle(4, n, lx, g, 0, 1.0, 2)
    u, t, H = ora.steps(ora.init(eta, phi), 0.0, 0.1, 10)
    assert h5.read(tmp_path / "data1.1.h5", "time")[0, 0] == t
    assert rel(h5.read(tmp_path / "data1.1.h5", "eta"), ora.ifft2(u[0])) < TOL
    assert len((tmp_path / "runtime.dat").read_text().splitlines()) == 10
    # the command line overrides the file
    r = subprocess.run([HOS_RUN, "-C", str(tmp_path), "-q", "-M", "3", "-dt", "0.2"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    ora3 = _Oracle(3, n, lx, g, 0, 1.0, 2)
    u3, t3, _ = ora3.steps(ora3.init(eta, phi), 0.0, 0.2, 5)
    assert rel(h5.read(tmp_path / "data1.1.h5", "eta"), ora3.ifft2(u3[0])) < TOL


def test_hos_run_reports_missing_input(tmp_path):
    r = subprocess.run([HOS_RUN, "-C", str(tmp_path), "-q"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "initpars.h5" in r.stderr
