"""Writes a run's input files: initpars.h5 and initdata.<runsubid>.h5.

    python -m hos_b200.make_inputs OUTDIR jonswap --n 256 --lx 3807.99 --g 9.81 --kp-index 8 --steepness 0.08
    python -m hos_b200.make_inputs OUTDIR stokes --n 64 --kmode 4 --ka 0.1 --T 10 --dtsave 1

The files hold what the reference's python/write_hdf5.py:5-40 writes (the
parameters get_params reads, KP and h, and eta0, phi0, bat0), so both the
reference's driver and hos_run read them; --order, --scheme and --dt add the
optional /M, /scheme and /dt datasets that hos_run uses in place of the
values the reference compiles in.  The sea comes from hos_b200.ic: a
directional JONSWAP spectrum (peak wavenumber kp = kp_index * 2 pi / Lx,
kp*Hs/2 = steepness, gamma, cos^(2s)(theta/2) spreading, seeded amplitudes,
linear phi_s) or a third-order Stokes wave along x.
"""
from __future__ import annotations

import argparse
import math
import sys

from . import h5, ic


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m hos_b200.make_inputs", description=__doc__.split("\n\n")[0])
    ap.add_argument("outdir")
    ap.add_argument("kind", choices=["jonswap", "stokes"])
    ap.add_argument("--n", type=int, default=256, help="grid points in x and in y (unless --ny)")
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--lx", type=float, default=2 * math.pi)
    ap.add_argument("--ly", type=float, default=None)
    ap.add_argument("--g", type=float, default=9.81)
    ap.add_argument("--kp-index", type=float, default=8.0, help="JONSWAP peak as a mode index along x")
    ap.add_argument("--steepness", type=float, default=0.08, help="JONSWAP kp*Hs/2")
    ap.add_argument("--gamma", type=float, default=3.3)
    ap.add_argument("--spread", type=float, default=15.0, help="s of cos^(2s)(theta/2)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--depth", type=float, default=None, help="finite depth h for the linear phi_s (deep if absent)")
    ap.add_argument("--kmode", type=int, default=4, help="Stokes wave mode index along x")
    ap.add_argument("--ka", type=float, default=0.1, help="Stokes wave steepness")
    ap.add_argument("--T", type=float, default=50.0, help="end time")
    ap.add_argument("--dtsave", type=float, default=1.0)
    ap.add_argument("--runsubid", type=int, default=1)
    ap.add_argument("--saveflg", type=int, default=1)
    ap.add_argument("--rampflg", type=int, default=1)
    ap.add_argument("--tramp", type=float, default=200.0)
    ap.add_argument("--h", type=float, default=1000.0, help="stored as /h (the reference does not read it)")
    ap.add_argument("--order", type=int, default=None, help="HOS order M for hos_run (/M)")
    ap.add_argument("--scheme", type=int, default=None, help="RK scheme 1..5 for hos_run (/scheme)")
    ap.add_argument("--dt", type=float, default=None, help="time step for hos_run (/dt)")
    a = ap.parse_args(argv)
    ny = a.ny or a.n
    ly = a.ly or a.lx
    if a.kind == "jonswap":
        kp = a.kp_index * 2 * math.pi / a.lx
        eta, phi, info = ic.jonswap(a.n, ny, lx=a.lx, ly=ly, g=a.g, kp=kp, steepness=a.steepness, gamma=a.gamma,
                                    spread_s=a.spread, seed=a.seed, depth=a.depth)
        desc = f"JONSWAP kp={kp:.6g} Hs={info['Hs']:.6g} Tp={info['Tp']:.6g}"
    else:
        eta, phi, omega = ic.stokes3(a.n, ny, lx=a.lx, ly=ly, g=a.g, kmode=a.kmode, ka=a.ka)
        desc = f"Stokes mode {a.kmode} ka={a.ka} period={2 * math.pi / omega:.6g}"
    h5.write_inputs(a.outdir, eta, phi, a.lx, ly, a.g, T=a.T, dtsave=a.dtsave, runsubid=a.runsubid,
                    saveflg=a.saveflg, rampflg=a.rampflg, tramp=a.tramp, h=a.h, order=a.order, scheme=a.scheme,
                    dt=a.dt)
    print(f"wrote {a.outdir}/initpars.h5 and initdata.{a.runsubid}.h5: {a.n}x{ny}, {desc}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
