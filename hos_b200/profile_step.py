"""Small driver for ncu captures of the RK step kernels.

    python -m hos_b200.profile_step N M PRECISION WARMUP STEPS

Creates one N x N field of order M (JONSWAP sea, kp = 24 N/1024,
kp*Hs/2 = 0.12), loads it, and advances WARMUP + STEPS RK4 steps with the
shapes the autotuner chose on B200 at 1024^2, M = 5.  It prints one line
and exits; it is meant to run under ncu, with the launches of interest
selected by -s/-c.
"""
import sys

from . import HosField, ic

TUNED = {"fp32": [8, 8, 8, 8, 1, 0, 0, 0, 5, 0, 16, -1], "fp64": [8, 8, 8, 8, -1, 0, -1, -1, 5, 0, 16, -1]}


def main(argv):
    n, M, prec, warm, steps = int(argv[0]), int(argv[1]), argv[2], int(argv[3]), int(argv[4])
    eta, phi, info = ic.jonswap(n, n, kp=24.0 * n / 1024, steepness=0.12, seed=1)
    with HosField(n, n, order=M, precision=prec, tune=TUNED[prec]) as f:
        f.set_state_physical(eta, phi)
        f.step(info["Tp"] / 50, warm + steps)
        f.sync()
        print("ok", f.is_finite())


if __name__ == "__main__":
    main(sys.argv[1:])
