"""Ensembles: members advanced together (one launch per pass per size class,
one graph per step) must end bitwise equal to the same members advanced one
by one with hos_step."""
import numpy as np
import pytest

from hos_b200 import HosEnsemble, HosField, ic

pytestmark = pytest.mark.gpu

SPECS = [  # (n, order, precision, depth, kp, seed)
    (128, 3, "fp32", None, 8.0, 1),
    (128, 5, "fp32", 0.4, 8.0, 2),
    (256, 4, "fp32", None, 12.0, 3),
    (128, 4, "fp32", None, 6.0, 4),
    (256, 3, "fp64", 0.3, 10.0, 5),
    (64, 6, "fp64", None, 4.0, 6),
    (64, 3, "fp64", None, 5.0, 7),
]


def make(spec):
    n, M, prec, depth, kp, seed = spec
    eta, phi, info = ic.jonswap(n, n, kp=kp, steepness=0.08, seed=seed, depth=depth)
    f = HosField(n, n, order=M, precision=prec, depth=depth)
    f.set_state_physical(eta, phi)
    return f, info["Tp"] / 50


def test_ensemble_matches_individual_steps():
    nsteps = 7
    solo = []
    for spec in SPECS:
        f, dt = make(spec)
        f.step(dt, nsteps)
        solo.append((f.state_spectral()[0], f.energy_history()[1]))
        f.close()
    fields, dts = zip(*[make(s) for s in SPECS])
    with HosEnsemble(fields, dts) as ens:
        assert ens.info["classes"] == 4  # (128, fp32), (256, fp32), (256, fp64), (64, fp64)
        ens.step(nsteps)
        ens.sync()
        for f, (u, H) in zip(fields, solo):
            got, _ = f.state_spectral()
            assert np.array_equal(got, u)
            assert np.array_equal(f.energy_history()[1], H)
    for f in fields:
        f.close()


def test_ensemble_of_identical_class():
    fields, dts = zip(*[make((128, 4, "fp32", None, 8.0, s)) for s in range(20)])
    with HosEnsemble(fields, dts) as ens:
        assert ens.info["classes"] == 1
        ens.step(3)
        ens.sync()
    for f in fields:
        assert f.is_finite()
        f.close()
