"""Ensembles: members advanced together must end bitwise equal to the same
members advanced one by one with hos_step, in both modes: size classes (one
launch per pass per class, one graph per step) and the persistent kernel
(one launch per step for every member).  The persistent kernel's bounded
waits are made to run out by withholding a dependency on the host side
(hos_ensemble_withhold_dependency): the step must end with HOS_ERR_TIMEOUT
and the ensemble must work again once the plan is restored."""
import numpy as np
import pytest

from hos_b200 import HosEnsemble, HosError, HosField, ic

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


def solo_runs(specs, nsteps):
    out = []
    for spec in specs:
        f, dt = make(spec)
        f.step(dt, nsteps)
        out.append((f.state_spectral()[0], f.energy_history()[1]))
        f.close()
    return out


def test_ensemble_matches_individual_steps():
    nsteps = 7
    solo = solo_runs(SPECS, nsteps)
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


PERSIST_SPECS = SPECS + [
    (512, 5, "fp32", None, 16.0, 8),
    (128, 4, "fp64", 0.5, 8.0, 9),
]


def test_persistent_ensemble_matches_individual_steps():
    """Mixed grids (64..512), orders (3..6), precisions and depths in one
    persistent launch per step: states and energy records bitwise as hos_step."""
    nsteps = 6
    solo = solo_runs(PERSIST_SPECS, nsteps)
    fields, dts = zip(*[make(s) for s in PERSIST_SPECS])
    with HosEnsemble(fields, dts, mode="persistent") as ens:
        assert ens.info["launches_per_step"] == 1
        ens.step(nsteps)
        ens.sync()
        for i, (f, (u, H)) in enumerate(zip(fields, solo)):
            got, _ = f.state_spectral()
            assert np.array_equal(got, u), i
            assert np.array_equal(f.energy_history()[1], H), i
    for f in fields:
        f.close()


def test_persistent_ensemble_wait_runs_out_and_recovers():
    specs = [(128, 4, "fp32", None, 8.0, 11), (256, 3, "fp32", None, 10.0, 12)]
    nsteps = 3
    solo = solo_runs(specs, nsteps)
    made = [make(s) for s in specs]
    fields, dts = zip(*made)
    with HosEnsemble(fields, dts, mode="persistent") as ens:
        ens.set_wait_limit(0.05)
        ens.withhold_dependency(True)
        ens.step(1)
        with pytest.raises(HosError) as ei:
            ens.sync()
        assert ei.value.code == 6  # HOS_ERR_TIMEOUT
        assert "waited past the limit" in str(ei.value)
        # restore the plan and the states: the same launches now run to the end
        ens.withhold_dependency(False)
        for (f, _), spec in zip(made, specs):
            n, M, prec, depth, kp, seed = spec
            eta, phi, info = ic.jonswap(n, n, kp=kp, steepness=0.08, seed=seed, depth=depth)
            f.set_state_physical(eta, phi)
            f.clear_history()
        ens.step(nsteps)
        ens.sync()
        for f, (u, H) in zip(fields, solo):
            assert np.array_equal(f.state_spectral()[0], u)
            assert np.array_equal(f.energy_history()[1], H)
    for f in fields:
        f.close()


@pytest.mark.parametrize("mode", ["persistent", "classes"])
def test_ensemble_step_budgets(mode):
    """Members stop after their own number of steps inside a run of
    launches: each ends bitwise as hos_step after that many steps."""
    specs = [(128, 3, "fp32", None, 8.0, 21), (256, 5, "fp32", 0.4, 12.0, 22), (64, 4, "fp32", None, 4.0, 23)]
    budgets = [2, 5, 0]
    solo = [solo_runs([s], b)[0] for s, b in zip(specs, budgets)]
    fields, dts = zip(*[make(s) for s in specs])
    with HosEnsemble(fields, dts, mode=mode) as ens:
        ens.set_steps(budgets)
        ens.step(7)
        ens.sync()
        assert ens.remaining() == [0, 0, 0]
        for f, (u, H), b in zip(fields, solo, budgets):
            assert np.array_equal(f.state_spectral()[0], u)
            assert np.array_equal(f.energy_history()[1], H)
            assert len(f.energy_history()[1]) == b
    for f in fields:
        f.close()
