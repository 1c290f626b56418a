"""Failure detection on the device, without faulting it: a non-finite state
(NaN planted in the host input) is flagged by the step-end energy check and
reported by hos_sync / hos_ensemble_sync; the other members of an ensemble
and the other requests of a server are unaffected; an allocation failure
injected on the host returns HOS_ERR_NOMEM and leaves no device memory
behind."""
import copy

import numpy as np
import pytest

from hos_b200 import HosEnsemble, HosError, HosField, ic
from hos_b200._lib import HOS_ERR_NOMEM, HOS_ERR_NONFINITE, load
from hos_b200.serve import Request, Server

pytestmark = pytest.mark.gpu


def _sea(n=64, seed=3):
    return ic.jonswap(n, n, kp=n / 8, steepness=0.1, seed=seed)


def test_sync_reports_nonfinite_step():
    eta, phi, info = _sea()
    dt = info["Tp"] / 50
    with HosField(64, 64, order=4) as f:
        f.set_state_physical(eta, phi)
        f.step(dt, 3)
        f.sync()
        assert f.health() is None
        bad = eta.copy()
        bad[5, 7] = np.nan
        f.set_state_physical(bad, phi, t=0.0)
        f.step(dt, 4)
        with pytest.raises(HosError) as ei:
            f.sync()
        # steps are counted from the handle's creation: the three good ones
        # were steps 0-2
        assert ei.value.code == HOS_ERR_NONFINITE and "step 3" in str(ei.value)
        assert f.health() == 3
        # a new state clears the flag
        f.set_state_physical(eta, phi)
        f.step(dt, 2)
        f.sync()
        assert f.health() is None


def test_ensemble_member_failure_is_isolated():
    eta, phi, info = _sea()
    dt = info["Tp"] / 50
    with HosField(64, 64, order=4) as solo:
        solo.set_state_physical(eta, phi)
        solo.step(dt, 10)
        solo.sync()
        want = solo.state_spectral()[0]
    good = HosField(64, 64, order=4)
    bad = HosField(64, 64, order=4)
    try:
        good.set_state_physical(eta, phi)
        b = phi.copy()
        b[0, 0] = np.inf
        bad.set_state_physical(eta, b)
        with HosEnsemble([bad, good], [dt, dt]) as ens:
            ens.step(10)
            with pytest.raises(HosError) as ei:
                ens.sync()
            assert ei.value.code == HOS_ERR_NONFINITE
        assert bad.health() == 0 and good.health() is None
        assert np.array_equal(good.state_spectral()[0], want)
    finally:
        good.close()
        bad.close()


def test_server_fails_only_the_nonfinite_request():
    reqs = [Request(rid=i, n=64, order=4, steps=30, seed=40 + i) for i in range(3)]
    reqs[1].steepness = float("nan")
    alone = copy.deepcopy(reqs[2])
    Server(chunk=10, reserve_bytes=0).run([alone], realtime=False)
    m = Server(chunk=10, reserve_bytes=0).run(reqs, realtime=False)
    assert m["completed"] == 2 and m["failed"] == 1
    assert reqs[1].status == "failed" and "non-finite" in reqs[1].error
    assert reqs[0].status == "done" and reqs[2].status == "done"
    assert np.array_equal(reqs[2].result[0], alone.result[0])


def test_injected_allocation_failure_cleans_up():
    import torch

    lib = load()
    torch.cuda.init()
    HosField(256, 256, order=5).close()  # context and library warm
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    try:
        for k in range(0, 40):
            lib.hos_inject_alloc_failure(k)
            try:
                f = HosField(256, 256, order=5)
            except HosError as e:
                assert e.code == HOS_ERR_NOMEM and "injected" in str(e)
                failures += 1
                continue
            f.close()
            break
        assert failures >= 10  # a field makes at least that many allocations
        # an ensemble whose own allocation fails
        lib.hos_inject_alloc_failure(-1)
        a, b = HosField(64, 64, order=3), HosField(64, 64, order=3)
        lib.hos_inject_alloc_failure(0)
        with pytest.raises(HosError) as ei:
            HosEnsemble([a, b], [0.1, 0.1])
        assert ei.value.code == HOS_ERR_NOMEM
        lib.hos_inject_alloc_failure(-1)
        with HosEnsemble([a, b], [0.1, 0.1]) as ens:
            ens.step(2)
            ens.sync()
        a.close()
        b.close()
    finally:
        lib.hos_inject_alloc_failure(-1)
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (4 << 20)
