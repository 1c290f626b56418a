"""Serving: continuous batching must not change results.  Each request's
final eta, phi must be the same when it is served alone and when it is
served in a mix of arrivals (bit for bit: every field runs the same kernel
sequence either way), and admission must respect the memory budget."""
import copy

import numpy as np
import pytest

from hos_b200.serve import Request, Server

pytestmark = pytest.mark.gpu

REQS = [
    Request(rid=0, n=128, order=4, steps=37, arrival=0.0, seed=11),
    Request(rid=1, n=256, order=3, steps=20, arrival=0.0, seed=12, depth=0.2),
    Request(rid=2, n=128, order=5, steps=50, arrival=0.0, seed=13),
    Request(rid=3, n=64, order=6, steps=61, arrival=0.0, seed=14, precision="fp64"),
    Request(rid=4, n=128, order=4, steps=25, arrival=0.0, seed=15, depth=0.5),
]


def test_result_same_alone_and_in_mix():
    alone = {}
    for r in REQS:
        rr = copy.deepcopy(r)
        m = Server(chunk=16).run([rr], realtime=False)
        assert m["completed"] == 1
        alone[r.rid] = rr.result
    mix = [copy.deepcopy(r) for r in REQS]
    # staggered arrivals so that requests join and leave while others run
    for i, r in enumerate(mix):
        r.arrival = 0.02 * i
    m = Server(chunk=9).run(mix, realtime=True)
    assert m["completed"] == len(REQS)
    assert m["ensemble_rebuilds"] >= 2
    for r in mix:
        eta, phi = r.result
        assert np.array_equal(eta, alone[r.rid][0]), r.rid
        assert np.array_equal(phi, alone[r.rid][1]), r.rid
    assert m["p50_s"] is not None and m["p99_s"] >= m["p50_s"]


def test_admission_by_memory_budget():
    from hos_b200 import HosField

    one = HosField.footprint_bytes(256, 256, 4, "fp32")
    reqs = [Request(rid=i, n=256, order=4, steps=10, arrival=0.0, seed=i) for i in range(6)]
    srv = Server(chunk=5, hbm_budget_bytes=int(2.5 * one), reserve_bytes=0)
    m = srv.run(reqs, realtime=False)
    assert m["completed"] == 6
    # at most two fields fit at a time, so six requests need at least three ensembles
    assert m["ensemble_rebuilds"] >= 3


def test_device_free_bytes_counts_memory_of_released_fields():
    """Fields take their memory from a stream-ordered pool; memory a closed
    field leaves there counts as free for the next one."""
    import ctypes

    import torch

    from hos_b200 import HosField, _lib

    L = _lib.load()
    out = ctypes.c_size_t()
    f = HosField(512, 512, order=4, precision="fp32")
    f.close()
    torch.cuda.synchronize()
    assert L.hos_device_free_bytes(ctypes.byref(out)) == 0
    assert out.value >= torch.cuda.mem_get_info()[0]
    g = HosField(512, 512, order=4, precision="fp32")  # reuses the pool's memory
    assert L.hos_device_free_bytes(ctypes.byref(out)) == 0 and out.value > 0
    g.close()
