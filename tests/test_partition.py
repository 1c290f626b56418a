"""Independent fields spread over ranks (hos_b200.partition): the work
split, and two gloo ranks on the CPU that each advance their share of an
ensemble and gather the results, which must equal what one rank computes
alone.  The fields are advanced by the oracle's numpy restatement here (no
GPU in these tests); on GPUs each rank runs its share through the library."""
import math
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from hos_b200.partition import Partition, assign, transforms_per_rhs, work

# (n, M, steps, seed): small fields of the restatement
SPECS = [(16, 3, 4, 1), (32, 4, 3, 2), (16, 5, 5, 3), (32, 3, 2, 4), (16, 4, 6, 5), (32, 5, 2, 6), (16, 3, 3, 7)]


def advance(spec):
    """The field's spectral state after its steps (RK4, dt = Tp/50)."""
    from hos_b200 import ic
    from oracle.hos_np import HosNumpy

    n, M, steps, seed = spec
    eta, phi, info = ic.jonswap(n, n, kp=n / 8.0, steepness=0.05, seed=seed)
    hn = HosNumpy(n, n, 2 * math.pi, 2 * math.pi, 1.0, M)
    e, p = hn.init_state(eta, phi)
    t = 0.0
    for _ in range(steps):
        e, p, t, _h = hn.step(e, p, t, info["Tp"] / 50, 2)
    return np.stack([e, p])


def work_of(spec):
    n, M, steps, _ = spec
    return work(n, M, steps)


def test_transforms_per_rhs():
    assert [transforms_per_rhs(M) for M in (3, 4, 5, 6)] == [15, 20, 26, 33]


def test_assignment_covers_every_field_and_balances():
    rng = np.random.default_rng(0)
    # the batched-ensemble mix: 256 fields, grids 128/256/512 (0.5/0.3/0.2), M in 3..5, 500 steps
    ns = rng.choice([128, 256, 512], size=256, p=[0.5, 0.3, 0.2])
    Ms = rng.choice([3, 4, 5], size=256)
    works = [work(int(n), int(M), 500) for n, M in zip(ns, Ms)]
    for world in (1, 2, 4, 8):
        ranks, load = assign(works, world)
        assert sorted(set(ranks)) == list(range(world))
        assert abs(sum(load) - sum(works)) < 1e-6 * sum(works)
        assert max(load) / (sum(load) / world) < 1.02
        # every rank computes the same assignment
        assert assign(works, world)[0] == ranks
    p = Partition(list(range(5)), lambda s: 1.0, rank=1, world=2)
    assert [i for i, _ in p.mine] == [1, 3]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from hos_b200.replicas import Replicas

    with Replicas("gloo", timeout_s=60) as rep:
        part = Partition(SPECS, work_of, rank=rep.rank, world=rep.world)
        results = [advance(s) for _, s in part.mine]
        allres = part.gather(results)
        q.put((rank, [i for i, _ in part.mine], allres))


def test_two_ranks_gather_what_one_rank_computes():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(60)
    assert [p.exitcode for p in procs] == [0, 0]
    out.sort(key=lambda x: x[0])
    mine0, mine1 = out[0][1], out[1][1]
    assert sorted(mine0 + mine1) == list(range(len(SPECS))) and not set(mine0) & set(mine1)
    alone = [advance(s) for s in SPECS]
    for _, _, allres in out:
        assert len(allres) == len(SPECS)
        for got, want in zip(allres, alone):
            assert np.array_equal(got, want)


def test_single_rank_partition_is_the_identity():
    part = Partition(SPECS, work_of, rank=0, world=1)
    assert [i for i, _ in part.mine] == list(range(len(SPECS)))
    assert part.gather(list(range(len(SPECS)))) == list(range(len(SPECS)))
