"""The multi-GPU path is replicas only: N processes, each advancing its own
field, joined by a barrier and a max over ranks of the timed region.  These
tests run that plumbing as two gloo ranks on the CPU, including a rank that
leaves before a collective (the other rank's collective ends with an error
instead of waiting for good)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})


def _collectives(rank, world, port, q):
    _env(rank, world, port)
    from hos_b200.replicas import Replicas

    with Replicas("gloo", timeout_s=30) as rep:
        assert rep.distributed and rep.world == world and rep.rank == rank
        rep.barrier()
        mx = rep.max(10.0 * (rank + 1))
        sm = rep.sum(rank + 1)
        rate, ms = rep.rate(50, 100.0 + rank)  # 50 steps per rank; slowest rank 101 ms
        q.put((rank, rep.seed(1000), mx, sm, rate, ms))


def _leaver(rank, world, port, q):
    _env(rank, world, port)
    from hos_b200.replicas import Replicas

    rep = Replicas("gloo", timeout_s=5)
    rep.barrier()
    if rank == 1:
        _put_and_exit(q, (rank, "left"))  # leaves between steps, before the next collective
    try:
        rep.max(1.0)
        res = (rank, "no error")
    except Exception as e:  # noqa: BLE001
        res = (rank, type(e).__name__)
    _put_and_exit(q, res)


def _put_and_exit(q, item):
    q.put(item)
    q.close()
    q.join_thread()  # the item is through the pipe before the process ends
    os._exit(0)


def _run(fn, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank did not finish"
    out = []
    while not q.empty():
        out.append(q.get())
    return sorted(out), [p.exitcode for p in procs]


def test_two_rank_collectives():
    out, codes = _run(_collectives, 2)
    assert codes == [0, 0] and len(out) == 2
    for rank, seed, mx, sm, rate, ms in out:
        assert seed == 1000 + rank
        assert mx == 20.0 and sm == 3.0
        assert ms == 101.0 and rate == pytest.approx(2 * 50 / 0.101)


def test_rank_that_leaves_ends_the_other_ranks_collective():
    out, codes = _run(_leaver, 2)
    res = dict(out)
    assert res[1] == "left"
    assert res[0] != "no error"


def test_single_process_is_the_identity():
    from hos_b200.replicas import Replicas

    saved = {k: os.environ.pop(k, None) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        with Replicas("gloo") as rep:
            assert not rep.distributed and rep.world == 1
            rep.barrier()
            assert rep.max(3.5) == 3.5 and rep.sum(2) == 2.0
            assert rep.rate(10, 1000.0) == (10.0, 1000.0)
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v
