"""The serving loop's host logic (queueing, admission by free memory,
cancellation, per-request failure, thread-safe submission) against a fake
device backend: no GPU.  The device side of the same loop is covered by
tests/test_gpu_serve.py."""
import threading
import time

from hos_b200.serve import Request, Server


class FakeField:
    def __init__(self, r):
        self.r = r
        self.steps = 0
        self.closed = False


class FakeGroup:
    def __init__(self, fields, budgets):
        self.fields = list(fields)
        self.left = list(budgets)
        self.closed = False
        self.ok = True


class FakeBackend:
    """Footprint n*n*order bytes from a device of `capacity` bytes.  A request
    with seed < 0 'goes non-finite' at step -seed."""

    def __init__(self, capacity, on_advance=None):
        self.capacity = capacity
        self.held = 0
        self.peak_held = 0
        self.max_group = 0
        self.opened = []
        self.on_advance = on_advance

    def footprint(self, r):
        return r.n * r.n * r.order

    def free_bytes(self):
        return self.capacity - self.held

    def open(self, r):
        f = FakeField(r)
        self.held += self.footprint(r)
        self.peak_held = max(self.peak_held, self.held)
        self.opened.append(f)
        return f, 0.1

    def group(self, fields, dts, budgets):
        assert all(not f.closed for f in fields)
        assert all(b > 0 for b in budgets)
        self.max_group = max(self.max_group, len(fields))
        return FakeGroup(fields, budgets)

    def launch(self, g, steps):
        """Every member takes min(steps, its budget) steps, as the device does."""
        assert not g.closed
        g.ok = True
        for i, f in enumerate(g.fields):
            took = min(steps, g.left[i])
            f.steps += took
            g.left[i] -= took
            if f.r.seed < 0 and f.steps >= -f.r.seed:
                g.ok = False
        if self.on_advance:
            self.on_advance(self)

    def wait(self, g):
        return g.ok

    def remaining(self, g):
        return list(g.left)

    def failed_step(self, f):
        return -f.r.seed if f.r.seed < 0 and f.steps >= -f.r.seed else None

    def result(self, f):
        return (f.steps,)

    def close(self, obj):
        assert not obj.closed
        obj.closed = True
        if isinstance(obj, FakeField):
            self.held -= self.footprint(obj.r)


def reqs(k, n=8, order=2, steps=10):
    return [Request(rid=i, n=n, order=order, steps=steps + i, arrival=0.0, seed=i) for i in range(k)]


def test_every_request_gets_exactly_its_steps():
    be = FakeBackend(1 << 30)
    rs = reqs(7)
    m = Server(chunk=4, reserve_bytes=0, backend=be).run(rs, realtime=False)
    assert m["completed"] == 7 and m["submitted"] == 7
    for r in rs:
        assert r.status == "done" and r.result == (r.steps,) and r.steps_done == r.steps
    assert be.held == 0 and all(f.closed for f in be.opened)


def test_admission_respects_free_memory_and_budget():
    one = 8 * 8 * 2
    be = FakeBackend(3 * one + one // 2)
    m = Server(chunk=3, reserve_bytes=0, backend=be).run(reqs(9), realtime=False)
    assert m["completed"] == 9 and be.peak_held <= 3 * one and be.max_group == 3
    be = FakeBackend(1 << 30)
    m = Server(chunk=3, reserve_bytes=0, hbm_budget_bytes=2 * one, backend=be).run(reqs(5), realtime=False)
    assert m["completed"] == 5 and be.peak_held <= 2 * one


def test_small_requests_pass_a_large_one_that_does_not_fit_yet():
    be = FakeBackend(64 * 64 * 2)
    big = Request(rid=0, n=64, order=2, steps=5)
    small = [Request(rid=i, n=8, order=2, steps=30) for i in (1, 2)]
    # the small ones are admitted first (in arrival order) and hold memory;
    # the big one waits, is not rejected, and finishes after they leave
    for r in small:
        r.arrival = 0.0
    big.arrival = 0.001
    m = Server(chunk=10, reserve_bytes=0, backend=be).run(small + [big], realtime=False)
    assert m["completed"] == 3 and big.status == "done"
    assert big.admitted >= max(r.finished for r in small) - 1e-9


def test_request_larger_than_the_device_is_rejected():
    be = FakeBackend(1000)
    rs = [Request(rid=0, n=64, order=3, steps=5), Request(rid=1, n=8, order=2, steps=5)]
    m = Server(chunk=5, reserve_bytes=0, backend=be).run(rs, realtime=False)
    assert m["rejected"] == 1 and m["completed"] == 1
    assert rs[0].status == "rejected" and "bytes" in rs[0].error and rs[1].status == "done"


def test_nonfinite_request_fails_alone():
    be = FakeBackend(1 << 30)
    rs = reqs(4, steps=20)
    rs[2].seed = -7  # goes non-finite at step 7
    m = Server(chunk=5, reserve_bytes=0, backend=be).run(rs, realtime=False)
    assert m["failed"] == 1 and m["completed"] == 3
    assert rs[2].status == "failed" and "step 7" in rs[2].error and rs[2].result is None
    for r in rs[:2] + rs[3:]:
        assert r.status == "done" and r.result == (r.steps,)
    assert be.held == 0


def test_cancel_queued_and_active():
    srv = None
    calls = []

    def on_advance(be):
        calls.append(1)
        if len(calls) == 1:
            srv.cancel(1)  # active: leaves at the next chunk boundary

    be = FakeBackend(1 << 30, on_advance=on_advance)
    srv = Server(chunk=2, reserve_bytes=0, backend=be)
    rs = reqs(3, steps=20)
    srv.cancel(2)  # queued: never admitted
    m = srv.run(rs, realtime=False)
    assert m["cancelled"] == 2 and m["completed"] == 1
    assert rs[2].status == "cancelled" and rs[2].admitted is None
    assert rs[1].status == "cancelled" and rs[1].result is None
    assert rs[0].status == "done" and rs[0].result == (20,)
    assert be.held == 0 and all(f.closed for f in be.opened)


def test_submit_from_another_thread_while_running():
    be = FakeBackend(1 << 30)
    srv = Server(chunk=3, reserve_bytes=0, backend=be)
    late = reqs(4, steps=6)
    out = {}

    def serve():
        out["m"] = srv.run([], realtime=True, wait_for_more=True)

    th = threading.Thread(target=serve)
    th.start()
    for r in late:
        r.arrival = 0.0
        srv.submit(r)
        time.sleep(0.005)
    deadline = time.time() + 10
    while any(r.status != "done" for r in late) and time.time() < deadline:
        time.sleep(0.005)
    srv.stop()
    th.join(10)
    assert not th.is_alive()
    assert out["m"]["completed"] == 4 and out["m"]["submitted"] == 4
    assert all(r.result == (r.steps,) for r in late)


def test_inflight_work_bound_keeps_the_rest_queued():
    """With no room for admitted work beyond one request (max_inflight_s=0),
    requests run one at a time, in arrival order, and every one completes."""
    be = FakeBackend(1 << 30)
    rs = reqs(4, steps=8)
    m = Server(chunk=3, reserve_bytes=0, backend=be, max_inflight_s=0.0).run(rs, realtime=False)
    assert m["completed"] == 4 and be.max_group == 1
    assert [r.rid for r in sorted(rs, key=lambda r: r.admitted)] == [0, 1, 2, 3]
    assert all(r.result == (r.steps,) for r in rs)


def test_fields_created_on_the_opener_thread():
    """The same service with fields created on a thread beside the loop."""
    be = FakeBackend(3 * 8 * 8 * 2 + 10)
    rs = reqs(7)
    m = Server(chunk=4, reserve_bytes=0, backend=be, open_thread=True).run(rs, realtime=False)
    assert m["completed"] == 7 and be.peak_held <= 3 * 8 * 8 * 2
    for r in rs:
        assert r.status == "done" and r.result == (r.steps,)
    assert be.held == 0 and all(f.closed for f in be.opened)


def test_arrivals_while_others_run_join_at_a_replan():
    """Requests that arrive while a chunk runs are created in the chunk's
    window and join at a later re-plan (built during the chunk before it);
    each still gets exactly its steps."""
    be = FakeBackend(1 << 30, on_advance=lambda b: time.sleep(0.002))
    rs = reqs(6, steps=40)
    for i, r in enumerate(rs):
        r.arrival = 0.004 * i
    m = Server(chunk=2, reserve_bytes=0, backend=be, rebuild_seconds=0.01).run(rs, realtime=True)
    assert m["completed"] == 6 and m["ensemble_rebuilds"] >= 2
    # re-plans are built while the chunk before them runs
    assert m["rebuilds_prebuilt"] >= 1
    for r in rs:
        assert r.status == "done" and r.result == (r.steps,)
    assert be.held == 0 and all(f.closed for f in be.opened)
