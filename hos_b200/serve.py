"""Serving: a continuous-batching request loop for HOS simulations.

A request asks for one wave field (grid n x n, order M, depth, sea state,
number of RK4 steps).  The server

* admits arrived requests while their device footprint
  (hos_footprint_bytes) fits in the free device memory (cudaMemGetInfo, less
  a reserve) and a slot is free; admission is in arrival order, and a
  request that does not fit does not block smaller ones behind it;
* keeps each admitted field's FP64 spectral state resident on the device
  (one ``HosField`` per request) until it finishes;
* advances all active fields together as one ``HosEnsemble`` (each member
  with its own step budget on the device) in chunks of about
  ``chunk_seconds``; requests that arrive meanwhile are admitted while the
  chunk runs, and a request stops at exactly its own number of steps, inside
  a chunk, and is read back at the chunk's end;
* re-plans the ensemble (new members join, finished ones leave and their
  memory is freed) at most every ``rebuild_seconds`` while members are still
  running: a finished member stays in the plan until then with its budget
  spent, so the device skips it;
* records for each request its arrival, admission and completion times; the
  time-to-result is completion minus arrival and includes reading the
  result (eta, phi) back to the host;
* fails a request alone when its state becomes non-finite (the step-end
  energy check on the device flags the member; the others continue), and
  takes cancellations between chunks.

Each field advances by exactly the same kernel sequence whether it runs
alone or among others, so a result does not depend on the mix
(tests/test_gpu_serve.py checks this bit for bit).

Initial conditions are generated on the device with torch (seeded JONSWAP
seas, the formulas of ``hos_b200.ic.jonswap``) so that input generation
does not hold the loop.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import HOS_ERR_NONFINITE, HosError
from ._lib import check as _lib_check
from .ensemble import HosEnsemble
from .field import HosField


@dataclass
class Request:
    rid: int
    n: int
    order: int
    steps: int
    arrival: float = 0.0  # seconds after the start of the run
    depth: float | None = None
    kp: float | None = None  # default n/16 (as a wavenumber on a 2 pi domain)
    steepness: float = 0.08
    seed: int = 0
    precision: str = "fp32"
    # filled by the server
    steps_done: int = 0  # steps taken so far (all of them once done)
    admitted: float | None = None
    finished: float | None = None
    status: str = "queued"  # queued, active, done, failed, cancelled, rejected
    error: str | None = None
    result: tuple | None = field(default=None, repr=False)

    @property
    def kp_value(self):
        return self.kp if self.kp is not None else max(2.0, self.n / 16.0)


def jonswap_device(n, kp, steepness, seed, depth=None, gamma=3.3, spread_s=10.0, g=1.0, device="cuda"):
    """Seeded directional JONSWAP sea on a 2 pi domain generated on the device
    (same spectrum, spreading, scaling and linear phi as hos_b200.ic.jonswap;
    the random numbers come from torch's generator).  Returns (eta, phi, Tp)
    as float64 device tensors [n, n]."""
    import torch

    # a stream of the greatest priority: a server generates seas while an
    # ensemble's chunk occupies the device
    side = torch.cuda.Stream(device=device, priority=-100)
    with torch.cuda.stream(side):
        eta, phi, tp = _jonswap_on_current_stream(n, kp, steepness, seed, depth, gamma, spread_s, g, device)
    # the library reads these on its own (non-blocking) streams: finish them here
    side.synchronize()
    return eta, phi, tp


def _jonswap_on_current_stream(n, kp, steepness, seed, depth, gamma, spread_s, g, device):
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    k1 = torch.fft.fftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    KX, KY = torch.meshgrid(k1, k1, indexing="ij")
    K = torch.hypot(KX, KY)
    Ks = torch.clamp(K, min=1e-300)

    def omega(k):
        return torch.sqrt(g * k * (torch.tanh(k * depth) if depth else 1.0))

    wp = math.sqrt(g * kp * (math.tanh(kp * depth) if depth else 1.0))
    W = omega(Ks)
    sigma = torch.where(W <= wp, 0.07, 0.09)
    r = torch.exp(-((W - wp) ** 2) / (2 * sigma**2 * wp**2))
    Sw = g * g * W**-5 * torch.exp(-1.25 * (wp / W) ** 4) * gamma**r
    if depth:
        th = torch.tanh(Ks * depth)
        dwdk = g * (th + Ks * depth * (1 - th * th)) / (2 * W)
    else:
        dwdk = 0.5 * torch.sqrt(g / Ks)
    theta = torch.atan2(KY, KX)
    F = Sw * dwdk * torch.cos(0.5 * theta) ** (2 * spread_s) / Ks
    F = torch.where(torch.isfinite(F) & (K > 0), F, torch.zeros_like(F))
    F[n // 2, :] = 0.0
    F[:, n // 2] = 0.0
    amp = torch.sqrt(2 * F)
    xr = torch.randn((n, n), generator=gen, device=device, dtype=torch.float64)
    xi = torch.randn((n, n), generator=gen, device=device, dtype=torch.float64)
    A = amp * torch.complex(xr, xi) / math.sqrt(2.0)
    P = torch.where(K > 0, -1j * g / W * A, torch.zeros_like(A))
    eta = torch.fft.ifft2(A).real * (n * n)
    phi = torch.fft.ifft2(P).real * (n * n)
    std = float(eta.std())
    scale = (2.0 * steepness / kp) / (4.0 * std) if std > 0 else 0.0
    eta, phi = (eta * scale).contiguous(), (phi * scale).contiguous()
    return eta, phi, 2 * math.pi / wp


class DeviceBackend:
    """The server's device side: one ``HosField`` per admitted request, one
    ``HosEnsemble`` over the active fields with a step budget per member
    (``mode``: "classes", one launch per pass per size class in a CUDA graph
    per step, the faster on B200 for this mix of grids; or "persistent", one
    launch per step).  The request loop in ``Server`` only calls these
    methods, so that its queueing, admission, cancellation and failure
    handling can be exercised without a GPU."""

    def __init__(self, mode="classes"):
        self.mode = mode

    def footprint(self, r):
        return HosField.footprint_bytes(r.n, r.n, r.order, r.precision)

    def free_bytes(self):
        """Free device memory, counting what the library's memory pool holds
        unused for new fields."""
        import ctypes

        from . import _lib

        out = ctypes.c_size_t()
        if _lib.load().hos_device_free_bytes(ctypes.byref(out)) == 0:
            return int(out.value)
        import torch  # the pool's figures are not available: the driver's free memory

        return torch.cuda.mem_get_info()[0]

    def open(self, r):
        """Creates the request's field with its initial sea; returns (field, dt)."""
        eta, phi, tp = jonswap_device(r.n, r.kp_value, r.steepness, r.seed, depth=r.depth)
        f = HosField(r.n, r.n, order=r.order, precision=r.precision, depth=r.depth)
        try:
            _lib_check(f._lib.hos_set_state_physical(f._h, _dptr(eta), _dptr(phi), 0.0))
        except Exception:
            f.close()
            raise
        return f, tp / 50

    def group(self, fields, dts, budgets):
        """One ensemble over the fields; member i takes at most budgets[i]
        more steps, whatever number of steps is launched."""
        g = HosEnsemble(fields, dts, mode=self.mode)
        try:
            g.set_steps(budgets)
        except Exception:
            g.close()
            raise
        return g

    def launch(self, group, steps):
        """Queues `steps` steps of every member that still has budget; returns at once."""
        group.step(steps)

    def busy(self, group):
        """Whether the group's queued steps are still running."""
        import torch

        st = getattr(group, "_query_stream", None)
        if st is None:
            st = group._query_stream = torch.cuda.ExternalStream(group.stream)
        return not st.query()

    def wait(self, group):
        """Waits for the queued steps; returns False when some member's
        state became non-finite (the others are unaffected)."""
        try:
            group.sync()
        except HosError as e:
            if e.code != HOS_ERR_NONFINITE:
                raise
            return False
        return True

    def remaining(self, group):
        return group.remaining()

    def failed_step(self, f):
        return f.health()

    def result(self, f):
        return f.state_physical()

    def close(self, obj):
        obj.close()


class Server:
    """Continuous-batching request loop (see the module docstring).

    ``run(requests)`` serves a list and returns metrics; ``submit`` and
    ``cancel`` may be called from other threads while ``run`` is active (a
    cancelled request leaves at the next chunk boundary, or before admission
    if it is still queued).  With ``wait_for_more=True`` the loop idles for
    new submissions until ``stop()`` is called.

    Admission takes requests in arrival order while their footprint fits the
    free device memory and the work already admitted (remaining grid-point
    steps over the measured rate) stays under ``max_inflight_s`` seconds;
    a request that does not fit does not block smaller ones behind it.

    The loop runs the active fields in chunks of ensemble steps, ``chunk``
    steps at most and about ``chunk_seconds`` of device time (sized from the
    previous chunk).  Every member has a step budget on the device, so a
    request stops at exactly its own number of steps inside a chunk and the
    others go on; it is read back at the chunk's end.  While a chunk runs, the
    loop admits arrived requests (creates their fields and uploads their
    initial seas) and closes the fields that left at the last re-plan.  The
    work list is re-planned (joins and leaves applied) at most every
    ``rebuild_seconds`` while members are running, at once when none is.

    Each request ends with ``status``: "done" (result read back), "failed"
    (its state became non-finite; ``error`` says at which step; the other
    fields of the batch continue unaffected), "cancelled", or "rejected" (its
    footprint exceeds what the device offers with the server holding
    nothing)."""

    def __init__(self, chunk=64, chunk_seconds=0.1, max_slots=4096, reserve_bytes=2 << 30, hbm_budget_bytes=None,
                 keep_results=True, backend=None, max_inflight_s=4.0, rebuild_seconds=0.5,
                 open_thread=False, prebuild=True):
        self.chunk = int(chunk)
        self.chunk_seconds = float(chunk_seconds)
        # joins and leaves are applied (the ensemble re-planned) at most this
        # often while members are still running
        self.rebuild_seconds = float(rebuild_seconds)
        # create fields on a thread beside the loop instead of inside the
        # chunk windows (measured slower on B200: the two threads' device
        # waits and frees contend)
        self.open_thread = bool(open_thread)
        # build the next plan while a chunk runs (the device does not wait
        # for the host's re-planning between chunks)
        self.prebuild = bool(prebuild)
        # admission also stops while the admitted work would take longer than
        # this at the measured rate (grid-point-steps/s), so that under
        # overload what is admitted finishes and the rest waits in the queue
        self.max_inflight_s = float(max_inflight_s)
        self.rate = 1e9
        self.max_slots = int(max_slots)
        self.reserve = int(reserve_bytes)
        self.budget = hbm_budget_bytes  # optional cap on what the server may hold
        self.keep_results = keep_results
        self.backend = backend if backend is not None else DeviceBackend()
        self.rebuilds = 0
        self.prebuilt_used = 0  # re-plans built while the previous chunk ran
        self.prebuilt_dropped = 0  # built during a chunk that did not go as predicted
        self.chunks = 0
        self._mu = threading.Lock()
        self._incoming = []
        self._cancelled = set()
        self._stop = threading.Event()

    # ------------------------------------------------------------ other threads
    def submit(self, req):
        """Queues a request; its ``arrival`` is taken as seconds after the
        start of the current (or next) ``run``."""
        with self._mu:
            self._incoming.append(req)

    def cancel(self, rid):
        with self._mu:
            self._cancelled.add(rid)

    def stop(self):
        self._stop.set()

    # ------------------------------------------------------------ the loop
    def _avail(self, held, booked=0):
        """Bytes a new field may take: the device's free memory less the
        reserve and less `booked` (admitted fields not yet allocated), and
        at most what the budget leaves beside the `held` bytes."""
        avail = self.backend.free_bytes() - self.reserve - booked
        if self.budget is not None:
            avail = min(avail, self.budget - held)
        return avail

    def run(self, requests=(), realtime=True, time_limit=None, wait_for_more=False):
        """Serve the requests (sorted by arrival) and any submitted meanwhile.
        With realtime, a request becomes visible at its arrival time on the
        wall clock; otherwise all are visible at once.  With time_limit the
        loop stops after that many seconds and reports what is still queued
        or running as backlog.  Returns a metrics dict."""
        be = self.backend
        self._stop.clear()
        pending = sorted(requests, key=lambda r: r.arrival)
        submitted = len(pending)
        active = []  # [req, field, dt, remaining steps], in ensemble order
        staged = []  # opened fields waiting for the next re-plan to join
        done = []
        ended = []  # failed, cancelled and rejected requests
        st = {"held": 0}
        ens = None
        dirty = False
        gp_steps = 0.0
        step_s = None  # seconds per step of the last chunk
        # host seconds spent in each part of the loop (the rest is waiting
        # for the device in `wait` or idling for arrivals); "open" runs on
        # the opener thread, beside the loop
        spent = {"open": 0.0, "group": 0.0, "wait": 0.0, "result": 0.0, "close": 0.0}
        t0 = time.perf_counter()
        last_build = None  # run time of the last ensemble build
        to_close = []  # finished members dropped from the ensemble: closed while the next chunk runs
        nxt = None  # (ensemble, kept members, joining fields, predicted budgets) built during a chunk

        # The loop decides what to admit (memory and in-flight work are booked
        # at once) and queues it; the fields are created (initial sea,
        # allocation, upload: each waits on the device) while a chunk runs,
        # for as long as it runs, or on a thread of their own with
        # open_thread.  They come back through `opened` and join at a re-plan.
        olock = threading.Lock()
        to_open = queue.Queue()
        opening = []  # requests handed to the opener and not yet back
        opened = []  # [req, field, dt, steps] ready to join
        open_failed = []  # (req, error) of fields that could not be created
        skipped = []  # admitted, not opened when the run ended (backlog)
        stop_open = threading.Event()

        def open_one(r):
            to = time.perf_counter()
            try:
                f, dt = be.open(r)
                item, err = [r, f, dt, r.steps], None
            except Exception as e:  # this request fails alone
                item, err = None, e
            with olock:
                spent["open"] += time.perf_counter() - to
                opening.remove(r)
                if item is not None:
                    opened.append(item)
                else:
                    open_failed.append((r, err))

        def opener():
            while True:
                r = to_open.get()
                if r is None:
                    return
                if stop_open.is_set():
                    with olock:
                        opening.remove(r)
                        skipped.append(r)
                    continue
                open_one(r)

        def open_inline(running):
            """Opens queued requests on this thread: all of them when the
            device is idle (`running` None), else while the chunk `running`
            is still in flight (at least one)."""
            k = 0
            while True:
                if running is not None and k > 0 and not busy(running):
                    return
                try:
                    r = to_open.get_nowait()
                except queue.Empty:
                    return
                open_one(r)
                k += 1

        othread = None
        if self.open_thread:
            othread = threading.Thread(target=opener, name="hos-serve-opener", daemon=True)
            othread.start()

        def retire(a, status, error=None):
            r = a[0]
            r.status, r.error = status, error
            r.finished = time.perf_counter() - t0
            tc = time.perf_counter()
            be.close(a[1])
            spent["close"] += time.perf_counter() - tc
            st["held"] -= be.footprint(r)
            ended.append(r)

        def intake():
            nonlocal pending, submitted
            with self._mu:
                if self._incoming:
                    submitted += len(self._incoming)
                    pending = sorted(pending + self._incoming, key=lambda r: r.arrival)
                    self._incoming = []
                return set(self._cancelled)

        def collect(cancelled):
            """Moves the fields the opener finished into `staged`."""
            with olock:
                got, bad = opened[:], open_failed[:]
                opened.clear()
                open_failed.clear()
            for a in got:
                if a[0].rid in cancelled:
                    retire(a, "cancelled")
                else:
                    staged.append(a)
            for r, e in bad:
                r.status, r.error = "failed", f"could not create the field: {e}"
                r.finished = time.perf_counter() - t0
                st["held"] -= be.footprint(r)
                ended.append(r)

        def admit(inflight):
            """Admits visible requests in arrival order while they fit and
            hands them to the opener; a request that does not fit does not
            block smaller ones behind it.  `inflight` lists the admitted
            [req, field, dt, remaining] entries; requests being opened count
            too."""
            now = time.perf_counter() - t0
            with olock:
                busy_open = list(opening)
            nslots = len(inflight) + len(busy_open)
            work = sum(a[3] * a[0].n * a[0].n for a in inflight) + sum(r.steps * r.n * r.n for r in busy_open)
            booked = sum(be.footprint(r) for r in busy_open)  # not yet in the device's free memory
            taken = 0
            for r in [r for r in pending if (not realtime) or r.arrival <= now]:
                if nslots + taken >= self.max_slots:
                    break
                rwork = r.steps * r.n * r.n
                if nslots + taken > 0 and work + rwork > self.max_inflight_s * self.rate:
                    continue
                need = be.footprint(r)
                if need > self._avail(st["held"], booked):
                    if nslots + taken == 0 and st["held"] == 0:
                        r.status, r.error = "rejected", f"needs {need} bytes of device memory"
                        pending.remove(r)
                        ended.append(r)
                    continue
                r.admitted = time.perf_counter() - t0
                r.status = "active"
                work += rwork
                st["held"] += need
                booked += need
                pending.remove(r)
                with olock:
                    opening.append(r)
                to_open.put(r)
                taken += 1
            return taken

        def busy(group):
            f = getattr(be, "busy", None)
            return True if f is None else f(group)

        def release(items):
            tc = time.perf_counter()
            for a in items:
                be.close(a[1])
                st["held"] -= be.footprint(a[0])
            spent["close"] += time.perf_counter() - tc

        def n_opening():
            with olock:
                return len(opening)

        try:
            while True:
                cancelled = intake()
                collect(cancelled)
                if not (pending or active or staged or n_opening()):
                    if wait_for_more and not self._stop.is_set():
                        time.sleep(0.002)
                        continue
                    break
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit:
                    break
                # cancellation: queued requests leave at once, admitted ones here
                for r in [r for r in pending if r.rid in cancelled]:
                    r.status = "cancelled"
                    pending.remove(r)
                    ended.append(r)
                for a in [a for a in staged if a[0].rid in cancelled]:
                    retire(a, "cancelled")
                    staged.remove(a)
                for a in [a for a in active if a[0].rid in cancelled and a[0].status == "active"]:
                    retire(a, "cancelled")
                    active.remove(a)
                    dirty = True  # the ensemble holds a closed field: re-plan before the next launch
                admit(active + staged)
                if not any(a[3] > 0 for a in active):
                    # nothing left to run: drop the finished members; the device
                    # is idle, so wait for the fields being opened and start
                    # with all of them
                    if ens is not None:
                        be.close(ens)
                        ens = None
                    if active or to_close:
                        release(active + to_close)
                        active, to_close = [], []
                    if n_opening():
                        if othread is None:
                            open_inline(None)
                        else:
                            time.sleep(0.0005)
                        continue
                    if not staged:
                        if pending and realtime:
                            time.sleep(max(0.0, min(0.002, pending[0].arrival - now)))
                        continue
                # membership changes (joins, finished members leaving) are
                # applied at most every rebuild_seconds while members are still
                # running, so that the ensemble is not re-planned after every
                # chunk under load
                zombies = [a for a in active if a[3] == 0]
                runnable = len(active) > len(zombies)
                due = last_build is None or now - last_build >= self.rebuild_seconds
                if ens is None or dirty or not runnable or ((staged or zombies) and due):
                    tg = time.perf_counter()
                    if ens is not None:
                        be.close(ens)
                        ens = None
                    pre, nxt = nxt, None
                    if pre is not None:
                        # the plan built during the last chunk holds when that
                        # chunk went as predicted and its new fields are still here
                        p_ens, p_keep, p_new, p_left = pre
                        if (not dirty and all(a[3] == left for a, left in zip(p_keep, p_left))
                                and all(any(x is a for x in staged) for a in p_new)):
                            kept = {id(a) for a in p_keep}
                            to_close += [a for a in active if id(a) not in kept]
                            joined = {id(a) for a in p_new}
                            active = p_keep + p_new
                            staged = [a for a in staged if id(a) not in joined]
                            ens = p_ens
                            self.prebuilt_used += 1
                        else:
                            be.close(p_ens)
                            self.prebuilt_dropped += 1
                    if ens is None:
                        to_close += zombies
                        active = [a for a in active if a[3] > 0] + staged
                        staged = []
                        if active:
                            ens = be.group([a[1] for a in active], [a[2] for a in active], [a[3] for a in active])
                    dirty = False
                    if ens is not None:
                        self.rebuilds += 1
                        last_build = now
                    spent["group"] += time.perf_counter() - tg
                    if not active:
                        continue
                elif nxt is not None:
                    be.close(nxt[0])
                    nxt = None
                    self.prebuilt_dropped += 1
                longest = max(a[3] for a in active)
                steps = self.chunk if step_s is None else int(max(1, min(self.chunk, self.chunk_seconds / step_s)))
                steps = min(steps, longest)
                t_launch = time.perf_counter()
                be.launch(ens, steps)
                # while the chunk runs: create the admitted fields (they join at
                # a later re-plan), then close the fields that left at the last
                # re-plan (closing waits for the device, which keeps running)
                if othread is None:
                    open_inline(ens)
                if to_close:
                    release(to_close)
                    to_close = []
                # when a re-plan is due after this chunk, build it now, while
                # the chunk runs: the members that keep running (with the
                # budgets they will have) and the fields opened so far
                t_end = time.perf_counter() - t0 + (step_s * steps if step_s else 0.0)  # when the chunk should end
                leaving = any(a[3] <= steps for a in active)
                if (not dirty and (staged or leaving) and self.prebuild
                        and (last_build is None or t_end - last_build >= self.rebuild_seconds)):
                    keep = [a for a in active if a[3] > steps]
                    new_fields = list(staged)
                    if keep or new_fields:
                        tg = time.perf_counter()
                        left = [a[3] - steps for a in keep]
                        members = keep + new_fields
                        g = be.group([a[1] for a in members], [a[2] for a in members],
                                     left + [a[3] for a in new_fields])
                        nxt = (g, keep, new_fields, left)
                        spent["group"] += time.perf_counter() - tg
                tw = time.perf_counter()
                healthy = be.wait(ens)
                spent["wait"] += time.perf_counter() - tw
                chunk_s = time.perf_counter() - t_launch
                step_s = chunk_s / steps
                self.chunks += 1
                rem = be.remaining(ens)
                chunk_gp = 0.0
                for a, left in zip(active, rem):
                    took = a[3] - left
                    chunk_gp += took * a[0].n * a[0].n
                    a[3] = left
                    a[0].steps_done = a[0].steps - left
                gp_steps += chunk_gp
                if chunk_gp > 0 and chunk_s > 0:
                    self.rate = 0.7 * self.rate + 0.3 * (chunk_gp / chunk_s)
                if not healthy:
                    bad = [(a, be.failed_step(a[1])) for a in active if a[0].status == "active"]
                    bad = [(a, s) for a, s in bad if s is not None]
                    for a, s in bad:
                        retire(a, "failed", f"state became non-finite at step {s}")
                    ids = {id(a) for a, _ in bad}
                    active = [a for a in active if id(a) not in ids]
                    dirty = dirty or bool(bad)
                # finished members are read back now and leave the ensemble at
                # the next re-plan (their budget is spent: the device skips them)
                for a in [a for a in active if a[3] == 0 and a[0].status == "active"]:
                    r, f = a[0], a[1]
                    tr = time.perf_counter()
                    res = be.result(f)
                    spent["result"] += time.perf_counter() - tr
                    r.finished = time.perf_counter() - t0
                    r.status = "done"
                    if self.keep_results:
                        r.result = res
                    done.append(r)
        finally:
            # the opener skips what it has not started, finishes what it has
            stop_open.set()
            if othread is not None:
                to_open.put(None)
                othread.join()
            while True:
                try:
                    r = to_open.get_nowait()
                except queue.Empty:
                    break
                if r is not None:
                    opening.remove(r)
                    skipped.append(r)
        collect(set())
        if nxt is not None:
            be.close(nxt[0])
        if ens is not None:
            be.close(ens)
        backlog_running = sum(1 for a in active if a[0].status == "active") + len(staged) + len(skipped)
        for a in active + staged + to_close:
            be.close(a[1])
        wall = time.perf_counter() - t0
        ttr = np.array([r.finished - r.arrival for r in done]) if done else np.zeros(0)
        count = lambda s: sum(1 for r in ended if r.status == s)  # noqa: E731
        return {
            "completed": len(done),
            "submitted": submitted,
            "failed": count("failed"),
            "cancelled": count("cancelled"),
            "rejected": count("rejected"),
            "backlog_queued": len(pending),
            "backlog_running": backlog_running,
            "wall_s": wall,
            "p50_s": float(np.percentile(ttr, 50)) if len(ttr) else None,
            "p99_s": float(np.percentile(ttr, 99)) if len(ttr) else None,
            "grid_point_steps": gp_steps,
            "grid_point_steps_per_s": gp_steps / wall if wall > 0 else 0.0,
            "ensemble_rebuilds": self.rebuilds,
            "rebuilds_prebuilt": self.prebuilt_used,
            "prebuilt_dropped": self.prebuilt_dropped,
            "chunks": self.chunks,
            "host_seconds": {k: round(v, 3) for k, v in spent.items()},
        }


def _dptr(t):
    import ctypes

    return ctypes.c_void_p(t.data_ptr())


def poisson_requests(rate, duration, seed=0, sizes=(64, 128, 256, 512, 1024, 2048), orders=(3, 4, 5, 6),
                     steps=(100, 2000), finite_depth_frac=0.5, precision="fp32", max_requests=None):
    """Poisson arrivals (rate per second for duration seconds); grid uniform
    over sizes, order uniform over orders, steps uniform in [steps], half
    deep water and half finite depth with kp*h uniform in [1, 3]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and len(out) >= max_requests):
            break
        n = int(rng.choice(sizes))
        kp = max(2.0, n / 16.0)
        depth = None
        if rng.random() < finite_depth_frac:
            depth = float(rng.uniform(1.0, 3.0)) / kp
        out.append(Request(rid=len(out), n=n, order=int(rng.choice(orders)), steps=int(rng.integers(steps[0], steps[1] + 1)),
                           arrival=t, depth=depth, kp=kp, seed=int(rng.integers(1 << 30)), precision=precision))
    return out
