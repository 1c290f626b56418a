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
  ``chunk_seconds``; requests
  that arrive meanwhile are admitted while the chunk runs and join at its
  end, and a request stops at exactly its own number of steps, inside a
  chunk, and leaves at the chunk's end (its slot and memory are freed);
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
    # the library reads these on its own (non-blocking) streams: finish them here
    torch.cuda.current_stream(eta.device).synchronize()
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
        import torch

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
    previous chunk).  Every member has a step budget on the device, so a request stops at exactly its own number of
    steps inside a chunk and the others go on.  While a chunk runs, the loop
    admits arrived requests (creates their fields and uploads their initial
    seas); they join at the chunk's end, when the work list is re-planned.

    Each request ends with ``status``: "done" (result read back), "failed"
    (its state became non-finite; ``error`` says at which step; the other
    fields of the batch continue unaffected), "cancelled", or "rejected" (its
    footprint exceeds what the device offers with the server holding
    nothing)."""

    def __init__(self, chunk=64, chunk_seconds=0.05, max_slots=4096, reserve_bytes=2 << 30, hbm_budget_bytes=None,
                 keep_results=True, backend=None, max_inflight_s=4.0):
        self.chunk = int(chunk)
        self.chunk_seconds = float(chunk_seconds)
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
    def _avail(self, held):
        avail = self.backend.free_bytes() - self.reserve
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
        active = []  # [req, field, dt, remaining steps]
        staged = []  # admitted while a chunk ran; they join at its end
        done = []
        ended = []  # failed, cancelled and rejected requests
        st = {"held": 0}
        ens = None
        dirty = False
        gp_steps = 0.0
        step_s = None  # seconds per step of the last chunk
        t0 = time.perf_counter()

        def retire(a, status, error=None):
            r = a[0]
            r.status, r.error = status, error
            r.finished = time.perf_counter() - t0
            be.close(a[1])
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

        def admit(inflight):
            """Admits visible requests in arrival order while they fit; a
            request that does not fit does not block smaller ones behind it.
            `inflight` lists the admitted [req, field, dt, remaining] entries."""
            now = time.perf_counter() - t0
            out = []
            nslots = len(inflight)
            work = sum(a[3] * a[0].n * a[0].n for a in inflight)
            for r in [r for r in pending if (not realtime) or r.arrival <= now]:
                if nslots + len(out) >= self.max_slots:
                    break
                rwork = r.steps * r.n * r.n
                if nslots + len(out) > 0 and work + rwork > self.max_inflight_s * self.rate:
                    continue
                need = be.footprint(r)
                if need > self._avail(st["held"]):
                    if nslots + len(out) == 0 and st["held"] == 0:
                        r.status, r.error = "rejected", f"needs {need} bytes of device memory"
                        pending.remove(r)
                        ended.append(r)
                    continue
                f, dt = be.open(r)
                r.admitted = time.perf_counter() - t0
                r.status = "active"
                out.append([r, f, dt, r.steps])
                work += rwork
                st["held"] += need
                pending.remove(r)
            return out

        while True:
            cancelled = intake()
            if not (pending or active or staged):
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
            for group_list in (active, staged):
                gone = [a for a in group_list if a[0].rid in cancelled]
                for a in gone:
                    retire(a, "cancelled")
                    group_list.remove(a)
                    dirty = True
            if staged:
                active += staged
                staged = []
                dirty = True
            new = admit(active)
            if new:
                active += new
                dirty = True
            if not active:
                if pending and realtime:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - now)))
                continue
            if dirty or ens is None:
                if ens is not None:
                    be.close(ens)
                ens = be.group([a[1] for a in active], [a[2] for a in active], [a[3] for a in active])
                self.rebuilds += 1
                dirty = False
            longest = max(a[3] for a in active)
            steps = self.chunk if step_s is None else int(max(1, min(self.chunk, self.chunk_seconds / step_s)))
            steps = min(steps, longest)
            t_launch = time.perf_counter()
            be.launch(ens, steps)
            # while the chunk runs: admit what has arrived (joins at its end)
            cancelled = intake()
            staged += admit(active + staged)
            healthy = be.wait(ens)
            chunk_s = time.perf_counter() - t_launch
            step_s = chunk_s / steps
            self.chunks += 1
            rem = be.remaining(ens)
            chunk_gp = 0.0
            for a, left in zip(active, rem):
                took = a[3] - left
                chunk_gp += took * a[0].n * a[0].n
                a[3] = left
            gp_steps += chunk_gp
            if chunk_gp > 0 and chunk_s > 0:
                self.rate = 0.7 * self.rate + 0.3 * (chunk_gp / chunk_s)
            if not healthy:
                bad = [(a, be.failed_step(a[1])) for a in active]
                bad = [(a, s) for a, s in bad if s is not None]
                for a, s in bad:
                    retire(a, "failed", f"state became non-finite at step {s}")
                ids = {id(a) for a, _ in bad}
                active = [a for a in active if id(a) not in ids]
                dirty = dirty or bool(bad)
            finished = [a for a in active if a[3] == 0]
            for a in finished:
                r, f = a[0], a[1]
                res = be.result(f)
                r.finished = time.perf_counter() - t0
                r.status = "done"
                if self.keep_results:
                    r.result = res
                be.close(f)
                st["held"] -= be.footprint(r)
                done.append(r)
            if finished:
                active = [a for a in active if a[3] > 0]
                dirty = True
            if dirty and ens is not None:
                be.close(ens)
                ens = None
        if ens is not None:
            be.close(ens)
        backlog_running = len(active) + len(staged)
        for a in active + staged:
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
            "chunks": self.chunks,
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
