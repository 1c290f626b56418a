"""Serving: a continuous-batching request loop for HOS simulations.

A request asks for one wave field (grid n x n, order M, depth, sea state,
number of RK4 steps).  The server

* admits arrived requests while their device footprint
  (hos_footprint_bytes) fits in the free device memory (cudaMemGetInfo, less
  a reserve) and a slot is free; admission is in arrival order, and a
  request that does not fit does not block smaller ones behind it;
* keeps each admitted field's FP64 spectral state resident on the device
  (one ``HosField`` per request) until it finishes;
* advances all active fields together as one ``HosEnsemble`` (one launch
  per pass per size class, one CUDA graph per step) in chunks of at most
  ``chunk`` steps; requests that arrive meanwhile join at the next chunk
  boundary, and finished ones leave (their slot and memory are freed);
* records for each request its arrival, admission and completion times; the
  time-to-result is completion minus arrival and includes reading the
  result (eta, phi) back to the host.

Each field advances by exactly the same kernel sequence whether it runs
alone or among others, so a result does not depend on the mix
(tests/test_gpu_serve.py checks this bit for bit).

Initial conditions are generated on the device with torch (seeded JONSWAP
seas, the formulas of ``hos_b200.ic.jonswap``) so that input generation
does not hold the loop.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

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
    return (eta * scale).contiguous(), (phi * scale).contiguous(), 2 * math.pi / wp


class Server:
    def __init__(self, chunk=25, max_slots=4096, reserve_bytes=2 << 30, hbm_budget_bytes=None, keep_results=True):
        self.chunk = int(chunk)
        self.max_slots = int(max_slots)
        self.reserve = int(reserve_bytes)
        self.budget = hbm_budget_bytes  # optional cap on what the server may hold
        self.keep_results = keep_results
        self.rebuilds = 0
        self.chunks = 0

    def _free_bytes(self, held):
        import torch

        free, _total = torch.cuda.mem_get_info()
        avail = free - self.reserve
        if self.budget is not None:
            avail = min(avail, self.budget - held)
        return avail

    def run(self, requests, realtime=True, time_limit=None):
        """Serve the requests (sorted by arrival).  With realtime, a request
        becomes visible at its arrival time on the wall clock; otherwise all
        are visible at once.  Returns a metrics dict."""
        pending = sorted(requests, key=lambda r: r.arrival)
        active = []  # [req, field, dt, remaining]
        done = []
        held = 0
        ens = None
        dirty = False
        gp_steps = 0.0
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit:
                break
            # admission
            visible = [r for r in pending if (not realtime) or r.arrival <= now]
            for r in visible:
                if len(active) >= self.max_slots:
                    break
                need = HosField.footprint_bytes(r.n, r.n, r.order, r.precision)
                if need > self._free_bytes(held):
                    continue
                eta, phi, tp = jonswap_device(r.n, r.kp_value, r.steepness, r.seed, depth=r.depth)
                f = HosField(r.n, r.n, order=r.order, precision=r.precision, depth=r.depth)
                f._lib.hos_set_state_physical(f._h, _dptr(eta), _dptr(phi), 0.0)
                r.admitted = time.perf_counter() - t0
                active.append([r, f, tp / 50, r.steps])
                held += need
                pending.remove(r)
                dirty = True
            if not active:
                if pending and realtime:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - now)))
                elif pending:
                    raise RuntimeError("a request does not fit in device memory even alone")
                continue
            if dirty:
                if ens is not None:
                    ens.close()
                ens = HosEnsemble([a[1] for a in active], [a[2] for a in active])
                self.rebuilds += 1
                dirty = False
            steps = min(self.chunk, min(a[3] for a in active))
            ens.step(steps)
            ens.sync()
            self.chunks += 1
            for a in active:
                a[3] -= steps
                gp_steps += steps * a[0].n * a[0].n
            finished = [a for a in active if a[3] == 0]
            if finished:
                for a in finished:
                    r, f = a[0], a[1]
                    eta, phi = f.state_physical()
                    r.finished = time.perf_counter() - t0
                    if self.keep_results:
                        r.result = (eta, phi)
                    f.close()
                    held -= HosField.footprint_bytes(r.n, r.n, r.order, r.precision)
                    done.append(r)
                active = [a for a in active if a[3] > 0]
                if ens is not None:
                    ens.close()
                    ens = None
                dirty = bool(active)
        if ens is not None:
            ens.close()
        for a in active:
            a[1].close()
        wall = time.perf_counter() - t0
        ttr = np.array([r.finished - r.arrival for r in done]) if done else np.zeros(0)
        return {
            "completed": len(done),
            "submitted": len(requests),
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
