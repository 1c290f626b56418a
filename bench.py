#!/usr/bin/env python
"""Benchmark of the HOS time advance on B200: RK4 steps/s at 1024^2, M = 5.

Workload (the precision-form configuration): a directional JONSWAP sea on a
2 pi x 2 pi doubly periodic domain, Nx = Ny = 1024, HOS order M = 5, peak
wavenumber kp = 24, kp*Hs/2 = 0.12, gamma = 3.3, cos^(2s)(theta/2) spreading
with s = 10, seeded complex-Gaussian mode amplitudes, linear phi_s, g = 1,
deep water, RK4 with dt = Tp/50.  Synthetic data (seeded); the reference
ships no benchmark inputs.

One bench step = one RK4 step of that field.  ``value`` is the FP32-compute
form (FP32 transforms/products/RHS, FP64 RK state and diagnostics); the FP64
drop-in path is timed beside it, and both are run on to 1000 steps to report
the FP32 form's eta error relative to Hs.  Inputs are resident in HBM when
the timed region starts; the per-step working set (about 230 MB in FP32,
400 MB in FP64) exceeds the 126 MB L2, so no explicit flush is used.

``e2e`` is the same metric through the C ABI with host buffers: every step
uploads the packed spectral state from pinned host memory, advances one RK4
step and reads the state back.

With --gpus N (torchrun, one rank per GPU) every rank advances its own
independent field (replicas: the path does not shard); ``value`` counts the
steps of all ranks over the slowest rank's time.

--impl reference times the reference's own CPU implementation of the path
(the Csource/2dpar hot-path sources built with the single-rank FFTW-MPI shim,
oracle/_ref) on the same workload and prints the same JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 steps/s at 1024^2 M=5, FP32 vs FP64 (eta err<=1e-5); ensemble p50/p99 latency"
UNIT = "RK4 steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--order", type=int, default=5)
    ap.add_argument("--accuracy-steps", type=int, default=1000)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--ensemble-fields", type=int, default=256)
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--ensemble-mode", default="classes", choices=["persistent", "classes"])
    ap.add_argument("--serve-utilization", type=float, default=0.7)
    ap.add_argument("--serve-duration", type=float, default=20.0)
    ap.add_argument("--serve-limit", type=float, default=80.0)
    ap.add_argument("--serve-nominal-limit", type=float, default=25.0)
    return ap.parse_args()


def workload(n, order, seed):
    from hos_b200 import ic

    eta, phi, info = ic.jonswap(n, n, kp=24.0 * n / 1024, steepness=0.12, gamma=3.3, spread_s=10.0, seed=seed)
    dt = info["Tp"] / 50
    desc = (f"{n}x{n} M={order} JONSWAP kp={24.0 * n / 1024:g} kp*Hs/2=0.12 gamma=3.3 s=10 deep water, "
            f"RK4 dt=Tp/50, 2pi domain, g=1")
    return eta, phi, info, dt, desc


def config(args, desc):
    return {
        "workload": desc,
        "n": args.n,
        "order": args.order,
        "scheme": "RK4",
        "state": "FP64 spectral, resident in HBM",
        "l2": "per-step working set > 126 MB L2 (no flush)",
        "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU",
    }


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ------------------------------------------------------------------ helpers
def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the pass kinds from the committed ncu summary
    (profiles/ncu_traffic.txt: lines '<pass> <precision> <n> <bytes>')."""
    out = {}
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if os.path.exists(path):
        for line in open(path):
            f = line.split()
            if len(f) == 4 and not line.startswith("#"):
                out[(f[0], f[1], int(f[2]))] = float(f[3])
    return out


def algorithmic_step_bytes(n, order, prec_bytes):
    """Algorithmic bytes per RK4 step, 4*T_M*(R_p + C_p) + 26*C_64: each of the
    T_M transforms of the 4 RHS evaluations reads its input once and writes
    its output once, plus the FP64 state traffic of the stages."""
    tm = 6 + order + order * (order + 1) // 2
    R = n * n * prec_bytes
    C = n * (n // 2 + 1) * 2 * prec_bytes
    C64 = n * (n // 2 + 1) * 16
    return 4 * tm * (R + C) + 26 * C64


def pass_units(name, order):
    """Algorithmic work of one launch of a pass kind, in the units of the
    step model 4*T_M*(R_p + C_p) + 26*C_64: (2-D transforms the launch
    completes, FP64 spectral fields of RK state it moves).  A c2r transform
    completes in a y-inverse pass and an r2c one in an x-forward pass, so
    per RHS the stage y-inverse completes 5 + M, the level y-inverses
    M - n (n = 1..M-1, M/2 on average), each level x-forward 1 and the RHS
    x-forward 2: T_M = 6 + M + M(M+1)/2 in all.  The state share: the stage
    x-inverse reads u and one k (4 fields), the RHS x-forward writes k
    (2 fields) and, on the last of the 4 stages, u (2 more): 26 per RK4
    step.  Summed over a step's launches this is exactly the step model."""
    M = order
    return {
        "xinv_stage": (0.0, 4.0),
        "yinv_stage": (5.0 + M, 0.0),
        "yfwd_level": (0.0, 0.0),
        "xfwd_level": (1.0, 0.0),
        "yinv_level": (M / 2.0, 0.0),
        "yfwd_rhs": (0.0, 0.0),
        "xfwd_rhs": (2.0, 2.5),
    }.get(name, (0.0, 0.0))


def cpu_reference_rate(args, eta, phi, info, dt, max_seconds):
    """The reference's own hot path (oracle/_ref, all host threads) on the
    workload: RK4 steps/s over a bounded number of steps."""
    from oracle import ref_c

    if not ref_c.available(args.order):
        return None
    ref = ref_c.RefC(args.order, args.n, args.n, g=1.0, scheme=2)
    u = ref.init_state(eta, phi)
    t0 = time.perf_counter()
    u, t, _ = ref.steps(u, 0.0, dt, 1)
    first = time.perf_counter() - t0
    nsteps = max(1, min(20, int(max_seconds / max(first, 1e-9))))
    t0 = time.perf_counter()
    u, t, _ = ref.steps(u, t, dt, nsteps)
    el = time.perf_counter() - t0
    return {"value": nsteps / el, "steps": nsteps, "seconds": el}


# ------------------------------------------------------------------ ensemble and serving
def run_ensemble(args, rep):
    """256 independent JONSWAP fields (grids 128/256/512 with weights
    0.5/0.3/0.2, M in {3,4,5}, kp*Hs/2 uniform in [0.05, 0.12], kp = n/16,
    half deep water and half finite depth with kp*h uniform in [1, 3]) in
    FP32 compute / FP64 state, 500 RK4 steps each (dt = Tp/50), advanced as
    one ensemble; compared with the same fields advanced one after another
    in plain FP64.  With several GPUs the 256 fields are split over the
    ranks by estimated work (hos_b200.partition); the time is the slowest
    rank's."""
    import numpy as np
    import torch

    from hos_b200 import HosEnsemble, HosField
    from hos_b200.partition import Partition, work
    from hos_b200.serve import _dptr, jonswap_device

    rng = np.random.default_rng(0)
    specs = []
    for i in range(args.ensemble_fields):
        n = int(rng.choice([128, 256, 512], p=[0.5, 0.3, 0.2]))
        M = int(rng.choice([3, 4, 5]))
        kp = n / 16.0
        depth = None if i % 2 == 0 else float(rng.uniform(1.0, 3.0)) / kp
        specs.append((n, M, kp, float(rng.uniform(0.05, 0.12)), depth, 7000 + i))
    all_specs = specs
    part = Partition(all_specs, lambda sp: work(sp[0], sp[1], args.ensemble_steps), rep.rank, rep.world)
    specs = [sp for _, sp in part.mine]
    fields, dts, hs = [], [], []
    for (n, M, kp, st, depth, sd) in specs:
        eta, phi, tp = jonswap_device(n, kp, st, sd, depth=depth)
        f = HosField(n, n, order=M, precision="fp32", depth=depth)
        f._lib.hos_set_state_physical(f._h, _dptr(eta), _dptr(phi), 0.0)
        fields.append(f)
        dts.append(tp / 50)
        hs.append(2 * st / kp)
    def timed(mode, nsteps):
        ens = HosEnsemble(fields, dts, mode=mode)
        ens.step(3)
        ens.sync()
        torch.cuda.synchronize()
        rep.barrier()
        stream = torch.cuda.ExternalStream(ens.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        ens.step(nsteps)
        e1.record(stream)
        ens.sync()
        wall = time.perf_counter() - t0
        info = ens.info
        ens.close()
        return rep.max(e0.elapsed_time(e1) / 1e3), wall, info

    # the other mode first, on fewer steps, for comparison
    other = "classes" if args.ensemble_mode == "persistent" else "persistent"
    n_other = max(10, args.ensemble_steps // 5)
    el_o, _, info_o = timed(other, n_other)
    el, wall, info = timed(args.ensemble_mode, args.ensemble_steps)
    gp1 = sum(n * n for (n, *_r) in all_specs)
    gp = gp1 * args.ensemble_steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # sequential plain FP64: each (n, M, depth?) kind timed alone, weighted by the mix
    seq_s = 0.0
    rates = {}
    for (n, M, kp, st, depth, sd) in specs:
        key = (n, M, depth is not None)
        if key not in rates:
            eta, phi, tp = jonswap_device(n, kp, st, sd, depth=depth)
            g = HosField(n, n, order=M, precision="fp64", depth=depth)
            g._lib.hos_set_state_physical(g._h, _dptr(eta), _dptr(phi), 0.0)
            g.step(tp / 50, 3)
            g.sync()
            gs = torch.cuda.ExternalStream(g.stream)
            e0.record(gs)
            g.step(tp / 50, 30)
            e1.record(gs)
            g.sync()
            rates[key] = e0.elapsed_time(e1) / 1e3 / 30
            g.close()
        seq_s += rates[key] * args.ensemble_steps
    # accuracy of the FP32 members: four members rerun in FP64
    seq_s = rep.sum(seq_s)  # all fields one after another on one GPU
    errs = []
    for i in range(min(4, len(specs))):
        (n, M, kp, st, depth, sd) = specs[i]
        eta, phi, tp = jonswap_device(n, kp, st, sd, depth=depth)
        g = HosField(n, n, order=M, precision="fp64", depth=depth)
        g._lib.hos_set_state_physical(g._h, _dptr(eta), _dptr(phi), 0.0)
        g.step(tp / 50, 3 + n_other + 3 + args.ensemble_steps)  # every step the two timed ensembles took
        e64, _ = g.state_physical()
        e32, _ = fields[i].state_physical()
        errs.append(float(np.max(np.abs(e32 - e64)) / hs[i]))
        g.close()
    for f in fields:
        f.close()
    return {
        "fields": len(all_specs),
        "steps": args.ensemble_steps,
        "mode": args.ensemble_mode,
        "size_classes": info["classes"],
        "launches_per_step": info["launches_per_step"],
        "other_mode": {"mode": other, "steps": n_other, "launches_per_step": info_o["launches_per_step"],
                       "grid_point_steps_per_s": gp1 * n_other / el_o},
        "seconds": el,
        "grid_point_steps_per_s": gp / el,
        "sequential_fp64_seconds": seq_s,
        "sequential_fp64_grid_point_steps_per_s": gp / seq_s,
        "speedup_vs_sequential_fp64": seq_s / el,
        "eta_err_over_Hs_max_of_4_fp64_reruns": rep.max(max(errs) if errs else 0.0),
        "ranks": rep.world,
        "rank_work_imbalance": part.imbalance(),
        "wall_seconds": wall,
        "timing": "CUDA events on the ensemble's stream around the step-graph launches",
    }


def sequential_fp64_rate(reqs, cache):
    """Grid-point-steps/s of the requests run one after another in plain
    FP64 (each (n, M, depth?) kind timed once on 20 steps, weighted by the
    work the server did on each request: the steps it took, all of them for
    a completed request)."""
    import torch

    from hos_b200 import HosField
    from hos_b200.serve import _dptr, jonswap_device

    work = secs = 0.0
    for r in reqs:
        key = (r.n, r.order, r.depth is not None)
        if key not in cache:
            eta, phi, tp = jonswap_device(r.n, r.kp_value, r.steepness, r.seed, depth=r.depth)
            g = HosField(r.n, r.n, order=r.order, precision="fp64", depth=r.depth)
            g._lib.hos_set_state_physical(g._h, _dptr(eta), _dptr(phi), 0.0)
            g.step(tp / 50, 3)
            g.sync()
            st = torch.cuda.ExternalStream(g.stream)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            g.step(tp / 50, 20)
            e1.record(st)
            g.sync()
            cache[key] = e0.elapsed_time(e1) / 1e3 / 20
            g.close()
        work += r.n * r.n * r.steps_done
        secs += cache[key] * r.steps_done
    return work / secs if secs > 0 else None


def run_serving(args, capacity_gps):
    """The serving configuration: Poisson arrivals of JONSWAP simulations
    (grid uniform over 64^2..2048^2, M in 3..6, steps uniform in [100, 2000],
    half finite depth), FP32 compute / FP64 state, admitted by free HBM.
    Run twice: the nominal stream (200 requests/s for 10 s, about 100x what
    one B200 can absorb) with a time limit, reporting completions, backlog
    and the latency of what completed; and a stream at `serve_utilization`
    of the measured ensemble capacity, where continuous batching keeps up."""
    import numpy as np

    from hos_b200.serve import Server, poisson_requests

    sizes = np.array([64, 128, 256, 512, 1024, 2048], float)
    mean_work = float(np.mean(sizes**2)) * 1050.0  # E[n^2] * E[steps]
    nominal = poisson_requests(200.0, 10.0, seed=3)
    offered = sum(r.n * r.n * r.steps for r in nominal) / 10.0
    m_nom = Server(keep_results=False).run(nominal, realtime=True, time_limit=args.serve_nominal_limit)
    rate = args.serve_utilization * capacity_gps / mean_work
    reqs = poisson_requests(rate, args.serve_duration, seed=4)
    m = Server(keep_results=False).run(reqs, realtime=True, time_limit=args.serve_limit)
    done = [r for r in reqs if r.status == "done"]
    cache = {}
    seq = sequential_fp64_rate(done, cache) if done else None
    # the nominal stream ends at its time limit with requests still running:
    # the comparison covers every step the server took, finished or not
    worked = [r for r in nominal if r.steps_done > 0]
    seq_nom = sequential_fp64_rate(worked, cache) if worked else None
    m.update({
        "arrival_rate_per_s": rate,
        "arrival_window_s": args.serve_duration,
        "target_utilization": args.serve_utilization,
        "request_mix": "grid uniform over 64^2..2048^2 (powers of two), M in 3..6, steps uniform in [100, 2000], "
                       "half finite depth kp*h in [1,3], FP32 compute / FP64 state",
        "sequential_fp64_grid_point_steps_per_s": seq,
        "vs_sequential_fp64": (m["grid_point_steps_per_s"] / seq) if seq else None,
        "throughput_note": "arrival-limited: below capacity the aggregate over the wall clock is the offered load; "
                           "the nominal stream (overload) measures throughput",
        "nominal_stream": {
            "rate_per_s": 200.0, "window_s": 10.0, "requests": len(nominal), "time_limit_s": args.serve_nominal_limit,
            "offered_grid_point_steps_per_s": offered,
            "offered_over_capacity": offered / capacity_gps if capacity_gps else None,
            "completed": m_nom["completed"], "backlog_queued": m_nom["backlog_queued"],
            "backlog_running": m_nom["backlog_running"], "p50_s_of_completed": m_nom["p50_s"],
            "p99_s_of_completed": m_nom["p99_s"], "grid_point_steps_per_s": m_nom["grid_point_steps_per_s"],
            "sequential_fp64_grid_point_steps_per_s": seq_nom,
            "vs_sequential_fp64": (m_nom["grid_point_steps_per_s"] / seq_nom) if seq_nom else None,
            "ensemble_rebuilds": m_nom["ensemble_rebuilds"], "host_seconds": m_nom["host_seconds"],
        },
    })
    return m


# ------------------------------------------------------------------ reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    cores = int(os.environ["OMP_NUM_THREADS"])
    eta, phi, info, dt, desc = workload(args.n, args.order, seed=1000)
    from oracle import ref_c

    if not ref_c.available(args.order):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle)"}))
        return
    ref = ref_c.RefC(args.order, args.n, args.n, g=1.0, scheme=2)
    u = ref.init_state(eta, phi)
    t = 0.0
    # bounded: warm-up and timed counts are clipped so the run ends in a few minutes
    t0 = time.perf_counter()
    u, t, _ = ref.steps(u, t, dt, 1)
    per = time.perf_counter() - t0
    budget = 150.0
    warm = max(0, min(args.warmup - 1, int(0.2 * budget / per)))
    if warm:
        u, t, _ = ref.steps(u, t, dt, warm)
    k = max(1, min(args.steps, int(0.8 * budget / per)))
    t0 = time.perf_counter()
    u, t, _ = ref.steps(u, t, dt, k)
    el = time.perf_counter() - t0
    v = k / el
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": k,
        "warmup": warm + 1,
        "ms_per_step": 1e3 * el / k,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded JONSWAP)",
        "config": config(args, desc),
        "cpu_baseline": {
            "value": v,
            "unit": UNIT,
            "cores": cores,
            "kind": "reference",
            "sample": f"{k} RK4 steps of the {args.n}^2 M={args.order} field after {warm + 1} warm-up steps "
                      "(Csource/2dpar hot-path sources, single-rank FFTW-MPI shim, OpenMP FFT lines)",
        },
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line))


def run_configs(args):
    """The 512^2, M = 4 configuration of the benchmark set on the same GPU:
    a JONSWAP sea (kp = 16, kp*Hs/2 = 0.1, gamma = 3.3, s = 15, seed 2),
    RK4 with dt = Tp/50, 1000 timed steps, once with the reference's dealias
    rule (mx = floor(0.5 Nx/(1+0.5 L)) = 102) and once with the 2/3 rule
    (mx = my = 170): steps/s of both forms, and the FP64 energy and volume
    drift over the run."""
    import torch

    from hos_b200 import HosField, ic

    out = []
    eta, phi, info = ic.jonswap(512, 512, kp=16.0, steepness=0.1, gamma=3.3, spread_s=15.0, seed=2)
    dt = info["Tp"] / 50
    for rule, mx in (("reference rule, mx=102", None), ("2/3 rule, mx=my=170", 512 // 3)):
        rec = {"workload": f"512x512 M=4 JONSWAP kp=16 kp*Hs/2=0.1 s=15, dealias {rule}", "steps": 1000}
        for prec in ("fp64", "fp32"):
            f = HosField(512, 512, order=4, precision=prec, mx=mx, my=mx)
            f.set_state_physical(eta, phi)
            v0 = f.volume()
            f.step(dt, 5)
            f.sync()
            stream = torch.cuda.ExternalStream(f.stream)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            f.step(dt, 1000)
            e1.record(stream)
            f.sync()
            rec[prec] = {"steps_per_s": 1000 / (e0.elapsed_time(e1) / 1e3)}
            if prec == "fp64":
                _, H = f.energy_history()
                rec["fp64_energy_drift_rel"] = float(abs(H[-1] - H[0]) / abs(H[0]))
                rec["fp64_volume_drift"] = float(abs(f.volume() - v0))
            f.close()
        out.append(rec)
    return out


# ------------------------------------------------------------------ our arm
def run_legacy(args, eta, phi, dt, calls=40):
    """The reference's own entry point, sol_update_RK (time_schemes_par.c:28-121),
    called as its driver calls it (main_2d_par.c:304): FP64, the caller's
    pageable packed state advanced in place, runtime.dat appended every call.
    Calls per second by the host clock around `calls` calls, in the default
    mode (state copied in and out every call) and in resident mode."""
    import ctypes
    import math
    import tempfile
    import time

    import numpy as np

    from hos_b200 import _lib

    L = _lib.load()
    P = ctypes.c_void_p
    L.sol_update_RK.argtypes = [P, P, ctypes.c_double, P]
    L.fft_2d.argtypes = [P, P, P]
    L.hos_legacy_set_nlevs.argtypes = [ctypes.c_int]
    L.hos_legacy_set_resident.argtypes = [ctypes.c_int]
    L.Setup_TimeScheme.argtypes = [ctypes.c_int]
    n = args.n
    ctypes.c_int.in_dll(L, "Nx").value = n
    ctypes.c_int.in_dll(L, "Ny").value = n
    for name in ("Lx", "Ly"):
        ctypes.c_double.in_dll(L, name).value = 2 * math.pi
    for name in ("Kx0", "Ky0", "g"):
        ctypes.c_double.in_dll(L, name).value = 1.0
    ctypes.c_int.in_dll(L, "rampflg").value = 0
    al = n * (n // 2 + 1)
    ctypes.c_ssize_t.in_dll(L, "alloc_local").value = al
    ctypes.c_ssize_t.in_dll(L, "local_N").value = al
    ctypes.c_ssize_t.in_dll(L, "local_Nyhpo").value = n // 2 + 1
    ctypes.c_ssize_t.in_dll(L, "local_1_start").value = 0
    ctypes.c_int.in_dll(L, "mpi_rank").value = 0
    out = {}
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)  # runtime.dat
        try:
            L.hos_legacy_set_nlevs(args.order - 1)
            L.Setup_TimeScheme(2)  # RK4
            L.rhs_hos_setup()
            u = np.zeros((2, n // 2 + 1, n), complex)  # pageable, as fftw_alloc_complex returns
            for k, x in enumerate((eta, phi)):
                xp = np.zeros((n, n + 2))
                xp[:, :n] = x
                L.fft_2d(P(xp.ctypes.data), P(u[k].ctypes.data), None)
            t = np.zeros(1)
            for mode, res in (("default", 0), ("resident", 1)):
                L.hos_legacy_set_resident(res)
                for _ in range(3):
                    L.sol_update_RK(P(u.ctypes.data), P(t.ctypes.data), dt, None)
                t0 = time.perf_counter()
                for _ in range(calls):
                    L.sol_update_RK(P(u.ctypes.data), P(t.ctypes.data), dt, None)
                L.hos_legacy_sync()
                out[mode] = calls / (time.perf_counter() - t0)
            L.hos_legacy_set_resident(0)
            L.rhs_hos_clean()
        finally:
            os.chdir(cwd)
    return {"calls_per_s": out, "calls": calls, "precision": "fp64", "order": args.order, "grid": [n, n],
            "state_bytes_per_call": 2 * al * 16}


def run_ours(args, rep):
    import ctypes

    import numpy as np
    import torch

    from hos_b200 import HosField

    rank, world, local_rank = rep.rank, rep.world, rep.local_rank
    torch.cuda.set_device(local_rank)
    barrier, max_over_ranks = rep.barrier, rep.max

    eta, phi, info, dt, desc = workload(args.n, args.order, seed=rep.seed(1000))
    fields = {p: HosField(args.n, args.n, order=args.order, precision=p, tune="auto") for p in ("fp64", "fp32")}
    for f in fields.values():
        f.set_state_physical(eta, phi)
    clocks = Clocks(local_rank)
    timings = {}
    clocks.start()
    for p in ("fp64", "fp32"):
        f = fields[p]
        stream = torch.cuda.ExternalStream(f.stream)
        f.step(dt, args.warmup)
        f.sync()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f.step(dt, args.steps)
        e1.record(stream)
        f.sync()
        torch.cuda.synchronize()
        barrier()
        timings[p] = max_over_ranks(e0.elapsed_time(e1))
    clk = clocks.stop()
    steps_done = args.warmup + args.steps
    v64 = world * args.steps / (timings["fp64"] / 1e3)
    v32 = world * args.steps / (timings["fp32"] / 1e3)

    # per-pass live timing of the FP32 form -> dominant kernel roofline
    passes = fields["fp32"].profile_stage(dt, reps=5)
    dom = max(passes, key=lambda d: d["launches_per_stage"] * d["ms_per_launch"])
    peak, peak_kind = peaks()
    unit_bytes = args.n * args.n * 4 + args.n * (args.n // 2 + 1) * 8  # R_32 + C_32: one FP32 2-D transform
    c64 = args.n * (args.n // 2 + 1) * 16
    for d in passes:
        tr, st = pass_units(d["name"], args.order)
        d["transforms_per_launch"] = tr
        d["state_fields_per_launch"] = st
        d["algorithmic_bytes_per_launch"] = tr * unit_bytes + st * c64
    dom_bytes = dom["algorithmic_bytes_per_launch"]
    achieved = dom_bytes / (dom["ms_per_launch"] * 1e-3) / 1e9
    traffic = ncu_traffic().get((dom["name"], "fp32", args.n))
    stage_ms = sum(d["launches_per_stage"] * d["ms_per_launch"] for d in passes)

    # accuracy: both forms on to accuracy_steps, eta error relative to Hs
    for f in fields.values():
        if args.accuracy_steps > steps_done:
            f.step(dt, args.accuracy_steps - steps_done)
        f.sync()
    e64, p64 = fields["fp64"].state_physical()
    e32, p32 = fields["fp32"].state_physical()
    _, H64 = fields["fp64"].energy_history()
    _, H32 = fields["fp32"].energy_history()
    eta_err = float(np.max(np.abs(e32 - e64)) / info["Hs"])
    phi_err = float(np.max(np.abs(p32 - p64)) / np.max(np.abs(p64)))
    ham_err = float(np.max(np.abs(H32 - H64)) / np.max(np.abs(H64)))
    energy_drift = float(abs(H64[-1] - H64[0]) / abs(H64[0]))
    nsteps_acc = max(args.accuracy_steps, steps_done)

    # e2e through the C ABI with pinned host buffers
    f = fields["fp32"]
    u0, _ = f.state_spectral()
    host = torch.empty((2, args.n // 2 + 1, args.n), dtype=torch.complex128, pin_memory=True)
    hnp = host.numpy()
    hnp[...] = u0
    stream = torch.cuda.ExternalStream(f.stream)
    for _ in range(2):
        f.set_state_spectral(hnp)
        f.step(dt, 1)
        st = f.state_spectral()  # noqa: F841 (warm-up of the path)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    hp = ctypes.c_void_p(hnp.ctypes.data)
    rcs = 0
    for _ in range(args.e2e_steps):
        rcs |= f._lib.hos_set_state_spectral(f._h, hp, 0.0)
        rcs |= f._lib.hos_step(f._h, dt, 1)
        rcs |= f._lib.hos_get_state_spectral(f._h, hp, None)
    e1.record(stream)
    if rcs:
        raise RuntimeError("e2e path returned an error")
    f.sync()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    state_bytes = 2 * (args.n // 2 + 1) * args.n * 16

    line = {
        "metric": METRIC,
        "value": v32,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": timings["fp32"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 compute, f64 state",
        "data": "synthetic (seeded JONSWAP)",
        "config": config(args, desc),
        "roofline": {
            "bound": "hbm",
            "kernel": dom["name"],
            "achieved": achieved,
            "peak": peak,
            "peak_kind": f"{peak_kind} copy bandwidth (burst)",
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": traffic,
            "bytes_per_launch": dom_bytes,
            "bytes_rule": "2-D transforms completed per launch x (R_32 + C_32) + FP64 state fields x C_64",
            "transforms_per_launch": dom["transforms_per_launch"],
            "unit_bytes": unit_bytes,
            "pass_model_bytes_per_launch": dom["bytes_per_launch"],
            "ms_per_launch": dom["ms_per_launch"],
            "share_of_stage": dom["launches_per_stage"] * dom["ms_per_launch"] / stage_ms,
        },
        "passes": passes,
        "step_roofline": {
            "model_bytes_per_step": algorithmic_step_bytes(args.n, args.order, 4),
            "achieved_gbs": algorithmic_step_bytes(args.n, args.order, 4) / (timings["fp32"] / args.steps * 1e-3) / 1e9,
            "peak": peak,
        },
        "e2e": {
            "value": world * args.e2e_steps / (e2e_ms / 1e3),
            "unit": UNIT,
            "h2d_bytes_per_step": state_bytes + 8,
            "d2h_bytes_per_step": state_bytes + 8,
            "path": "hos_set_state_spectral (pinned host) + hos_step + hos_get_state_spectral",
        },
        "gpu_launches": args.steps * f.launches_per_step,
        "clocks": clk,
    }
    if not args.no_configs:
        line["other_configs"] = run_configs(args)
    if not args.no_ensemble:
        ens = run_ensemble(args, rep)
        line["ensemble"] = ens
        line["serving"] = run_serving(args, ens["grid_point_steps_per_s"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        cb = cpu_reference_rate(args, eta, phi, info, dt, max_seconds=20.0)
        if cb is not None:
            line["cpu_baseline"] = {
                "value": cb["value"],
                "unit": UNIT,
                "cores": int(os.environ["OMP_NUM_THREADS"]),
                "kind": "reference",
                "sample": f"{cb['steps']} RK4 steps ({cb['seconds']:.1f} s) of the same field on the host "
                          "(Csource/2dpar hot-path sources with the single-rank FFTW-MPI shim)",
            }
    dropin = run_legacy(args, eta, phi, dt)
    # the figures that describe the configurations, last so that a reader of
    # the line's tail sees them
    line["dropin"] = dropin
    line["fp64"] = {"value": v64, "ms_per_step": timings["fp64"] / args.steps}
    line["fp32_over_fp64"] = v32 / v64
    line["accuracy"] = {
        "steps": nsteps_acc,
        "eta_err_over_Hs": eta_err,
        "phi_err_rel": phi_err,
        "energy_err_rel": ham_err,
        "fp64_energy_drift_rel": energy_drift,
        "target_eta_err_over_Hs": 1e-5,
    }
    summ = {
        "fp32_steps_per_s": round(v32, 1),
        "fp64_steps_per_s": round(v64, 1),
        "fp32_over_fp64": round(v32 / v64, 3),
        "eta_err_over_Hs_1000_steps": eta_err,
        "phi_err_rel": phi_err,
        "energy_err_rel": ham_err,
        "step_roofline_frac": round(line["step_roofline"]["achieved_gbs"] / peak, 4),
        "dominant_pass_frac": round(achieved / peak, 4),
        "dropin_sol_update_RK_fp64_calls_per_s": {k: round(v, 1) for k, v in dropin["calls_per_s"].items()},
    }
    if "ensemble" in line:
        e = line["ensemble"]
        summ["ensemble"] = {k: e.get(k) for k in ("fields", "mode", "launches_per_step", "grid_point_steps_per_s",
                                                  "speedup_vs_sequential_fp64")}
        o = e.get("other_mode", {})
        seq_gps = e.get("sequential_fp64_grid_point_steps_per_s")
        summ["ensemble_" + str(o.get("mode"))] = {
            "launches_per_step": o.get("launches_per_step"), "grid_point_steps_per_s": o.get("grid_point_steps_per_s"),
            "speedup_vs_sequential_fp64": (o["grid_point_steps_per_s"] / seq_gps) if seq_gps and o else None}
    if "serving" in line:
        sv = line["serving"]
        summ["serving"] = {k: sv.get(k) for k in ("arrival_rate_per_s", "completed", "p50_s", "p99_s",
                                                  "grid_point_steps_per_s", "vs_sequential_fp64", "throughput_note")}
        nm = sv.get("nominal_stream", {})
        summ["serving_nominal_200_per_s"] = {k: nm.get(k) for k in ("completed", "backlog_queued", "backlog_running",
                                                                     "p50_s_of_completed", "p99_s_of_completed",
                                                                     "grid_point_steps_per_s", "vs_sequential_fp64")}
    line["summary"] = summ
    for fl in fields.values():
        fl.close()
    if rank == 0:
        print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    from hos_b200.replicas import Replicas

    with Replicas("nccl", timeout_s=120) as rep:
        run_ours(args, rep)


if __name__ == "__main__":
    main()
