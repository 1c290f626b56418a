"""Autotuner of the kernel shapes (elements per thread E and lines per block)
of the four pass kinds, and of the z-derivative orders per block of the
level x-forward pass, per grid, order and precision.

The objective is the time of a whole graph-launched RK step (CUDA events on
the handle's stream), so that the passes are measured as they run together.
Starting from the library's default shapes, each pass kind in turn tries
every candidate (E, lines-per-block scale, and for the x-forward kind the
orders per block) with the other kinds at their best so far, and keeps a
candidate only if it makes the step faster.  The result (the 8
``hos_params.tune`` values and ``tune_opb``) is cached in a JSON file keyed
by GPU name, grid, order and precision (``HOS_AUTOTUNE_CACHE``, default
``~/.cache/hos_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os

KINDS = {  # tune index of E, tune index of the scale, pass names of the kind
    "xi": (0, 4, ("xinv_stage",)),
    "xf": (1, 5, ("xfwd_level", "xfwd_rhs")),
    "yi": (2, 6, ("yinv_level",)),
    "yf": (3, 7, ("yfwd_level", "yfwd_rhs")),
    "ys": (10, 11, ("yinv_stage",)),
}


def cache_path():
    return os.environ.get("HOS_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "hos_b200", "autotune.json"))


def _gpu_name():
    try:
        import torch

        return torch.cuda.get_device_name()
    except Exception:
        return "unknown"


def _key(nx, ny, order, precision):
    return f"step12|{_gpu_name()}|{nx}x{ny}|M{order}|{precision}"


def _load():
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _valid_elems(precision, n):
    out = []
    for e in (8, 16, 32):
        if e == 32 and precision != "fp32":
            continue
        if n >= e and n // e <= 256 and (e != 32 or n >= 64):
            out.append(e)
    return out


# The library's default shapes (ElemChoice / default_elems in hos_engine.cu):
# E = 8 for every kind; lines-per-block scales xi, xf, yi, yf; all orders in
# one block; levels fused; the stage y-inverse with E = 16, scale -1.  The 12 values
# are hos_params.tune[8], tune_opb, tune_nofuse, tune_ys, tune_sys.
DEFAULT_SCALES = {"fp32": (1, 0, 0, 0), "fp64": (-1, 0, -1, -1)}


def default_tune(order, precision):
    return [8, 8, 8, 8, *DEFAULT_SCALES[precision], order, 0, 16, -1]


def _step_ms(field, dt, steps=20, reps=3):
    """Best of `reps` timings of `steps` graph-launched RK steps, ms per step."""
    import torch

    stream = torch.cuda.ExternalStream(field.stream)
    field.step(dt, 3)
    field.sync()
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        field.step(dt, steps)
        e1.record(stream)
        field.sync()
        best = min(best, e0.elapsed_time(e1) / steps)
    return best


def tune(nx, ny, order=5, precision="fp32", reps=3, use_cache=True, scales=(-1, 0, 1)):
    """Return the 12 tune values (see default_tune) for
    (nx, ny, order, precision), measuring and caching them if needed."""
    from . import ic
    from .field import HosField

    key = _key(nx, ny, order, precision)
    db = _load() if use_cache else {}
    if key in db:
        return list(db[key]["tune"])
    kp = max(2.0, min(nx, ny) / 42.0)
    eta, phi, info = ic.jonswap(nx, ny, kp=kp, steepness=0.08, seed=123)
    dt = info["Tp"] / 50
    report = {}
    failed = []

    def measure(t):
        try:
            f = HosField(nx, ny, order=order, precision=precision, tune=t)
        except Exception as ex:  # a shape this grid cannot use
            failed.append({"tune": list(t), "error": str(ex)})
            return None
        try:
            f.set_state_physical(eta, phi)
            return _step_ms(f, dt, reps=reps)
        except Exception as ex:  # a shape this device cannot launch: skip it
            failed.append({"tune": list(t), "error": str(ex)})
            return None
        finally:
            f.close()

    best = default_tune(order, precision)
    best_ms = measure(best)
    report["default"] = {"tune": list(best), "ms": best_ms}
    for kind, (ie, isc, _names) in KINDS.items():
        n = nx if kind[0] == "x" else ny // 2
        opbs = (1, 2, order) if kind == "xf" else (best[8],)
        tried = 0
        for e, s, ob in [(e, s, ob) for e in _valid_elems(precision, n) for s in scales for ob in opbs]:
            t = list(best)
            t[ie], t[isc], t[8] = e, s, ob
            if t == best:
                continue
            ms = measure(t)
            tried += 1
            if ms is not None and (best_ms is None or ms < 0.99 * best_ms):  # 1 % margin over timing noise
                best, best_ms = t, ms
        report[kind] = {"E": best[ie], "scale": best[isc], "opb": best[8], "ms": best_ms, "tried": tried}
    if use_cache:
        db = _load()
        db[key] = {"tune": best, "report": report, "failed": failed}
        path = cache_path()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"  # concurrent ranks each write their own
        with open(tmp, "w") as fh:
            json.dump(db, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return best
