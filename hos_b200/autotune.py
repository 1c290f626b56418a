"""Autotuner of the kernel shapes (elements per thread E and lines per block)
of the four pass kinds, and of the z-derivative orders per block of the
level x-forward pass, per grid, order and precision.

Each pass kind (x-inverse, x-forward, y-inverse, y-forward) is tuned on its
own: for every candidate (E, lines-per-block scale) a handle is created with
that shape for the kind and defaults for the rest, a seeded sea is loaded,
and the kind's passes of one RK stage are timed with CUDA events on the
handle's stream (hos_profile_stage).  The fastest shape of each kind wins;
the result (the 8 ``hos_params.tune`` values and ``tune_opb``) is cached in a JSON file keyed
by GPU name, grid, order and precision (``HOS_AUTOTUNE_CACHE``, default
``~/.cache/hos_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os

KINDS = {  # tune index of E, tune index of the scale, pass names of the kind
    "xi": (0, 4, ("xinv_stage",)),
    "xf": (1, 5, ("xfwd_level", "xfwd_rhs")),
    "yi": (2, 6, ("yinv_stage", "yinv_level")),
    "yf": (3, 7, ("yfwd_level", "yfwd_rhs")),
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
    return f"{_gpu_name()}|{nx}x{ny}|M{order}|{precision}"


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


def _kind_ms(field, dt, names, reps):
    stats = field.profile_stage(dt, reps)
    return sum(s["launches_per_stage"] * s["ms_per_launch"] for s in stats if s["name"] in names)


def tune(nx, ny, order=5, precision="fp32", reps=5, use_cache=True, scales=(-1, 0, 1)):
    """Return the 9 tune values (8 shapes, then orders per block) for
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
    best = [0] * 9
    report = {}
    failed = []
    for kind, (ie, isc, names) in KINDS.items():
        n = nx if kind[0] == "x" else ny // 2
        results = []
        opbs = (1, 2, order) if kind == "xf" else (0,)
        for e, s, ob in [(e, s, ob) for e in _valid_elems(precision, n) for s in scales for ob in opbs]:
            t = [0] * 9
            t[ie], t[isc], t[8] = e, s, ob
            try:
                f = HosField(nx, ny, order=order, precision=precision, tune=t)
            except Exception:
                continue
            try:
                f.set_state_physical(eta, phi)
                f.step(dt, 2)
                f.sync()
                results.append((_kind_ms(f, dt, names, reps), e, s, ob))
            except Exception as ex:  # a shape this device cannot launch: skip it
                failed.append({"kind": kind, "E": e, "scale": s, "opb": ob, "error": str(ex)})
            finally:
                f.close()
        if results:
            ms, e, s, ob = min(results)
            best[ie], best[isc] = e, s
            if kind == "xf":
                best[8] = ob
            report[kind] = {"E": e, "scale": s, "opb": ob, "ms": ms, "tried": len(results)}
    if use_cache:
        db = _load()
        db[key] = {"tune": best, "report": report, "failed": failed}
        path = cache_path()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(db, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return best
