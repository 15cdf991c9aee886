"""Autotuner of the temporal-blocking depths per grid size.

The Jacobi loops run K sweeps per DRAM pass (pressure K = 1..4, momentum
K = 1..2).  Deeper passes read less DRAM per sweep but recompute more halo and
need more z-chunk overlap; which depth wins depends on the grid (small grids
have fewer blocks than SMs, large ones are bandwidth-bound).  The tuner times
every depth on the case itself with CUDA events (wf_time_kernel, cold L2) and
keeps the fastest, cached as JSON keyed by device and grid so a grid size is
tuned once.  Results never depend on the depth; only speed does.
"""
from __future__ import annotations

import json
import os

from . import _lib

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "windfvm", "autotune.json")
PRES_DEPTHS = (1, 2, 3, 4)
VEL_DEPTHS = (1, 2)


def _key(solver, device_name: str) -> str:
    c = solver.cfg
    return f"{device_name}|{c.nx}x{c.ny}x{c.nz}"


def _device_name(device: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def load_cache(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(path: str, cache: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune_batch(batch, widths=(1, 2, 4, 0), steps: int = 2) -> dict:
    """Picks the concurrency width of a BatchSolver (cases per concurrent
    chain) by timing `steps` batched steps per candidate; leaves the batch
    on the fastest.  The timed steps advance the cases."""
    best = None
    times = {}
    for w in widths:
        batch.set_width(w)
        batch.step(1)
        batch.prepare_graphs()  # no capture inside the timed steps
        batch.step(steps)
        ms = batch.last_step_ms() / steps
        times[w] = ms
        if best is None or ms < times[best]:
            best = w
    batch.set_width(best)
    batch.step(1)
    batch.prepare_graphs()
    return {"width": best, "ms_per_step": times}


def tune(solver, cache_path: str | None = DEFAULT_CACHE, reps: int = 5, device_name: str | None = None) -> dict:
    """Picks and applies the fastest blocking depths for `solver`'s grid.
    Returns {"pres_k", "vel_k", "pres_us_per_sweep", "vel_us_per_sweep",
    "cached"}."""
    name = device_name or _device_name()
    key = _key(solver, name)
    cache = load_cache(cache_path) if cache_path else {}
    if key in cache:
        e = dict(cache[key])
        solver.set_blocking(e["pres_k"], e["vel_k"])
        e["cached"] = True
        return e
    saved = solver.get_blocking()
    best_p, best_v = None, None
    for k in PRES_DEPTHS:
        solver.set_blocking(k, saved[1])
        ms, _, sweeps = solver.time_kernel(_lib.KERNEL_PRES_SWEEP, reps=reps, flush_l2=True)
        us = ms * 1e3 / sweeps
        if best_p is None or us < best_p[1]:
            best_p = (k, us)
    for k in VEL_DEPTHS:
        solver.set_blocking(best_p[0], k)
        ms, _, sweeps = solver.time_kernel(_lib.KERNEL_VEL_SWEEP, reps=reps, flush_l2=True)
        us = ms * 1e3 / sweeps
        if best_v is None or us < best_v[1]:
            best_v = (k, us)
    solver.set_blocking(best_p[0], best_v[0])
    e = {"pres_k": best_p[0], "vel_k": best_v[0], "pres_us_per_sweep": best_p[1], "vel_us_per_sweep": best_v[1]}
    if cache_path:
        cache[key] = e
        save_cache(cache_path, cache)
    return dict(e, cached=False)
