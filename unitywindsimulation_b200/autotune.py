"""Autotuner of the Jacobi kernels' tile shapes and temporal-blocking
depths per grid size, and of the batched form's mode.

The Jacobi loops run K sweeps per DRAM pass (pressure K = 1..4, momentum
K = 1..2).  Deeper passes read less DRAM per sweep but recompute more halo and
need more z-chunk overlap; which depth wins depends on the grid (small grids
have fewer blocks than SMs, large ones are bandwidth-bound).  The pressure
wavefront's tile is 32 x 32 (one block per SM) or 32 x 16 (two per SM, more
tiles on small grids); the four-cell momentum sweep's block is one of
VEL_BLOCKS.  The tuner times every depth and tile on the case itself with CUDA
events (wf_time_kernel, cold L2) and keeps the fastest, cached as JSON keyed
by device and grid so a grid size is tuned once.  Results never depend on the
depth or tile; only speed does.  tune_batch picks the batched form's mode
(child graphs or persistent loops) and, for graphs, the chain width.
"""
from __future__ import annotations

import json
import os

from . import _lib

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "windfvm", "autotune.json")
PRES_DEPTHS = (1, 2, 3, 4)
PRES_ROWS = (32, 16)
VEL_DEPTHS = (1, 2)
VEL_BLOCKS = ((32, 4, 2), (32, 8, 1), (16, 8, 2), (64, 2, 2))


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


def tune_batch(batch, widths=(1, 2, 4, 0), steps: int = 2, modes=None) -> dict:
    """Picks the batched form's mode (_lib.BATCH_GRAPHS with a concurrency
    width, or _lib.BATCH_PERSISTENT) by timing `steps` batched steps per
    candidate; leaves the batch on the fastest.  The timed steps advance the
    cases."""
    modes = (_lib.BATCH_GRAPHS, _lib.BATCH_PERSISTENT) if modes is None else modes
    best = None
    times = {}
    for mode in modes:
        for w in (widths if mode == _lib.BATCH_GRAPHS else (None,)):
            batch.set_mode(mode)
            if w is not None:
                batch.set_width(w)
            batch.step(1)
            batch.prepare_graphs()  # no capture inside the timed steps
            batch.step(steps)
            ms = batch.last_step_ms() / steps
            key = "persistent" if mode == _lib.BATCH_PERSISTENT else w
            times[key] = ms
            if best is None or ms < times[best[0]]:
                best = (key, mode, w)
    batch.set_mode(best[1])
    if best[2] is not None:
        batch.set_width(best[2])
    batch.step(1)
    batch.prepare_graphs()
    return {"mode": "persistent" if best[1] == _lib.BATCH_PERSISTENT else "graphs",
            "width": best[2], "ms_per_step": times}


def tune(solver, cache_path: str | None = DEFAULT_CACHE, reps: int = 5, device_name: str | None = None) -> dict:
    """Picks and applies the fastest blocking depths and tile shapes for
    `solver`'s grid.  Returns {"pres_k", "pres_rows", "vel_k", "vel_block",
    "pres_us_per_sweep", "vel_us_per_sweep", "cached"}."""
    name = device_name or _device_name()
    key = _key(solver, name)
    cache = load_cache(cache_path) if cache_path else {}
    if key in cache and "pres_rows" in cache[key]:
        e = dict(cache[key])
        solver.set_blocking(e["pres_k"], e["vel_k"])
        solver.set_tiles(e["pres_rows"], tuple(e["vel_block"]))
        e["cached"] = True
        return e
    saved = solver.get_blocking()
    _, vblk0 = solver.get_tiles()
    best_p, best_v = None, None
    for rows in PRES_ROWS:
        solver.set_tiles(rows, vblk0)
        for k in PRES_DEPTHS:
            solver.set_blocking(k, saved[1])
            ms, _, sweeps = solver.time_kernel(_lib.KERNEL_PRES_SWEEP, reps=reps, flush_l2=True)
            us = ms * 1e3 / sweeps
            if best_p is None or us < best_p[2]:
                best_p = (k, rows, us)
    for k in VEL_DEPTHS:
        # the block shape applies to the one-sweep form only
        for blk in (VEL_BLOCKS if k == 1 else (vblk0,)):
            solver.set_tiles(best_p[1], blk)
            solver.set_blocking(best_p[0], k)
            ms, _, sweeps = solver.time_kernel(_lib.KERNEL_VEL_SWEEP, reps=reps, flush_l2=True)
            us = ms * 1e3 / sweeps
            if best_v is None or us < best_v[2]:
                best_v = (k, blk, us)
    solver.set_blocking(best_p[0], best_v[0])
    solver.set_tiles(best_p[1], best_v[1])
    e = {"pres_k": best_p[0], "pres_rows": best_p[1], "vel_k": best_v[0], "vel_block": list(best_v[1]),
         "pres_us_per_sweep": best_p[2], "vel_us_per_sweep": best_v[2]}
    if cache_path:
        cache[key] = e
        save_cache(cache_path, cache)
    return dict(e, cached=False)
