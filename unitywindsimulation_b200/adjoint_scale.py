"""Adjoint at scale: the objective's gradient for every wind direction of
the adjoint_batch workload (8 directions x 256 x 96(up) x 256 cells, 64 soft
buildings, 400-step window, checkpoints every 25), one direction after
another on one GPU, each against its own plain forward.

    python -m unitywindsimulation_b200.adjoint_scale [--directions 8] [--steps 400]

Prints one JSON line per direction and a summary line.  The directions run
one after another: one direction's step tapes already fill most of the
device memory, and one 6.3 M-cell case fills the GPU's bandwidth by itself.
"""
from __future__ import annotations

import argparse
import json
import time

from . import cases
from .adjoint import AdjointSolver, Objective
from .solver import FvmSolverCuda


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--directions", type=int, default=8)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--checkpoint", type=int, default=cases.ADJOINT_BATCH_CHECKPOINT)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    cs = cases.adjoint_batch(n_dirs=a.directions, steps=a.steps)
    ob = dict(cases.ADJOINT_BATCH_OBJECTIVE)
    ob["window"] = min(ob["window"], max(1, a.steps // 2))
    obj = Objective(**ob)
    tot_fwd = tot_adj = 0.0
    for c in cs:
        g = FvmSolverCuda(c.cfg, device=a.device)
        cases.apply_case(g, c)
        g.Step(3)
        g.prepare_graphs()
        g.Step(a.steps)
        fwd = g.last_step_ms()
        g.close()
        g = FvmSolverCuda(c.cfg, device=a.device)
        cases.apply_case(g, c)
        t0 = time.perf_counter()
        with AdjointSolver(g) as adj:
            r = adj.gradient(obj, a.steps, a.checkpoint, soft=c.soft)
        wall = time.perf_counter() - t0
        g.close()
        tot_fwd += fwd
        tot_adj += r["ms_total"]
        print(json.dumps({"case": c.name, "cells": c.n_cells, "steps": a.steps, "forward_ms": fwd,
                          "gradient_ms": r["ms_total"], "adjoint_over_forward": r["ms_total"] / fwd,
                          "wall_s": wall, "J": r["J"], "dJ_dustar": r["dJ_dustar"], "dJ_dz0": r["dJ_dz0"],
                          "dJ_dheights": [float(x) for x in r["dJ_dheights"]]}), flush=True)
    print(json.dumps({"summary": "adjoint_batch", "directions": len(cs), "forward_ms_total": tot_fwd,
                      "gradient_ms_total": tot_adj, "adjoint_over_forward": tot_adj / tot_fwd}), flush=True)


if __name__ == "__main__":
    main()
