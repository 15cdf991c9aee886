"""Runs a workload for a few steps and times its two Jacobi kernels.

    python -m unitywindsimulation_b200.profile_kernels [--workload urban_block] [--steps 2]
    python -m unitywindsimulation_b200.profile_kernels --workload adjoint_street --steps 2 --adjoint

Meant as the target program of an ncu capture (`ncu -k regex:<kernel> ...`)
and as a quick check of the per-sweep kernel times (CUDA events, cold L2).
"""
from __future__ import annotations

import argparse
import json

from . import _lib, cases
from .solver import FvmSolverCuda


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="urban_block", choices=sorted(cases.WORKLOADS))
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--adjoint", action="store_true",
                    help="also run the objective gradient over --steps steps (turbulence-off workloads)")
    a = ap.parse_args(argv)
    case = cases.WORKLOADS[a.workload]()
    s = FvmSolverCuda(case.cfg)
    cases.apply_case(s, case)
    s.Step(a.steps)
    out = {"workload": a.workload, "cells": case.n_cells, "step_ms": s.last_step_ms() / max(a.steps, 1)}
    if case.faces is None:  # the uniform grid's two Jacobi kernels
        for name, k in (("pres_sweep", _lib.KERNEL_PRES_SWEEP), ("vel_sweep", _lib.KERNEL_VEL_SWEEP)):
            ms, by, sw = s.time_kernel(k, reps=a.reps, flush_l2=True)
            out[name] = {"ms_per_launch": ms, "sweeps_per_launch": sw, "alg_gbs": by / (ms / 1e3) / 1e9}
    s.close()
    if a.adjoint:
        from .adjoint import AdjointSolver, Objective
        s = FvmSolverCuda(case.cfg)
        cases.apply_case(s, case)
        nx, nz = case.cfg.nx, case.cfg.nz
        obj = Objective(x0=nx // 4, x1=3 * nx // 4, z0=nz // 4, z1=3 * nz // 4, y=min(3, case.cfg.ny - 1), window=1)
        with AdjointSolver(s) as adj:
            r = adj.gradient(obj, a.steps, a.steps, soft=case.soft)
        out["adjoint"] = {"gradient_ms": r["ms_total"], "forward_pass_ms": r["ms_forward"], "J": r["J"]}
        s.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
