"""Runs a workload for a few steps and times its two Jacobi kernels.

    python -m unitywindsimulation_b200.profile_kernels [--workload urban_block] [--steps 2]

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
    a = ap.parse_args(argv)
    case = cases.WORKLOADS[a.workload]()
    s = FvmSolverCuda(case.cfg)
    cases.apply_case(s, case)
    s.Step(a.steps)
    out = {"workload": a.workload, "cells": case.n_cells, "step_ms": s.last_step_ms() / max(a.steps, 1)}
    for name, k in (("pres_sweep", _lib.KERNEL_PRES_SWEEP), ("vel_sweep", _lib.KERNEL_VEL_SWEEP)):
        ms, by, sw = s.time_kernel(k, reps=a.reps, flush_l2=True)
        out[name] = {"ms_per_launch": ms, "sweeps_per_launch": sw, "alg_gbs": by / (ms / 1e3) / 1e9}
    print(json.dumps(out))
    s.close()


if __name__ == "__main__":
    main()
