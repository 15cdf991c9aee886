"""Trajectory drift against the FP64 oracle after N steps (GPU tests).

Per-step parity bounds one step from a shared state; over many steps the
FP32 rounding of any implementation grows (LES on a central-difference
scheme amplifies it).  These tests run the CUDA library (FP32), the FP32
oracle (bit-identical to the reference's kernels step by step) and the FP64
oracle from the same set-up state for N steps and state the relative L2 of
velocity and pressure against FP64 after N steps:
  - plain_cube: 64 x 32(up) x 48 cells, the 100 steps of its workload;
  - urban_block: 256 x 96(up) x 192 cells, 20 steps (the bench's range).
The CUDA library may drift no further from FP64 than a bound set by the
reference arithmetic's own drift (the FP32 oracle against FP64 on the same
run): 4 x that plus 1e-5.  Each test prints one line with the figures.
"""
import json

import pytest

from unitywindsimulation_b200 import FvmSolverCuda, cases
from oracle import OracleSolver

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _drift(case, steps):
    g = FvmSolverCuda(case.cfg)
    o32 = OracleSolver(case.cfg, 32)
    o64 = OracleSolver(case.cfg, 64)
    for s in (g, o32, o64):
        cases.apply_case(s, case)
    for s in (g, o32, o64):
        s.Step(steps)
    g.check_finite()
    gu, gp = g.GetVelField(), g.GetPresField()
    u32, p32 = o32.GetVelField(), o32.GetPresField()
    u64, p64 = o64.GetVelField(), o64.GetPresField()
    out = {
        "workload": case.name, "cells": case.n_cells, "steps": steps,
        "gpu_vs_fp64": {"vel": rel_l2(gu, u64), "pres": rel_l2(gp, p64)},
        "oracle32_vs_fp64": {"vel": rel_l2(u32, u64), "pres": rel_l2(p32, p64)},
        "gpu_vs_oracle32": {"vel": rel_l2(gu, u32), "pres": rel_l2(gp, p32)},
    }
    print("DRIFT " + json.dumps(out))
    g.close()
    return out


@pytest.mark.parametrize("name,steps", [("plain_cube", 100), ("urban_block", 20)])
def test_drift_against_fp64_after_n_steps(built, name, steps):
    case = cases.WORKLOADS[name]()
    d = _drift(case, steps)
    for q in ("vel", "pres"):
        bound = 4.0 * d["oracle32_vs_fp64"][q] + 1e-5
        assert d["gpu_vs_fp64"][q] <= bound, (q, d)
