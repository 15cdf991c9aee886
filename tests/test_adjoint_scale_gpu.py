"""The adjoint gradient on the full adjoint workload (GPU test).

tests/golden/adjoint_street_fd.npz holds FP64 central differences (step
1e-4) of the objective on the whole workload (128 x 64(up) x 96 cells, 12
soft buildings, PISO laminar, 200-step window, objective over the last 100
steps; tests/golden/make_adjoint_fd.py).  The CUDA adjoint, run as the
benchmark runs it (checkpoints every 20 steps, tapes of the last steps kept
from the forward pass), must give J within 1e-4 of the FP64 oracle's J and
dJ/du*, dJ/dz0 and the three height derivatives within 1e-3 relative.
"""
import os

import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, cases
from unitywindsimulation_b200.adjoint import AdjointSolver, Objective

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "adjoint_street_fd.npz")
ADJ_TOL = 1e-3


def test_adjoint_street_gradient_vs_fp64_fd(built):
    fd = np.load(FIXTURE)
    case = cases.adjoint_street()
    obj = Objective(**cases.ADJOINT_STREET_OBJECTIVE)
    assert int(fd["steps"]) == case.steps and int(fd["window"]) == obj.window
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    with AdjointSolver(g) as adj:
        r = adj.gradient(obj, case.steps, cases.ADJOINT_STREET_CHECKPOINT, soft=case.soft)
    g.close()
    J0 = float(fd["J"])
    print(f"ADJSCALE J {r['J']:.9g} vs {J0:.9g}; u* {r['dJ_dustar']:.7g} vs {float(fd['dJ_dustar']):.7g}; "
          f"z0 {r['dJ_dz0']:.7g} vs {float(fd['dJ_dz0']):.7g}; heights "
          + ", ".join(f"{r['dJ_dheights'][i]:.7g} vs {v:.7g}" for i, v in zip(fd["heights"], fd["dJ_dheights"])))
    assert abs(r["J"] - J0) <= 1e-4 * abs(J0)
    assert abs(r["dJ_dustar"] - float(fd["dJ_dustar"])) <= ADJ_TOL * abs(float(fd["dJ_dustar"]))
    assert abs(r["dJ_dz0"] - float(fd["dJ_dz0"])) <= ADJ_TOL * abs(float(fd["dJ_dz0"]))
    for i, v in zip(fd["heights"], fd["dJ_dheights"]):
        assert abs(r["dJ_dheights"][int(i)] - v) <= ADJ_TOL * abs(v), (int(i), r["dJ_dheights"][int(i)], v)
