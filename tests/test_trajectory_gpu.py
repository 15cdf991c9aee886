"""The urban block's long trajectory against the reference arithmetic (GPU).

The bench workload (256 x 96(up) x 192, PISO + LES, CFL 0.5) leaves the
bounded range after about 150 steps.  tests/golden/urban_block_trajectory.npz
holds the FP32 oracle's run from the same set-up state (bit-identical to the
reference's kernels step by step; tests/golden/make_trajectory.py), with
max|u|, mean kinetic energy and max|p| over the fluid cells after every step,
up to the step where max|u| passes 20 x its initial value.  The CUDA library
must blow up at the same step and follow the same statistics until then: the
divergence is the reference scheme's, not the GPU path's.
"""
import os

import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, cases
from oracle.trajectory import step_stats

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "urban_block_trajectory.npz")


def test_urban_block_blows_up_where_the_reference_does(built):
    ref = np.load(FIXTURE)
    rows, u0_ref, blowup = ref["rows"], float(ref["u0"]), float(ref["blowup"])
    assert str(ref["status"]) == "blowup"
    n_ref = len(rows)
    case = cases.urban_block()
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    fluid = np.asarray(case.flags).reshape(-1) == 0
    u0 = step_stats(g.GetVelField(), g.GetPresField(), fluid)[0]
    assert u0 == pytest.approx(u0_ref, rel=1e-6)
    got = []
    for k in range(n_ref + 5):
        g.Step(1)
        st = step_stats(g.GetVelField(), g.GetPresField(), fluid)
        got.append(st)
        if not np.all(np.isfinite(st)) or st[0] > blowup * u0:
            break
    g.close()
    got = np.array(got)
    assert len(got) == n_ref, f"GPU left the bounded range after {len(got)} steps, the reference after {n_ref}"
    # the statistics agree step by step until the last few steps before the
    # blow-up, where the growing mode amplifies FP32 rounding
    rel = np.abs(got - rows) / np.abs(rows)
    bounded = n_ref - 10
    assert rel[:bounded, 0].max() <= 1e-5, rel[:bounded, 0].max()   # max |u|
    assert rel[:bounded, 1].max() <= 1e-6, rel[:bounded, 1].max()   # mean kinetic energy
    assert rel[:bounded, 2].max() <= 1e-5, rel[:bounded, 2].max()   # max |p|
