"""The momentum sweep (and the adjoint's transposed sweep) run four
x-consecutive cells per thread with 128-bit loads when nx is a multiple of
4, else one cell per thread; WF_VEC4=0 forces the latter.  Both forms
compute every cell with the same arithmetic, so every field must agree bit
for bit, and a grid with nx not a multiple of 4 must still match the
oracle."""
import os

import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from oracle import OracleSolver

from helpers import REL_TOL, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES, _lib.FIELD_VEL_CORRECT, _lib.FIELD_VEL, _lib.FIELD_AODU,
          _lib.FIELD_D, _lib.FIELD_B, _lib.FIELD_DP, _lib.FIELD_BP, _lib.FIELD_PRES_CORRECT)


def _solver(case, vec4):
    old = os.environ.get("WF_VEC4")
    os.environ["WF_VEC4"] = "1" if vec4 else "0"
    try:
        s = FvmSolverCuda(case.cfg)
    finally:
        if old is None:
            del os.environ["WF_VEC4"]
        else:
            os.environ["WF_VEC4"] = old
    cases.apply_case(s, case)
    return s


@pytest.mark.parametrize("kw", [dict(piso=True, les=True, seed=0), dict(piso=False, les=False, seed=1, inflow_log=False),
                                dict(piso=True, les=True, seed=2, compat=_lib.COMPAT_PISO_CONSISTENT)],
                         ids=["piso_les", "simple_laminar", "piso_consistent"])
def test_vector_and_scalar_sweeps_bit_identical(built, kw):
    case = cases.small_case(nx=48, ny=20, nz=28, **kw)
    a, b = _solver(case, True), _solver(case, False)
    for s in (a, b):
        s.Step(3)
    for f in FIELDS:
        assert np.array_equal(a.get_field(f), b.get_field(f)), _lib.FIELD_NAMES[f]
    a.close()
    b.close()


def test_odd_nx_uses_scalar_sweep_and_matches_oracle(built):
    case = cases.small_case(nx=27, ny=14, nz=18, seed=3)
    g = FvmSolverCuda(case.cfg)
    o = OracleSolver(case.cfg, 32)
    for s in (g, o):
        cases.apply_case(s, case)
        s.Step(2)
    for f in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES):
        assert rel_l2(g.get_field(f), o.get_field(f)) <= REL_TOL, _lib.FIELD_NAMES[f]
    g.close()


def test_adjoint_gradient_same_in_both_forms(built):
    """The adjoint's recorded steps and its reversed momentum loop use the
    four-cell sweeps and accumulation passes too; J and the gradient agree
    with the one-cell forms up to the order of the atomic additions."""
    from unitywindsimulation_b200.adjoint import AdjointSolver, Objective
    case = cases.small_soft_case(seed=9)
    obj = Objective(x0=4, x1=20, z0=2, z1=14, y=1, window=2)
    out = []
    for vec4 in (True, False):
        g = _solver(case, vec4)
        with AdjointSolver(g) as adj:
            out.append(adj.gradient(obj, 4, 2, soft=case.soft))
        g.close()
    # J sums each step's objective with double-precision atomics
    assert out[0]["J"] == pytest.approx(out[1]["J"], rel=1e-12)
    assert out[0]["dJ_dustar"] == pytest.approx(out[1]["dJ_dustar"], rel=1e-5)
    assert out[0]["dJ_dz0"] == pytest.approx(out[1]["dJ_dz0"], rel=1e-5)
