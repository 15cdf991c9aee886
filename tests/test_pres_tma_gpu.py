"""The four-sweep pressure pass stages its tiles with TMA loads (tensor-map
boxes completing on mbarriers) where nx is a multiple of 4; WF_TMA=0 selects
the kernel whose threads stage the planes themselves.  Both run the same
arithmetic in the same order on the same values, so every field must agree
bit for bit, including grids whose tiles overhang the domain, short z
extents and passes that also write iterate n-1.  The stage waits are
bounded: a wait that runs out is reported as WF_ERR_TIMEOUT and the handle
keeps working."""
import ctypes
import os

import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from oracle import OracleSolver

from helpers import ALL_FIELDS, REL_TOL, copy_state, rel_l2

pytestmark = pytest.mark.gpu


def _solver(cfg, tma):
    old = os.environ.get("WF_TMA")
    os.environ["WF_TMA"] = "1" if tma else "0"
    try:
        return FvmSolverCuda(cfg)
    finally:
        if old is None:
            del os.environ["WF_TMA"]
        else:
            os.environ["WF_TMA"] = old


SHAPES = [
    dict(nx=48, ny=20, nz=28, piso=True, les=True, seed=0),       # two tiles in x, one in y
    dict(nx=52, ny=30, nz=37, piso=False, les=True, seed=1),      # ragged tiles in x and y
    dict(nx=24, ny=12, nz=16, piso=True, les=False, seed=2),      # one tile larger than the domain
    dict(nx=100, ny=44, nz=9, piso=True, les=True, seed=3),       # z extent shorter than a chunk's halo
    dict(nx=28, ny=26, nz=61, piso=True, les=True, seed=4, inflow_log=False),
]


@pytest.mark.parametrize("kw", SHAPES, ids=lambda kw: "%dx%dx%d" % (kw["nx"], kw["ny"], kw["nz"]))
def test_tma_and_thread_staged_steps_bit_identical(built, kw):
    case = cases.small_case(**kw)
    a, b = _solver(case.cfg, True), _solver(case.cfg, False)
    for s in (a, b):
        cases.apply_case(s, case)
        s.Step(3)
    for f in ALL_FIELDS:
        assert np.array_equal(a.get_field(f), b.get_field(f)), _lib.FIELD_NAMES[f]
    a.close()
    b.close()


@pytest.mark.parametrize("n", [4, 5, 8, 11])
def test_tma_pass_iterates_n_and_n_minus_1(built, n):
    """Outside a step the last pass also writes iterate n-1
    (presCorrectFieldLastIter); both kernels and the FP32 oracle agree."""
    case = cases.small_case(nx=44, ny=28, nz=33, seed=7)
    o = OracleSolver(case.cfg, 32)
    o.InitFlags(case.flags)
    o.Step(2)
    o.op("vel_precompute"); o.op("vel_sweeps", 4); o.op("pres_precompute")
    got = []
    for tma in (True, False):
        g = _solver(case.cfg, tma)
        g.InitFlags(case.flags)
        copy_state(o, g)
        g.op("pres_sweeps", n)
        got.append([g.get_field(f) for f in (_lib.FIELD_PRES_CORRECT, _lib.FIELD_PRES_CORRECT_LAST_ITER)])
        g.close()
    o.op("pres_sweeps", n)
    for i, f in enumerate((_lib.FIELD_PRES_CORRECT, _lib.FIELD_PRES_CORRECT_LAST_ITER)):
        assert np.array_equal(got[0][i], got[1][i]), _lib.FIELD_NAMES[f]
        assert rel_l2(got[0][i], o.get_field(f)) <= REL_TOL, _lib.FIELD_NAMES[f]


def test_urban_block_step_bit_identical(built):
    """The benchmarked workload (256 x 96(up) x 192, nP = 40): one step from
    the set-up state by either kernel."""
    case = cases.WORKLOADS["urban_block"]()
    out = []
    for tma in (True, False):
        s = _solver(case.cfg, tma)
        cases.apply_case(s, case)
        s.Step(1)
        out.append((s.get_field(_lib.FIELD_PRES), s.get_field(_lib.FIELD_VEL_LAST_TIME),
                    s.get_field(_lib.FIELD_PRES_CORRECT)))
        s.close()
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_stage_wait_timeout_is_reported(built):
    lib = _lib.load()
    case = cases.small_case(nx=48, ny=20, nz=28, seed=5)
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    g.Step(1)
    st = ctypes.c_int(-1)
    # a stage that can never complete: the wait runs out, the pass returns
    assert lib.wf_stage_wait_selftest(g._h, 1, 20.0, ctypes.byref(st)) == _lib.WF_OK
    assert st.value == _lib.WF_ERR_TIMEOUT
    # the same pass with complete stages
    assert lib.wf_stage_wait_selftest(g._h, 0, 1000.0, ctypes.byref(st)) == _lib.WF_OK
    assert st.value == _lib.WF_OK
    # the handle keeps stepping and matches a handle that never timed out
    ref = FvmSolverCuda(case.cfg)
    cases.apply_case(ref, case)
    ref.Step(1)
    g.Step(2)
    ref.Step(2)
    for f in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES):
        assert np.array_equal(g.get_field(f), ref.get_field(f)), _lib.FIELD_NAMES[f]
    assert lib.wf_stage_wait_selftest(g._h, 0, 0.0, ctypes.byref(st)) == _lib.WF_ERR_INVALID_ARG
    g.close()
    ref.close()


def test_adjoint_same_with_both_pressure_kernels(built):
    """The adjoint's taped pressure loops (every iterate kept) and its
    reversed pressure loops run the TMA-staged pass too: the taped forward
    step is bit-identical, J agrees to its double-precision sums and the
    gradient to the order of the float atomics."""
    from unitywindsimulation_b200.adjoint import AdjointSolver, Objective
    case = cases.small_soft_case(nx=28, ny=14, nz=20, seed=9, np_=10)
    obj = Objective(x0=4, x1=24, z0=2, z1=18, y=1, window=2)
    fwd, grad = [], []
    for tma in (True, False):
        g = _solver(case.cfg, tma)
        cases.apply_case(g, case)
        with AdjointSolver(g) as adj:
            fwd.append(adj.step_forward())
            grad.append(adj.gradient(obj, 4, 2, soft=case.soft))
        g.close()
    for x, y in zip(fwd[0], fwd[1]):
        assert np.array_equal(x, y)
    assert grad[0]["J"] == pytest.approx(grad[1]["J"], rel=1e-12)
    assert grad[0]["dJ_dustar"] == pytest.approx(grad[1]["dJ_dustar"], rel=1e-5)
    assert grad[0]["dJ_dz0"] == pytest.approx(grad[1]["dJ_dz0"], rel=1e-5)
    a, b = np.asarray(grad[0]["dJ_dheights"]), np.asarray(grad[1]["dJ_dheights"])
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b) + 1e-12
