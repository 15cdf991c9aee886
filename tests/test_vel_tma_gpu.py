"""Two momentum sweeps per pass with TMA-staged tiles (blocking depth 2,
`set_blocking(_, 2)`) against one sweep per launch (depth 1, the four-cell
sweep): the same arithmetic in the same order, so every field agrees bit for
bit, including tiles that overhang the domain, symmetry faces (where the
three components of 1/D differ), an odd sweep count (a one-sweep remainder
pass) and loops outside a step that also write iterate n-1."""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from oracle import OracleSolver

from helpers import ALL_FIELDS, REL_TOL, rel_l2

pytestmark = pytest.mark.gpu


def _pair(case, vel_k):
    s = FvmSolverCuda(case.cfg)
    cases.apply_case(s, case)
    s.set_blocking(4, vel_k)
    return s


SHAPES = [
    dict(nx=48, ny=20, nz=28, piso=True, les=True, seed=0),
    dict(nx=52, ny=30, nz=37, piso=False, les=True, seed=1, nv=7),    # odd sweep count
    dict(nx=24, ny=12, nz=16, piso=True, les=False, seed=2),          # one tile larger than the domain
    dict(nx=60, ny=34, nz=5, piso=True, les=True, seed=3),            # z extent shorter than a chunk
    dict(nx=28, ny=26, nz=61, piso=True, les=True, seed=4, inflow_log=False),
]


@pytest.mark.parametrize("kw", SHAPES, ids=lambda kw: "%dx%dx%d" % (kw["nx"], kw["ny"], kw["nz"]))
def test_two_sweep_passes_bit_identical(built, kw):
    case = cases.small_case(**kw)
    a, b = _pair(case, 2), _pair(case, 1)
    for s in (a, b):
        s.Step(3)
    for f in ALL_FIELDS:
        assert np.array_equal(a.get_field(f), b.get_field(f)), _lib.FIELD_NAMES[f]
    a.close()
    b.close()


def test_two_sweep_passes_with_x_and_y_symmetry_faces(built):
    """Symmetry faces normal to x (outlet) and y (ground and top) on top of
    the z ones: the pass derives the third component of 1/D from the first
    two in x- and y-symmetry cells and reads it from memory on z-symmetry
    planes and on the x-y edges; every field still agrees bit for bit."""
    case = cases.small_case(nx=40, ny=22, nz=26, seed=8, les=True)
    for f in (_lib.FACE_XN, _lib.FACE_Y0, _lib.FACE_YN):
        case.cfg.vel_bc[f] = _lib.BND_SYMMETRY
    a, b = _pair(case, 2), _pair(case, 1)
    for s in (a, b):
        s.Step(3)
    for f in ALL_FIELDS:
        assert np.array_equal(a.get_field(f), b.get_field(f)), _lib.FIELD_NAMES[f]
    a.close()
    b.close()


@pytest.mark.parametrize("n", [1, 2, 3, 6])
def test_two_sweep_loop_iterates_n_and_n_minus_1(built, n):
    """A loop outside a step, started right after a step (velFieldLastIter
    then aliases velFieldLastTime): velField holds iterate n and
    velFieldLastIter iterate n-1 (iterate 0 = velFieldLastTime for n = 1),
    in both forms and in the FP32 oracle."""
    case = cases.small_case(nx=44, ny=28, nz=33, seed=7)
    fields = (_lib.FIELD_VEL, _lib.FIELD_VEL_LAST_ITER)
    out = []
    for k in (2, 1):
        s = _pair(case, k)
        s.Step(2)
        s.op("vel_precompute")
        s.op("vel_sweeps", n)
        out.append([s.get_field(f) for f in fields])
        s.close()
    o = OracleSolver(case.cfg, 32)
    cases.apply_case(o, case)
    o.Step(2)
    o.op("vel_precompute")
    o.op("vel_sweeps", n)
    for i, f in enumerate(fields):
        assert np.array_equal(out[0][i], out[1][i]), _lib.FIELD_NAMES[f]
        assert rel_l2(out[0][i], o.get_field(f)) <= REL_TOL, _lib.FIELD_NAMES[f]


def test_urban_block_two_sweep_passes_bit_identical(built):
    case = cases.WORKLOADS["urban_block"]()
    out = []
    for k in (2, 1):
        s = _pair(case, k)
        s.Step(1)
        out.append([s.get_field(f) for f in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES, _lib.FIELD_VEL)])
        s.close()
    for x, y in zip(*out):
        assert np.array_equal(x, y)
