"""Golden fixtures (tests/golden/, made by make_golden.py with the FP64
oracle): the reference's AIJ validation case on its OpenFOAM sample lines and
a small PISO + LES case with full fields."""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

from helpers import rel_l2  # noqa: E402


def _load():
    with open(os.path.join(HERE, "golden", "aij_building.json")) as f:
        aij = json.load(f)
    small = np.load(os.path.join(HERE, "golden", "small_piso.npz"))
    return aij, small


AIJ_CELLS = 80 * 40 * 40


def _compare_aij(got, ref, tol):
    """Sample-line error relative to the larger of the line's norm and the
    field's RMS over as many points (pressure is near 0 close to the p = 0
    outlet, where a plain relative norm is ill-conditioned)."""
    for k, v in ref.items():
        if k == "norms":
            for kk, vv in v.items():
                assert abs(got[k][kk] - vv) <= tol * abs(vv), (k, kk)
            continue
        for f in ("u", "p"):
            a = np.asarray(got[k][f], dtype=np.float64)
            b = np.asarray(v[f], dtype=np.float64)
            if k == "plane_sums":
                e = rel_l2(a, b)
            else:
                rms = ref["norms"][f + "_l2"] / np.sqrt(AIJ_CELLS * (3 if f == "u" else 1))
                e = np.linalg.norm(a - b) / max(np.linalg.norm(b), rms * np.sqrt(b.size))
            assert e <= tol, (k, f, e)


def test_oracle_fp64_reproduces_golden(built):
    from oracle import OracleSolver
    aij, small = _load()
    _compare_aij(make_golden.run_aij(OracleSolver, precision=64), aij, 1e-9)
    u, p = make_golden.run_small(OracleSolver, precision=64)
    assert rel_l2(u, small["u"]) <= 1e-7 and rel_l2(p, small["p"]) <= 1e-7


def test_oracle_fp32_near_golden(built):
    from oracle import OracleSolver
    aij, small = _load()
    _compare_aij(make_golden.run_aij(OracleSolver, precision=32), aij, 2e-5)
    u, p = make_golden.run_small(OracleSolver, precision=32)
    assert rel_l2(u, small["u"]) <= 2e-5 and rel_l2(p, small["p"]) <= 2e-5


@pytest.mark.gpu
def test_cuda_matches_golden(built):
    """The CUDA FP32 path against the FP64 golden fields: within 2 steps x
    1e-5 relative L2 (FP32 rounding of the FP64 result included)."""
    from unitywindsimulation_b200 import FvmSolverCuda
    aij, small = _load()
    _compare_aij(make_golden.run_aij(FvmSolverCuda), aij, 2e-5)
    u, p = make_golden.run_small(FvmSolverCuda)
    assert rel_l2(u, small["u"]) <= 2e-5 and rel_l2(p, small["p"]) <= 2e-5
