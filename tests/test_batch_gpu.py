"""Batched form and autotuner (GPU tests)."""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, autotune, cases
from unitywindsimulation_b200.solver import BatchSolver
from oracle import OracleSolver

from helpers import REL_TOL, rel_l2

pytestmark = pytest.mark.gpu


def _small_batch():
    return [cases.small_case(nx=24 + 8 * k, ny=12 + 2 * k, nz=16 + 4 * k, seed=40 + k, piso=(k % 2 == 0))
            for k in range(4)]


def test_batched_step_equals_individual_steps(built):
    """One graph launch per step for all cases gives exactly the fields of
    stepping every handle alone."""
    cs = _small_batch()
    alone = [FvmSolverCuda(c.cfg) for c in cs]
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(alone + batch, cs + cs):
        s.InitFlags(c.flags)
    for s in alone:
        s.Step(4)
    b = BatchSolver(batch)
    b.step(1)   # first step eager (fresh fields), then graph replays
    b.step(3)
    assert b.kernel_launches() > 0
    for a, s in zip(alone, batch):
        np.testing.assert_array_equal(a.GetVelField(), s.GetVelField())
        np.testing.assert_array_equal(a.GetPresField(), s.GetPresField())
        assert a.get_state()[2] == s.get_state()[2] == 4


@pytest.mark.parametrize("width", [1, 2, 0])
def test_batch_width_does_not_change_results(built, width):
    cs = _small_batch()
    alone = [FvmSolverCuda(c.cfg) for c in cs]
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(alone + batch, cs + cs):
        s.InitFlags(c.flags)
    for s in alone:
        s.Step(3)
    b = BatchSolver(batch)
    b.set_width(width)
    b.step(3)
    for a, s in zip(alone, batch):
        np.testing.assert_array_equal(a.GetVelField(), s.GetVelField())


def test_batch_prepare_graphs_keeps_results(built):
    cs = _small_batch()
    alone = [FvmSolverCuda(c.cfg) for c in cs]
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(alone + batch, cs + cs):
        s.InitFlags(c.flags)
    for s in alone:
        s.Step(6)
    b = BatchSolver(batch)
    b.step(1)
    b.prepare_graphs()  # captures only
    assert all(s.get_state()[2] == 1 for s in batch)
    b.step(5)
    for a, s in zip(alone, batch):
        np.testing.assert_array_equal(a.GetVelField(), s.GetVelField())
        np.testing.assert_array_equal(a.GetPresField(), s.GetPresField())


def test_batched_cases_match_oracle(built):
    cs = _small_batch()[:2]
    gs = [FvmSolverCuda(c.cfg) for c in cs]
    os_ = [OracleSolver(c.cfg, 32) for c in cs]
    for s, c in zip(gs + os_, cs + cs):
        s.InitFlags(c.flags)
    b = BatchSolver(gs)
    b.step(2)
    for o in os_:
        o.Step(2)
    for g, o in zip(gs, os_):
        assert rel_l2(g.GetVelField(), o.GetVelField()) <= 2 * REL_TOL
        assert rel_l2(g.GetPresField(), o.GetPresField()) <= 2 * REL_TOL


def test_batch_rejects_bad_input(built):
    c = cases.small_case(seed=50)
    s = FvmSolverCuda(c.cfg)
    with pytest.raises(_lib.WindFvmError):
        BatchSolver([s, s])
    with pytest.raises(_lib.WindFvmError):
        BatchSolver([])


def test_set_blocking_keeps_results(built):
    c = cases.small_case(nx=40, ny=20, nz=30, seed=51)
    outs = []
    for pk, vk in [(1, 1), (4, 2), (2, 1)]:
        s = FvmSolverCuda(c.cfg)
        s.set_blocking(pk, vk)
        assert s.get_blocking() == (pk, vk)
        s.InitFlags(c.flags)
        s.Step(3)
        outs.append(s.GetVelField())
    for o in outs[1:]:
        assert rel_l2(o, outs[0]) <= REL_TOL
    with pytest.raises(_lib.WindFvmError):
        s.set_blocking(5, 1)


def test_autotune_picks_and_caches(built, tmp_path):
    c = cases.small_case(nx=48, ny=24, nz=32, seed=52)
    s = FvmSolverCuda(c.cfg)
    s.InitFlags(c.flags)
    s.Step(1)
    path = str(tmp_path / "tune.json")
    first = autotune.tune(s, path, reps=2)
    assert not first["cached"]
    assert first["pres_k"] in autotune.PRES_DEPTHS and first["vel_k"] in autotune.VEL_DEPTHS
    assert s.get_blocking() == (first["pres_k"], first["vel_k"])
    s2 = FvmSolverCuda(c.cfg)
    again = autotune.tune(s2, path, reps=2)
    assert again["cached"] and (again["pres_k"], again["vel_k"]) == (first["pres_k"], first["vel_k"])
