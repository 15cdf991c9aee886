"""Pipelined stepping: wf_set_inflow_plane and wf_step_async return without
waiting for the GPU, so a host can upload step k+1's inlet and read step k's
fields while the GPU runs.  The fields must be exactly those of the blocking
calls, whatever the host does with its buffers in between."""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from unitywindsimulation_b200.solver import BatchSolver

pytestmark = pytest.mark.gpu


def _inlets(case, n, seed=0):
    rng = np.random.default_rng(seed)
    base = np.zeros((case.cfg.nz, case.cfg.ny, 3), np.float32)
    base[..., 0] = 2.0 + 0.1 * np.arange(case.cfg.ny, dtype=np.float32)[None, :]
    return [base * (1.0 + 0.05 * rng.standard_normal(base.shape).astype(np.float32)) for _ in range(n)]


def test_pipelined_loop_equals_blocking_loop(built):
    case = cases.small_case(nx=48, ny=24, nz=32, seed=3)
    planes = _inlets(case, 5)
    a, b = FvmSolverCuda(case.cfg), FvmSolverCuda(case.cfg)
    for s in (a, b):
        cases.apply_case(s, case)
        s.Step(2)
    n = case.n_cells
    # blocking reference
    ref = []
    for p in planes:
        a.set_inflow_plane(p)
        a.Step(1)
        u, pr, _ = a.get_state()
        ref.append((u.copy(), pr.copy()))
    # pipelined: one reusable host plane buffer, overwritten right after the
    # upload call returns; fields of step k arrive while step k+1 runs
    buf = np.empty_like(planes[0])
    vel = np.empty(3 * n, np.float32)
    pres = np.empty(n, np.float32)
    got = []
    for k, p in enumerate(planes):
        buf[...] = p
        b.set_inflow_plane(buf)
        buf[...] = -1.0e6  # the library must already hold its own copy
        b.step_async(1)
        if k > 0:
            b.readback_wait()
            got.append((vel.copy(), pres.copy()))
        b.readback_begin(vel, pres)
    b.readback_wait()
    got.append((vel.copy(), pres.copy()))
    for (u0, p0), (u1, p1) in zip(ref, got):
        assert np.array_equal(u0.reshape(-1), u1) and np.array_equal(p0.reshape(-1), p1)
    assert np.array_equal(a.get_field(_lib.FIELD_BND_X0), b.get_field(_lib.FIELD_BND_X0))
    a.close()
    b.close()


def test_batch_waits_for_queued_case_work(built):
    """An inflow upload and an asynchronous step still queued on a case's own
    stream are finished before a batched step touches the case."""
    cs = [cases.small_case(nx=32, ny=16, nz=24, seed=s) for s in (4, 5)]
    planes = [_inlets(c, 1, seed=9)[0] for c in cs]
    solo = [FvmSolverCuda(c.cfg) for c in cs]
    bat = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(solo + bat, cs + cs):
        cases.apply_case(s, c)
        s.Step(2)
    for s, p in zip(solo, planes):
        s.Step(1)
        s.set_inflow_plane(p)
        s.Step(2)
    for s, p in zip(bat, planes):
        s.step_async(1)
        s.set_inflow_plane(p)
    B = BatchSolver(bat)
    B.step(2)
    B.close()
    for s0, s1 in zip(solo, bat):
        assert np.array_equal(s0.get_field(_lib.FIELD_VEL_LAST_TIME), s1.get_field(_lib.FIELD_VEL_LAST_TIME))
        assert np.array_equal(s0.get_field(_lib.FIELD_PRES), s1.get_field(_lib.FIELD_PRES))
    for s in solo + bat:
        s.close()


def test_sync_and_async_zero_steps(built):
    case = cases.small_case(nx=24, ny=12, nz=16, seed=6)
    s = FvmSolverCuda(case.cfg)
    cases.apply_case(s, case)
    s.step_async(0)
    s.sync()
    s.step_async(2)
    s.sync()
    u1 = s.get_field(_lib.FIELD_VEL_LAST_TIME)
    t = FvmSolverCuda(case.cfg)
    cases.apply_case(t, case)
    t.Step(2)
    assert np.array_equal(u1, t.get_field(_lib.FIELD_VEL_LAST_TIME))
    with pytest.raises(Exception):
        s.step_async(-1)
    s.close()
    t.close()
