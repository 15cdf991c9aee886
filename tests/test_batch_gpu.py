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
    assert first["pres_rows"] in autotune.PRES_ROWS and tuple(first["vel_block"]) in autotune.VEL_BLOCKS
    assert s.get_blocking() == (first["pres_k"], first["vel_k"])
    assert s.get_tiles() == (first["pres_rows"], tuple(first["vel_block"]))
    s2 = FvmSolverCuda(c.cfg)
    again = autotune.tune(s2, path, reps=2)
    assert again["cached"] and (again["pres_k"], again["vel_k"]) == (first["pres_k"], first["vel_k"])
    assert s2.get_tiles() == s.get_tiles()


def test_tune_batch_picks_a_mode(built):
    cs = _persistent_batch()
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(batch, cs):
        s.InitFlags(c.flags)
    b = BatchSolver(batch)
    r = autotune.tune_batch(b, widths=(0, 1), steps=1)
    assert r["mode"] in ("graphs", "persistent") and set(r["ms_per_step"]) == {0, 1, "persistent"}
    assert b.get_mode() == (_lib.BATCH_PERSISTENT if r["mode"] == "persistent" else _lib.BATCH_GRAPHS)
    b.step(2)


def _persistent_batch():
    """Uneven PISO + LES grids (one with nx % 4 != 0: the one-cell momentum
    sweep) with the same step structure, as the persistent mode needs."""
    dims = [(24, 12, 16), (32, 14, 20), (42, 16, 24), (48, 18, 28)]
    return [cases.small_case(nx=nx, ny=ny, nz=nz, seed=60 + k, piso=True)
            for k, (nx, ny, nz) in enumerate(dims)]


@pytest.mark.parametrize("pres_k", [4, 3])
def test_persistent_batch_equals_individual_steps(built, pres_k):
    """One persistent launch per Jacobi loop over all cases (grid barrier
    between sweeps) gives exactly the fields of stepping every handle alone."""
    cs = _persistent_batch()
    alone = [FvmSolverCuda(c.cfg) for c in cs]
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(alone + batch, cs + cs):
        s.InitFlags(c.flags)
        s.set_blocking(pres_k, 1)
    for s in alone:
        s.Step(5)
    b = BatchSolver(batch)
    b.set_mode(_lib.BATCH_PERSISTENT)
    assert b.get_mode() == _lib.BATCH_PERSISTENT
    b.step(1)   # first step eager, then recorded segments + persistent loops
    l0 = b.kernel_launches()
    b.step(4)
    # 4 persistent loop launches per step plus the cases' once-per-step kernels
    assert 0 < b.kernel_launches() - l0 < 4 * 80 * len(cs)
    for a, s in zip(alone, batch):
        np.testing.assert_array_equal(a.GetVelField(), s.GetVelField())
        np.testing.assert_array_equal(a.GetPresField(), s.GetPresField())
        assert a.get_state()[2] == s.get_state()[2] == 5
    b.prepare_graphs()
    b.step(2)
    for s in alone:
        s.Step(2)
    for a, s in zip(alone, batch):
        np.testing.assert_array_equal(a.GetVelField(), s.GetVelField())


def test_persistent_batch_rejects_mixed_step_structures(built):
    cs = _small_batch()  # PISO and SIMPLE cases
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(batch, cs):
        s.InitFlags(c.flags)
    b = BatchSolver(batch)
    b.set_mode(_lib.BATCH_PERSISTENT)
    with pytest.raises(_lib.WindFvmError) as e:
        b.step(2)
    assert e.value.status == _lib.WF_ERR_UNSUPPORTED


def test_grid_barrier_releases_and_times_out(built):
    """The bounded grid barrier of the persistent loops: released when every
    block arrives; with arrivals that never come its wait runs out after the
    limit, every block returns and the status says so; the device stays
    usable."""
    import ctypes
    import time
    lib = _lib.load()
    st = ctypes.c_int(-1)
    assert lib.wf_grid_barrier_selftest(0, 16, 0, 1000.0, ctypes.byref(st)) == _lib.WF_OK
    assert st.value == _lib.WF_OK
    t0 = time.perf_counter()
    assert lib.wf_grid_barrier_selftest(0, 16, 1, 50.0, ctypes.byref(st)) == _lib.WF_OK
    assert st.value == _lib.WF_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    assert lib.wf_grid_barrier_selftest(0, 16, 0, 1000.0, ctypes.byref(st)) == _lib.WF_OK
    assert st.value == _lib.WF_OK
    assert lib.wf_grid_barrier_selftest(0, 100000, 0, 10.0, ctypes.byref(st)) == _lib.WF_ERR_INVALID_ARG


def test_persistent_batch_step_reports_barrier_timeout(built):
    """A barrier limit far below one sweep's time makes the waits run out:
    wf_batch_step returns WF_ERR_TIMEOUT instead of hanging, and the batch
    runs again with a normal limit."""
    cs = _persistent_batch()[:2]
    batch = [FvmSolverCuda(c.cfg) for c in cs]
    for s, c in zip(batch, cs):
        s.InitFlags(c.flags)
    b = BatchSolver(batch)
    b.set_mode(_lib.BATCH_PERSISTENT)
    b.step(1)
    b.set_barrier_timeout(1e-6)  # one nanosecond
    with pytest.raises(_lib.WindFvmError) as e:
        b.step(1)
    assert e.value.status == _lib.WF_ERR_TIMEOUT
    b.set_barrier_timeout(2000.0)
    b.step(1)
    with pytest.raises(_lib.WindFvmError):
        b.set_barrier_timeout(0.0)


@pytest.mark.parametrize("tiles", [(16, (32, 4, 2)), (32, (32, 8, 1)), (16, (16, 8, 2)), (32, (64, 2, 2))])
def test_tiles_do_not_change_results(built, tiles):
    c = cases.small_case(nx=48, ny=36, nz=30, seed=53)
    ref = FvmSolverCuda(c.cfg)
    s = FvmSolverCuda(c.cfg)
    s.set_tiles(tiles[0], tiles[1])
    assert s.get_tiles() == (tiles[0], tuple(tiles[1]))
    for x in (ref, s):
        x.InitFlags(c.flags)
        x.Step(3)
    np.testing.assert_array_equal(ref.GetVelField(), s.GetVelField())
    np.testing.assert_array_equal(ref.GetPresField(), s.GetPresField())
    with pytest.raises(_lib.WindFvmError):
        s.set_tiles(24, (32, 4, 2))
    with pytest.raises(_lib.WindFvmError):
        s.set_tiles(32, (32, 4, 1))
