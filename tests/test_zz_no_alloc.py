"""The allocation-free residual entry point against the solver's own one.

wf_pres_residual_noalloc serves callers that cannot allocate device memory
(engine plugins whose GPU memory the host application owns, real-time loops
that cannot take cudaMalloc's device synchronisation).  It reduces
caller-owned device arrays with a fixed scratch array compiled into the
library.  This file runs last (pytest collects it after the others) so a
stop-at-first-failure run has executed everything else first; it also
passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases

from helpers import REL_TOL

pytestmark = pytest.mark.gpu


def _noalloc(lib, dp, pc, pcl, n):
    out = ctypes.c_float(-1.0)
    st = lib.wf_pres_residual_noalloc(dp, pc, pcl, n, None, ctypes.byref(out))
    return st, out.value


def test_noalloc_residual_matches_solver_entry_point(built):
    import torch

    lib = _lib.load()
    case = cases.small_case(nx=40, ny=20, nz=30, seed=31)
    g = FvmSolverCuda(case.cfg)
    g.InitFlags(case.flags)
    g.Step(2)
    g.op("vel_precompute")
    g.op("pres_precompute")
    seen = []
    for call in range(2):  # two calls in a row, on different data
        g.op("pres_sweeps", 3 + 2 * call)
        ref = g.op_residual("pres")  # wf_op_pres_residual: solver-owned scratch
        dp = g.get_field(_lib.FIELD_DP)
        pc = g.get_field(_lib.FIELD_PRES_CORRECT)
        pcl = g.get_field(_lib.FIELD_PRES_CORRECT_LAST_ITER)
        d_dp, d_pc, d_pcl = (torch.from_numpy(a).cuda() for a in (dp, pc, pcl))
        torch.cuda.synchronize()
        st, got = _noalloc(lib, d_dp.data_ptr(), d_pc.data_ptr(), d_pcl.data_ptr(), dp.size)
        assert st == _lib.WF_OK
        assert abs(got - ref) <= REL_TOL * abs(ref), (call, got, ref)
        host = float(np.sqrt(np.mean((dp.astype(np.float64) * (pc.astype(np.float64) - pcl)) ** 2)))
        assert abs(got - host) <= REL_TOL * abs(host), (call, got, host)
        seen.append(got)
    assert seen[0] != seen[1]


def test_noalloc_leaves_free_device_memory_unchanged(built):
    """After a first call (which may load the library's device code into the
    context), further calls take no device memory: the device's free memory
    is the same before and after them."""
    import torch

    lib = _lib.load()
    n = 1 << 20
    d_dp = torch.ones(n, device="cuda")
    d_pc = torch.full((n,), 2.0, device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(lib, d_dp.data_ptr(), d_pc.data_ptr(), None, n)[0] == _lib.WF_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        st, got = _noalloc(lib, d_dp.data_ptr(), d_pc.data_ptr(), None, n)
        assert st == _lib.WF_OK and got == pytest.approx(2.0, rel=REL_TOL)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_null_last_iterate_and_limits(built):
    import torch

    lib = _lib.load()
    n = 100_003
    rng = np.random.default_rng(0)
    dp = rng.standard_normal(n).astype(np.float32)
    pc = rng.standard_normal(n).astype(np.float32)
    d_dp, d_pc = torch.from_numpy(dp).cuda(), torch.from_numpy(pc).cuda()
    torch.cuda.synchronize()
    for _ in range(2):
        st, got = _noalloc(lib, d_dp.data_ptr(), d_pc.data_ptr(), None, n)
        assert st == _lib.WF_OK
        host = float(np.sqrt(np.mean((dp.astype(np.float64) * pc) ** 2)))
        assert abs(got - host) <= REL_TOL * host
    assert _noalloc(lib, d_dp.data_ptr(), d_pc.data_ptr(), None, 0)[0] == _lib.WF_ERR_INVALID_ARG
    too_big = _lib.NOALLOC_MAX_CELLS + 1
    assert _noalloc(lib, d_dp.data_ptr(), d_pc.data_ptr(), None, too_big)[0] == _lib.WF_ERR_INVALID_ARG
    assert _noalloc(lib, None, d_pc.data_ptr(), None, n)[0] == _lib.WF_ERR_INVALID_ARG
