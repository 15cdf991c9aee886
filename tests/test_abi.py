"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, validates its inputs and reports failures by status code."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from unitywindsimulation_b200 import _lib
from unitywindsimulation_b200.config import default_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "windfvm.h")


def declared_functions(header=HEADER):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wf_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["wf_create", "wf_destroy", "wf_step", "wf_init_flags", "wf_init_vel_pres_fields",
                 "wf_set_fixed_value_vel_bnd_cond", "wf_get_vel", "wf_get_pres", "wf_get_flags",
                 "wf_get_state", "wf_set_state", "wf_residuals", "wf_last_error", "wf_strerror", "wf_version"]:
        assert must in names


def test_library_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(wf_[a-z0-9_]+)\b", out))
    assert set(declared_functions()) <= exported


def test_binding_covers_the_header(built):
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_config_struct_matches_c(built):
    lib = _lib.load()
    c = _lib.WfConfig()
    lib.wf_config_default(ctypes.byref(c))
    assert c.struct_size == ctypes.sizeof(_lib.WfConfig)
    assert bytes(c) == bytes(default_config())


def test_version_and_strerror(built):
    lib = _lib.load()
    assert lib.wf_version() == 1
    assert lib.wf_strerror(_lib.WF_ERR_NONFINITE) == b"non-finite value in the solution"
    assert lib.wf_strerror(12345) == b"unknown status"


def _create(cfg, device=0):
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.wf_create(ctypes.byref(cfg), device, ctypes.byref(h))
    if st == _lib.WF_OK:
        lib.wf_destroy(h)
    return st


@pytest.mark.parametrize("bad", [
    dict(nx=2), dict(ny=0), dict(dx=0.0), dict(dt=-1.0), dict(den=0.0),
    dict(vel_bc=[0, 1, 0, 2, 2, 7]), dict(solver_type=5), dict(turbulence=3), dict(inflow_type=9),
    dict(vel_iters=-1), dict(compat_flags=0x80),
])
def test_invalid_config_rejected_before_touching_the_device(built, bad):
    assert _create(default_config(**bad)) == _lib.WF_ERR_INVALID_ARG


def test_struct_size_checked(built):
    cfg = default_config()
    cfg.struct_size = 4
    assert _create(cfg) == _lib.WF_ERR_INVALID_ARG


def test_null_arguments(built):
    lib = _lib.load()
    assert lib.wf_create(None, 0, None) == _lib.WF_ERR_INVALID_ARG
    assert lib.wf_step(None, 1, None) == _lib.WF_ERR_INVALID_ARG
    assert lib.wf_destroy(None) == _lib.WF_ERR_INVALID_ARG
    assert lib.wf_get_vel(None, None, 0) == _lib.WF_ERR_INVALID_ARG


def test_fault_injection_oom(built, monkeypatch):
    """Allocation failure forced on the host: wf_create reports WF_ERR_OOM and
    returns no handle."""
    monkeypatch.setenv("WF_FAULT_INJECT", "oom")
    lib = _lib.load()
    h = ctypes.c_void_p(1234)
    st = lib.wf_create(ctypes.byref(default_config(nx=8, ny=8, nz=8)), 0, ctypes.byref(h))
    assert st == _lib.WF_ERR_OOM
    assert not h.value


def test_no_device_is_an_error_not_a_crash(built):
    """On a machine without a GPU wf_create fails with a status code."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert _create(default_config(nx=8, ny=8, nz=8)) == _lib.WF_ERR_CUDA
    with pytest.raises(_lib.WindFvmError):
        from unitywindsimulation_b200 import FvmSolverCuda
        FvmSolverCuda(default_config(nx=8, ny=8, nz=8))


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setenv("WINDFVM_LIB", str(tmp_path / "nope.so"))
    with pytest.raises(_lib.WindFvmError):
        _lib.load(str(tmp_path / "nope.so"))


@pytest.mark.timeout(60)
def test_tensor_map_probe_returns(built):
    """The TMA-staged passes ask whether the driver's tensor-map encoder is
    present before every launch; the probe must answer (False on a machine
    without a CUDA driver) rather than spin."""
    lib = ctypes.CDLL(_lib.LIB_PATH)
    probe = lib._ZN2wf13tma_availableEv
    probe.restype = ctypes.c_bool
    assert probe() in (True, False)
