"""ctypes binding of the windfvm C ABI (include/windfvm.h).

The shared library ``libwindfvm.so`` is built in-tree (``build.py``) and is the
only compute path: there is no CPU fallback.  Importing this module does not
need a GPU; creating a solver does, and fails with ``WindFvmError`` when the
library or the device is missing.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_uint32, c_void_p

LIB_NAME = "libwindfvm.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

# ---- status codes (windfvm.h) ----
WF_OK = 0
WF_ERR_INVALID_ARG = 1
WF_ERR_CUDA = 2
WF_ERR_OOM = 3
WF_ERR_NONFINITE = 4
WF_ERR_TIMEOUT = 5
WF_ERR_UNSUPPORTED = 6
WF_NOT_FINISHED = 7
WF_ERR_STATE = 8
WF_ERR_IO = 9

# batch modes (wf_batch_set_mode)
BATCH_GRAPHS = 0
BATCH_PERSISTENT = 1

# ---- enums ----
CELL_FLUID, CELL_SOLID = 0, 1
BND_FIXED_VALUE, BND_ZERO_GRAD, BND_SYMMETRY = 0, 1, 2
FACE_X0, FACE_XN, FACE_Y0, FACE_YN, FACE_Z0, FACE_ZN = range(6)
SOLVER_SIMPLE, SOLVER_PISO = 0, 1
TURB_NONE, TURB_SMAGORINSKY = 0, 1
INFLOW_CONSTANT, INFLOW_LOG = 0, 1
COMPAT_RFLOAT_FACE_EDDY_VIS = 0x1
COMPAT_INIT_PROFILE_CELL_CENTRE = 0x2
COMPAT_PISO_CONSISTENT = 0x4
LAYOUT_SOA, LAYOUT_XYZW, LAYOUT_XYZ = 0, 1, 2

FIELD_VEL = 0
FIELD_VEL_LAST_TIME = 1
FIELD_VEL_LAST_ITER = 2
FIELD_VEL_CORRECT = 3
FIELD_PRES = 4
FIELD_PRES_CORRECT = 5
FIELD_PRES_CORRECT_LAST_ITER = 6
FIELD_D = 7
FIELD_B = 8
FIELD_DP = 9
FIELD_BP = 10
FIELD_AODU = 11
FIELD_EDDY_VIS = 12
FIELD_FACE_EDDY_VIS = 13
FIELD_BND_X0 = 14
FIELD_BND_XN = 15
FIELD_BND_Y0 = 16
FIELD_BND_YN = 17
FIELD_BND_Z0 = 18
FIELD_BND_ZN = 19
FIELD_DRAG = 20
FIELD_COUNT = 21

FIELD_NAMES = {
    FIELD_VEL: "velField", FIELD_VEL_LAST_TIME: "velFieldLastTime", FIELD_VEL_LAST_ITER: "velFieldLastIter",
    FIELD_VEL_CORRECT: "velCorrectField", FIELD_PRES: "presFieldLastTime", FIELD_PRES_CORRECT: "presCorrectField",
    FIELD_PRES_CORRECT_LAST_ITER: "presCorrectFieldLastIter", FIELD_D: "DField", FIELD_B: "bField",
    FIELD_DP: "DFieldPresCorrect", FIELD_BP: "bFieldPresCorrect", FIELD_AODU: "AodUCorrectField",
    FIELD_EDDY_VIS: "eddyVisField", FIELD_FACE_EDDY_VIS: "faceEddyVisField", FIELD_BND_X0: "bndFieldX0",
    FIELD_BND_XN: "bndFieldXn", FIELD_BND_Y0: "bndFieldY0", FIELD_BND_YN: "bndFieldYn", FIELD_BND_Z0: "bndFieldZ0",
    FIELD_BND_ZN: "bndFieldZn", FIELD_DRAG: "dragField",
}


class WfConfig(ctypes.Structure):
    """Mirror of ``wf_config`` (FluidSimConfig + RuntimeConfig fields)."""

    _fields_ = [
        ("struct_size", c_uint32),
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("dx", c_float), ("dt", c_float), ("mu", c_float), ("den", c_float),
        ("ext_force", c_float * 3),
        ("vel_bc", c_int32 * 6), ("pres_bc", c_int32 * 6),
        ("solver_type", c_int32), ("piso_correctors", c_int32),
        ("turbulence", c_int32), ("cs", c_float),
        ("vel_iters", c_int32), ("pres_iters", c_int32),
        ("inflow_type", c_int32),
        ("wind_speed", c_float), ("inflow_ustar", c_float), ("inflow_z0", c_float),
        ("inflow_kappa", c_float), ("inflow_href", c_float),
        ("vel_zn", c_float * 3),
        ("calc_residual", c_int32), ("vel_res_interval", c_int32), ("pres_res_interval", c_int32),
        ("vel_tol", c_float), ("pres_tol", c_float),
        ("compat_flags", c_uint32),
        ("check_finite", c_int32),
        ("use_graph", c_int32),
    ]

    def copy(self) -> "WfConfig":
        c = WfConfig()
        ctypes.pointer(c)[0] = self
        return c

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class WfDeviceFields(ctypes.Structure):
    _fields_ = [("vel", c_void_p * 3), ("pres", c_void_p), ("flags", c_void_p), ("n_cells", c_int64),
                ("stream", c_void_p)]


class WfObjective(ctypes.Structure):
    _fields_ = [("x0", c_int32), ("x1", c_int32), ("z0", c_int32), ("z1", c_int32), ("y", c_int32),
                ("window", c_int32)]


class WindFvmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"windfvm status {status}: {message}")
        self.status = status


# name -> (restype, argtypes)
_SIGNATURES = {
    "wf_config_default": (None, [POINTER(WfConfig)]),
    "wf_create": (c_int, [POINTER(WfConfig), c_int, POINTER(c_void_p)]),
    "wf_destroy": (c_int, [c_void_p]),
    "wf_init_flags": (c_int, [c_void_p, POINTER(c_int32), c_size_t]),
    "wf_init_vel_pres_fields": (c_int, [c_void_p]),
    "wf_set_fixed_value_vel_bnd_cond": (c_int, [c_void_p, c_float]),
    "wf_change_phys_field_pos": (c_int, [c_void_p]),
    "wf_set_face_positions": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
    "wf_get_face_flux": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_set_face_flux": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_init_from_background": (c_int, [c_void_p, c_void_p, POINTER(c_float), POINTER(c_float), c_float]),
    "wf_set_inflow_plane": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_step": (c_int, [c_void_p, c_int, POINTER(c_int)]),
    "wf_get_vel": (c_int, [c_void_p, POINTER(c_float), c_int]),
    "wf_get_pres": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_get_flags": (c_int, [c_void_p, POINTER(c_int32)]),
    "wf_get_state": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), POINTER(c_int64)]),
    "wf_readback_begin": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "wf_readback_wait": (c_int, [c_void_p]),
    "wf_set_state": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), c_int64]),
    "wf_field_size": (c_int, [c_void_p, c_int, POINTER(c_size_t), POINTER(c_int)]),
    "wf_get_field": (c_int, [c_void_p, c_int, POINTER(c_float)]),
    "wf_set_field": (c_int, [c_void_p, c_int, POINTER(c_float)]),
    "wf_get_device_fields": (c_int, [c_void_p, POINTER(WfDeviceFields)]),
    "wf_residuals": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
    "wf_mass_imbalance": (c_int, [c_void_p, POINTER(c_double)]),
    "wf_check_finite": (c_int, [c_void_p]),
    "wf_op_wallfunc": (c_int, [c_void_p]),
    "wf_op_eddy_vis": (c_int, [c_void_p]),
    "wf_op_les_term": (c_int, [c_void_p]),
    "wf_op_vel_precompute": (c_int, [c_void_p]),
    "wf_op_vel_sweeps": (c_int, [c_void_p, c_int]),
    "wf_op_pres_precompute": (c_int, [c_void_p]),
    "wf_op_pres_sweeps": (c_int, [c_void_p, c_int]),
    "wf_op_apply_pres": (c_int, [c_void_p]),
    "wf_op_normalize": (c_int, [c_void_p]),
    "wf_op_apply_vel": (c_int, [c_void_p]),
    "wf_op_zero_pres_correct": (c_int, [c_void_p]),
    "wf_op_piso": (c_int, [c_void_p, c_int]),
    "wf_op_end_step": (c_int, [c_void_p]),
    "wf_op_vel_residual": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_op_pres_residual": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_last_error": (c_char_p, [c_void_p]),
    "wf_strerror": (c_char_p, [c_int]),
    "wf_version": (c_int, []),
    "wf_last_step_ms": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_kernel_launches": (c_int, [c_void_p, POINTER(c_int64)]),
    "wf_time_kernel": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_float), POINTER(c_double), POINTER(c_int)]),
    "wf_step_phases": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_rasterise_boxes": (c_int, [c_int, c_int, c_int, POINTER(c_double), c_int, c_double, c_int, c_int,
                                   POINTER(c_int32)]),
    "wf_step_async": (c_int, [c_void_p, c_int]),
    "wf_sync": (c_int, [c_void_p]),
    "wf_pres_residual_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, POINTER(c_float)]),
    "wf_batch_create": (c_int, [POINTER(c_void_p), c_int, POINTER(c_void_p)]),
    "wf_batch_destroy": (c_int, [c_void_p]),
    "wf_batch_step": (c_int, [c_void_p, c_int]),
    "wf_batch_last_step_ms": (c_int, [c_void_p, POINTER(c_float)]),
    "wf_batch_kernel_launches": (c_int, [c_void_p, POINTER(c_int64)]),
    "wf_batch_last_error": (c_char_p, [c_void_p]),
    "wf_batch_set_width": (c_int, [c_void_p, c_int]),
    "wf_batch_prepare_graphs": (c_int, [c_void_p]),
    "wf_prepare_graphs": (c_int, [c_void_p]),
    "wf_batch_set_mode": (c_int, [c_void_p, c_int]),
    "wf_batch_get_mode": (c_int, [c_void_p, POINTER(c_int)]),
    "wf_batch_set_barrier_timeout": (c_int, [c_void_p, c_double]),
    "wf_grid_barrier_selftest": (c_int, [c_int, c_int, c_int, c_double, POINTER(c_int)]),
    "wf_stage_wait_selftest": (c_int, [c_void_p, c_int, c_double, POINTER(c_int)]),
    "wf_set_tiles": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    "wf_get_tiles": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "wf_set_blocking": (c_int, [c_void_p, c_int, c_int]),
    "wf_get_blocking": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "wf_export_open": (c_int, [c_void_p, c_char_p, c_int, c_int, c_int, POINTER(c_void_p)]),
    "wf_export_frame": (c_int, [c_void_p, c_float]),
    "wf_export_frames_written": (c_int, [c_void_p, POINTER(c_int64)]),
    "wf_export_last_error": (c_char_p, [c_void_p]),
    "wf_export_close": (c_int, [c_void_p]),
    "wf_adj_create": (c_int, [c_void_p, POINTER(c_void_p)]),
    "wf_adj_destroy": (c_int, [c_void_p]),
    "wf_adj_last_error": (c_char_p, [c_void_p]),
    "wf_adj_set_max_tapes": (c_int, [c_void_p, c_int]),
    "wf_adj_set_segment_policy": (c_int, [c_void_p, c_int]),
    "wf_adj_step_forward": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "wf_adj_step_vjp": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "wf_adj_gradient": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, POINTER(c_double), POINTER(c_double),
                                POINTER(c_double), c_void_p, POINTER(c_float), POINTER(c_float)]),
}

NOALLOC_BLOCKS = 4096
NOALLOC_MAX_CELLS = NOALLOC_BLOCKS * 256 * 64

PHASE_NAMES = ("les", "vel_pre", "vel_sweeps", "pres_pre", "pres_sweeps", "correct", "piso", "end")
PHASE_COUNT = len(PHASE_NAMES)
KERNEL_PRES_SWEEP = 0
KERNEL_VEL_SWEEP = 1

_lib = None


def load(path: str | None = None):
    """Loads libwindfvm.so once and declares every exported signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("WINDFVM_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise WindFvmError(WF_ERR_UNSUPPORTED,
                           f"{p} is missing: build it with `python -m unitywindsimulation_b200.build`")
    lib = ctypes.CDLL(p)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def check(status: int, handle=None) -> None:
    if status == WF_OK:
        return
    lib = load()
    msg = lib.wf_strerror(status).decode()
    if handle:
        detail = lib.wf_last_error(handle)
        if detail:
            msg += f" ({detail.decode()})"
    raise WindFvmError(status, msg)
