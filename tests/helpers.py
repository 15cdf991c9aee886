"""Shared helpers of the parity tests."""
import numpy as np

from unitywindsimulation_b200 import _lib

VEC_FIELDS = [_lib.FIELD_VEL, _lib.FIELD_VEL_LAST_TIME, _lib.FIELD_VEL_LAST_ITER, _lib.FIELD_VEL_CORRECT,
              _lib.FIELD_D, _lib.FIELD_B, _lib.FIELD_AODU, _lib.FIELD_FACE_EDDY_VIS]
SCA_FIELDS = [_lib.FIELD_PRES, _lib.FIELD_PRES_CORRECT, _lib.FIELD_PRES_CORRECT_LAST_ITER, _lib.FIELD_DP,
              _lib.FIELD_BP, _lib.FIELD_EDDY_VIS]
BND_FIELDS = list(range(_lib.FIELD_BND_X0, _lib.FIELD_BND_ZN + 1))
ALL_FIELDS = VEC_FIELDS + SCA_FIELDS + BND_FIELDS

# Per-field, per-step parity bound of the CUDA FP32 fields against the FP32
# oracle: relative L2 norm of the difference.
REL_TOL = 1e-5


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    if nb == 0.0:
        return d
    return d / nb


def copy_state(src, dst, fields=ALL_FIELDS):
    """Copies every named field from one solver (GPU or oracle) to another."""
    for f in fields:
        dst.set_field(f, np.asarray(src.get_field(f), dtype=np.float64))


def fluid_mask(flags):
    return (np.asarray(flags).reshape(-1) == 0)
