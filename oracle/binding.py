"""ctypes binding of libwindfvm_oracle.so (test infrastructure only)."""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, byref, c_double, c_float, c_int, c_int32, c_size_t, c_void_p

import numpy as np

from unitywindsimulation_b200._lib import WfConfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwindfvm_oracle.so")

_lib = None


def build_oracle(force: bool = False) -> str:
    args = ["make", "-s", "-C", HERE]
    if force:
        args.append("-B")
    subprocess.run(args, check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build_oracle()
    lib = ctypes.CDLL(LIB_PATH)
    sig = {
        "wfo_create": (c_int, [POINTER(WfConfig), c_int, c_int, POINTER(c_void_p)]),
        "wfo_destroy": (c_int, [c_void_p]),
        "wfo_init_flags": (c_int, [c_void_p, POINTER(c_int32), c_size_t]),
        "wfo_init_vel_pres_fields": (c_int, [c_void_p]),
        "wfo_set_fixed_value_vel_bnd_cond": (c_int, [c_void_p, c_float]),
        "wfo_set_inflow_plane": (c_int, [c_void_p, POINTER(c_float)]),
        "wfo_init_from_background": (c_int, [c_void_p, c_void_p, POINTER(c_float), POINTER(c_float), c_float]),
        "wfo_step": (c_int, [c_void_p, c_int]),
        "wfo_set_face_positions": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
        "wfo_get_face_flux": (c_int, [c_void_p, POINTER(c_double)]),
        "wfo_field_size": (c_int, [c_void_p, c_int, POINTER(c_size_t), POINTER(c_int)]),
        "wfo_get_field": (c_int, [c_void_p, c_int, POINTER(c_double)]),
        "wfo_set_field": (c_int, [c_void_p, c_int, POINTER(c_double)]),
        "wfo_get_flags": (c_int, [c_void_p, POINTER(c_int32)]),
        "wfo_op_vel_sweeps": (c_int, [c_void_p, c_int]),
        "wfo_op_pres_sweeps": (c_int, [c_void_p, c_int]),
        "wfo_op_piso": (c_int, [c_void_p, c_int]),
        "wfo_op_vel_residual": (c_int, [c_void_p, POINTER(c_double)]),
        "wfo_op_pres_residual": (c_int, [c_void_p, POINTER(c_double)]),
        "wfo_residuals": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double)]),
        "wfo_mass_imbalance": (c_int, [c_void_p, POINTER(c_double)]),
        "wfo_log_law_wall_func": (c_double, [c_double, c_double, c_double, c_double, c_int]),
    }
    for op in ["wallfunc", "eddy_vis", "les_term", "vel_precompute", "pres_precompute", "apply_pres",
               "normalize", "apply_vel", "zero_pres_correct", "end_step"]:
        sig[f"wfo_op_{op}"] = (c_int, [c_void_p])
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def log_law_wall_func(uP: float, dx: float, nu: float, den: float = 1.0, precision: int = 64) -> float:
    return load().wfo_log_law_wall_func(uP, dx, nu, den, precision)


class OracleSolver:
    """CPU restatement of the step with the same operations as FvmSolverCuda."""

    def __init__(self, cfg: WfConfig, precision: int = 64, threads: int = 0):
        self._lib = load()
        self.cfg = cfg.copy()
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.n_cells = cfg.nx * cfg.ny * cfg.nz
        h = c_void_p()
        st = self._lib.wfo_create(byref(self.cfg), precision, threads, byref(h))
        if st != 0:
            raise RuntimeError(f"wfo_create failed with status {st}")
        self._h = h
        self.wind_speed = cfg.wind_speed

    def close(self):
        if getattr(self, "_h", None):
            self._lib.wfo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, st):
        if st != 0:
            raise RuntimeError(f"oracle call failed with status {st}")

    def Step(self, n_steps: int = 1) -> bool:
        self._ok(self._lib.wfo_step(self._h, int(n_steps)))
        return True

    def InitFlags(self, flags):
        f = np.ascontiguousarray(np.asarray(flags, dtype=np.int32).reshape(-1))
        self._ok(self._lib.wfo_init_flags(self._h, f.ctypes.data_as(POINTER(c_int32)), f.size))

    def InitVelPresFields(self):
        self._ok(self._lib.wfo_init_vel_pres_fields(self._h))

    def SetFixedValueVelBndCond(self, wind_speed=None):
        if wind_speed is not None:
            self.wind_speed = float(wind_speed)
        self._ok(self._lib.wfo_set_fixed_value_vel_bnd_cond(self._h, c_float(self.wind_speed)))

    def InitVelPresFieldsFromBackGroundFlow(self, background, pos=(0.0, 0.0, 0.0), pos_background=(0.0, 0.0, 0.0),
                                            rot_deg=0.0):
        p = (c_float * 3)(*[float(v) for v in pos])
        q = (c_float * 3)(*[float(v) for v in pos_background])
        self._ok(self._lib.wfo_init_from_background(self._h, background._h, p, q, float(rot_deg)))

    def set_inflow_plane(self, plane_xyz):
        a = np.ascontiguousarray(plane_xyz, dtype=np.float32).reshape(-1)
        self._ok(self._lib.wfo_set_inflow_plane(self._h, a.ctypes.data_as(POINTER(c_float))))

    def GetFlagField(self):
        out = np.empty(self.n_cells, dtype=np.int32)
        self._ok(self._lib.wfo_get_flags(self._h, out.ctypes.data_as(POINTER(c_int32))))
        return out.reshape(self.shape)

    def set_face_positions(self, fx, fy, fz):
        """Non-uniform collocated grid (gridType CollNonUniform): face
        positions fx[nx+1], fy[ny+1], fz[nz+1]; all None: uniform grid."""
        if fx is None and fy is None and fz is None:
            self._ok(self._lib.wfo_set_face_positions(self._h, None, None, None))
            return
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (fx, fy, fz)]
        self._ok(self._lib.wfo_set_face_positions(self._h, *[v.ctypes.data_as(POINTER(c_float)) for v in a]))

    def get_face_flux(self) -> np.ndarray:
        """velFaceFluxField: (3, nz+1, ny+1, nx+1)."""
        nz, ny, nx = self.shape
        out = np.empty(3 * (nx + 1) * (ny + 1) * (nz + 1), dtype=np.float64)
        self._ok(self._lib.wfo_get_face_flux(self._h, out.ctypes.data_as(POINTER(c_double))))
        return out.reshape(3, nz + 1, ny + 1, nx + 1)

    def field_size(self, field):
        pts, comps = c_size_t(0), c_int(0)
        self._ok(self._lib.wfo_field_size(self._h, field, byref(pts), byref(comps)))
        return pts.value, comps.value

    def get_field(self, field) -> np.ndarray:
        pts, comps = self.field_size(field)
        out = np.empty(pts * comps, dtype=np.float64)
        self._ok(self._lib.wfo_get_field(self._h, field, out.ctypes.data_as(POINTER(c_double))))
        return out.reshape((comps, pts)) if comps > 1 else out

    def set_field(self, field, data):
        a = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
        self._ok(self._lib.wfo_set_field(self._h, field, a.ctypes.data_as(POINTER(c_double))))

    def GetVelField(self):
        return self.get_field(1).reshape((3,) + self.shape)

    def GetPresField(self):
        return self.get_field(4).reshape(self.shape)

    def op(self, name, *args):
        self._ok(getattr(self._lib, f"wfo_op_{name}")(self._h, *[int(a) for a in args]))

    def op_residual(self, which) -> float:
        out = c_double(0)
        self._ok(getattr(self._lib, f"wfo_op_{which}_residual")(self._h, byref(out)))
        return out.value

    def residuals(self):
        v, p = c_double(0), c_double(0)
        self._ok(self._lib.wfo_residuals(self._h, byref(v), byref(p)))
        return v.value, p.value

    def mass_imbalance(self) -> float:
        m = c_double(0)
        self._ok(self._lib.wfo_mass_imbalance(self._h, byref(m)))
        return m.value


# ---- the reference's own kernels (oracle/ref_driver.cpp) --------------------

REF_LIB_PATH = os.path.join(HERE, "_ref", "libwindfvm_ref.so")
_ref_lib = None


def ref_available() -> bool:
    """True when the reference-kernel library has been built into _ref/."""
    return os.path.exists(REF_LIB_PATH)


def build_ref(reference_root: str) -> str:
    """Translates the reference's shaders found under `reference_root` and
    builds _ref/libwindfvm_ref.so (make ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE_ROOT={reference_root}"], check=True)
    return REF_LIB_PATH


def load_ref():
    global _ref_lib
    if _ref_lib is not None:
        return _ref_lib
    if not ref_available():
        raise FileNotFoundError(f"{REF_LIB_PATH} is not built (make -C oracle ref)")
    lib = ctypes.CDLL(REF_LIB_PATH)
    sig = {
        "wfr_create": (c_int, [POINTER(WfConfig), POINTER(c_void_p)]),
        "wfr_create_empty": (c_int, [POINTER(WfConfig), POINTER(c_void_p)]),
        "wfr_destroy": (c_int, [c_void_p]),
        "wfr_set_flags": (c_int, [c_void_p, POINTER(c_int32), c_size_t]),
        "wfr_set_field": (c_int, [c_void_p, c_int, POINTER(c_float)]),
        "wfr_get_field": (c_int, [c_void_p, c_int, POINTER(c_float)]),
        "wfr_step": (c_int, [c_void_p, c_int]),
        "wfr_get_flags": (c_int, [c_void_p, POINTER(c_int32)]),
        "wfr_init_flags": (c_int, [c_void_p, POINTER(c_int32), c_size_t]),
        "wfr_init_vel_pres_fields": (c_int, [c_void_p, c_float]),
        "wfr_set_fixed_value_vel_bnd_cond": (c_int, [c_void_p, c_float]),
        "wfr_init_from_background": (c_int, [c_void_p, c_void_p, POINTER(c_float), POINTER(c_float), c_float]),
        "wfr_set_face_positions": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
        "wfr_get_face_flux": (c_int, [c_void_p, POINTER(c_float)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _ref_lib = lib
    return lib


# Fields a step reads before writing them (everything else is rebuilt inside
# the step): the three velocity textures, pressure, the pressure-correction
# pair, face eddy viscosity and the six boundary planes.
REF_STATE_FIELDS = (0, 1, 2, 4, 5, 6, 13, 14, 15, 16, 17, 18, 19)


class RefSolver:
    """FvmSolverGpu replayed with the reference's own kernels on the CPU
    (FP32): the constructor's set-up, InitFlags, InitVelPresFields,
    SetFixedValueVelBndCond, InitVelPresFieldsFromBackGroundFlow and Step.
    copy_state_from takes another solver's state instead, to compare single
    steps from identical inputs."""

    def __init__(self, cfg: WfConfig, construct: bool = True):
        """construct=False skips the constructor's set-up (every field zero),
        for a state taken from another solver with copy_state_from."""
        self._lib = load_ref()
        self.cfg = cfg.copy()
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        self.n_cells = cfg.nx * cfg.ny * cfg.nz
        h = c_void_p()
        create = self._lib.wfr_create if construct else self._lib.wfr_create_empty
        st = create(byref(self.cfg), byref(h))
        if st != 0:
            raise RuntimeError(f"wfr_create failed with status {st}")
        self._h = h
        self.wind_speed = cfg.wind_speed

    def close(self):
        if getattr(self, "_h", None):
            self._lib.wfr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, st):
        if st != 0:
            raise RuntimeError(f"reference-kernel call failed with status {st}")

    def _points(self, field):
        c = self.cfg
        if field in (14, 15):
            return c.ny * c.nz
        if field in (16, 17):
            return c.nx * c.nz
        if field in (18, 19):
            return c.nx * c.ny
        return self.n_cells

    def _comps(self, field):
        return 1 if field in (4, 5, 6, 9, 10, 12) else 3

    def set_flags(self, flags):
        f = np.ascontiguousarray(np.asarray(flags, dtype=np.int32).reshape(-1))
        self._ok(self._lib.wfr_set_flags(self._h, f.ctypes.data_as(POINTER(c_int32)), f.size))

    def InitFlags(self, flags):
        f = np.ascontiguousarray(np.asarray(flags, dtype=np.int32).reshape(-1))
        self._ok(self._lib.wfr_init_flags(self._h, f.ctypes.data_as(POINTER(c_int32)), f.size))

    def GetFlagField(self):
        out = np.empty(self.n_cells, dtype=np.int32)
        self._ok(self._lib.wfr_get_flags(self._h, out.ctypes.data_as(POINTER(c_int32))))
        return out.reshape(self.shape)

    def InitVelPresFields(self):
        self._ok(self._lib.wfr_init_vel_pres_fields(self._h, c_float(self.wind_speed)))

    def SetFixedValueVelBndCond(self, wind_speed=None):
        if wind_speed is not None:
            self.wind_speed = float(wind_speed)
        self._ok(self._lib.wfr_set_fixed_value_vel_bnd_cond(self._h, c_float(self.wind_speed)))

    def InitVelPresFieldsFromBackGroundFlow(self, background, pos=(0.0, 0.0, 0.0), pos_background=(0.0, 0.0, 0.0),
                                            rot_deg=0.0):
        p = (c_float * 3)(*[float(v) for v in pos])
        q = (c_float * 3)(*[float(v) for v in pos_background])
        self._ok(self._lib.wfr_init_from_background(self._h, background._h, p, q, float(rot_deg)))

    def set_field(self, field, data):
        a = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
        if a.size != self._points(field) * self._comps(field):
            raise ValueError(f"field {field}: {a.size} values")
        self._ok(self._lib.wfr_set_field(self._h, int(field), a.ctypes.data_as(POINTER(c_float))))

    def get_field(self, field) -> np.ndarray:
        pts, comps = self._points(field), self._comps(field)
        out = np.empty(pts * comps, dtype=np.float32)
        self._ok(self._lib.wfr_get_field(self._h, int(field), out.ctypes.data_as(POINTER(c_float))))
        return out.reshape((comps, pts)) if comps > 1 else out

    def copy_state_from(self, other):
        """Takes flags and every field a step reads from `other` (an
        OracleSolver, or anything with get_field and GetFlagField)."""
        self.set_flags(np.asarray(other.GetFlagField()).reshape(-1))
        for f in REF_STATE_FIELDS:
            self.set_field(f, np.asarray(other.get_field(f), dtype=np.float32))

    def Step(self, n_steps: int = 1) -> bool:
        self._ok(self._lib.wfr_step(self._h, int(n_steps)))
        return True

    def set_face_positions(self, fx, fy, fz):
        """Non-uniform collocated grid (gridType CollNonUniform) with face
        positions fx[nx+1], fy[ny+1], fz[nz+1]; all None: uniform grid."""
        if fx is None and fy is None and fz is None:
            self._ok(self._lib.wfr_set_face_positions(self._h, None, None, None))
            return
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (fx, fy, fz)]
        self._keep_fpos = a
        self._ok(self._lib.wfr_set_face_positions(self._h, *[v.ctypes.data_as(POINTER(c_float)) for v in a]))

    def get_face_flux(self) -> np.ndarray:
        """velFaceFluxField: (3, nz+1, ny+1, nx+1)."""
        c = self.cfg
        m = (c.nx + 1) * (c.ny + 1) * (c.nz + 1)
        out = np.empty(3 * m, dtype=np.float32)
        self._ok(self._lib.wfr_get_face_flux(self._h, out.ctypes.data_as(POINTER(c_float))))
        return out.reshape(3, c.nz + 1, c.ny + 1, c.nx + 1)

    def GetVelField(self):
        return self.get_field(1).reshape((3,) + self.shape)

    def GetPresField(self):
        return self.get_field(4).reshape(self.shape)
