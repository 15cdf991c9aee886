"""Host-side mirror of the reference's ``IFvmSolver`` over the C ABI.

``FvmSolverCuda`` exposes the operations of ``IFvmSolver``
(Assets/Code/FvmSolver/IFvmSolver.cs:3-24) with the reference's names and
argument meaning -- ``Step``, ``InitFlags``, ``InitVelPresFields``,
``SetFixedValueVelBndCond``, ``ChangePhysFieldPos``, ``ChangePhysDomainSize``,
``GetVelField``, ``GetPresField``, ``GetFlagField`` -- plus snake_case aliases,
field access for parity checks and the per-kernel operations.

All compute runs in libwindfvm.so on the GPU; a missing library or device
raises ``WindFvmError``.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_void_p

import numpy as np

from . import _lib
from ._lib import WfConfig, WfDeviceFields, WindFvmError, check


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_float))


class FvmSolverCuda:
    """One solver handle on one GPU (FvmSolverGpu equivalent)."""

    def __init__(self, cfg: WfConfig, device: int = 0):
        self._lib = _lib.load()
        self.cfg = cfg.copy()
        self.shape = (cfg.nz, cfg.ny, cfg.nx)  # numpy order of the flat x-fastest arrays
        self.n_cells = cfg.nx * cfg.ny * cfg.nz
        h = c_void_p()
        st = self._lib.wf_create(byref(self.cfg), device, byref(h))
        if st != _lib.WF_OK:
            raise WindFvmError(st, f"wf_create failed: {self._lib.wf_strerror(st).decode()}")
        self._h = h
        self.wind_speed = cfg.wind_speed

    # ---- lifecycle ----
    def close(self):
        if getattr(self, "_h", None):
            self._lib.wf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        check(st, self._h)

    # ---- IFvmSolver ----
    def Step(self, n_steps: int = 1) -> bool:
        ready = c_int(0)
        self._check(self._lib.wf_step(self._h, int(n_steps), byref(ready)))
        return bool(ready.value)

    def prepare_graphs(self) -> None:
        """Captures the step graphs of every buffer-role state ahead of time
        (wf_prepare_graphs); runs no step."""
        self._check(self._lib.wf_prepare_graphs(self._h))

    def InitFlags(self, flags) -> None:
        f = np.ascontiguousarray(np.asarray(flags, dtype=np.int32).reshape(-1))
        if f.size != self.n_cells:
            raise ValueError(f"flags must hold {self.n_cells} values")
        self._check(self._lib.wf_init_flags(self._h, f.ctypes.data_as(POINTER(c_int32)), f.size))

    def InitVelPresFields(self) -> None:
        self._check(self._lib.wf_init_vel_pres_fields(self._h))

    def SetFixedValueVelBndCond(self, wind_speed: float | None = None) -> None:
        if wind_speed is not None:
            self.wind_speed = float(wind_speed)
        self._check(self._lib.wf_set_fixed_value_vel_bnd_cond(self._h, c_float(self.wind_speed)))

    def ChangePhysFieldPos(self) -> None:
        self._check(self._lib.wf_change_phys_field_pos(self._h))

    def set_face_positions(self, fx, fy, fz) -> None:
        """Non-uniform collocated grid (gridType CollNonUniform): face
        positions fx[nx+1], fy[ny+1], fz[nz+1] (wf_set_face_positions).
        Re-initialise the fields afterwards, as the reference's constructor
        builds the mesh first.  All None: back to the uniform grid."""
        if fx is None and fy is None and fz is None:
            self._check(self._lib.wf_set_face_positions(self._h, None, None, None))
            return
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (fx, fy, fz)]
        c = self.cfg
        if [v.size for v in a] != [c.nx + 1, c.ny + 1, c.nz + 1]:
            raise ValueError("face positions need nx+1, ny+1 and nz+1 values")
        self._check(self._lib.wf_set_face_positions(self._h, *[v.ctypes.data_as(POINTER(c_float)) for v in a]))

    def set_face_flux(self, flux) -> None:
        """Writes the face-flux texture, (3, nz+1, ny+1, nx+1) (wf_set_face_flux)."""
        c = self.cfg
        a = np.ascontiguousarray(flux, dtype=np.float32).reshape(-1)
        if a.size != 3 * (c.nx + 1) * (c.ny + 1) * (c.nz + 1):
            raise ValueError("face flux needs 3 (nx+1)(ny+1)(nz+1) values")
        self._check(self._lib.wf_set_face_flux(self._h, a.ctypes.data_as(POINTER(c_float))))

    def get_face_flux(self) -> np.ndarray:
        """Face-flux texture of the non-uniform grid, (3, nz+1, ny+1, nx+1)."""
        c = self.cfg
        m = (c.nx + 1) * (c.ny + 1) * (c.nz + 1)
        out = np.empty(3 * m, dtype=np.float32)
        self._check(self._lib.wf_get_face_flux(self._h, out.ctypes.data_as(POINTER(c_float))))
        return out.reshape(3, c.nz + 1, c.ny + 1, c.nx + 1)

    def InitVelPresFieldsFromBackGroundFlow(self, background: "FvmSolverCuda", pos=(0.0, 0.0, 0.0),
                                            pos_background=(0.0, 0.0, 0.0), rot_deg: float = 0.0) -> None:
        """Velocity and pressure from a background solver's current fields,
        sampled at this domain's cells (wf_init_from_background).  pos /
        pos_background: domain centres (physFieldPos), rot_deg: this domain's
        rotation about the vertical axis (flowFieldOrientation)."""
        p = (c_float * 3)(*[float(v) for v in pos])
        q = (c_float * 3)(*[float(v) for v in pos_background])
        self._check(self._lib.wf_init_from_background(self._h, background._h, p, q, float(rot_deg)))

    def ChangePhysDomainSize(self, cfg: WfConfig | None = None, device: int = 0) -> None:
        """Re-creates the handle for a new grid (the reference re-reads gridRes
        and re-initialises the fields, FvmSolverGpu.cs:1034-1046)."""
        new = (cfg or self.cfg).copy()
        self.close()
        self.__init__(new, device)

    def GetVelField(self, layout: int = _lib.LAYOUT_SOA, out: np.ndarray | None = None) -> np.ndarray:
        """Current velocity.  SOA -> (3, nz, ny, nx); XYZW -> (nz, ny, nx, 4).
        `out` (float32, contiguous, right size) may be a pinned host buffer."""
        n = self.n_cells
        per = {_lib.LAYOUT_SOA: 3, _lib.LAYOUT_XYZW: 4, _lib.LAYOUT_XYZ: 3}[layout]
        if out is None:
            out = np.empty(per * n, dtype=np.float32)
        elif out.dtype != np.float32 or out.size != per * n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array of the field's size")
        self._check(self._lib.wf_get_vel(self._h, _fptr(out), layout))
        if layout == _lib.LAYOUT_SOA:
            return out.reshape((3,) + self.shape)
        return out.reshape(self.shape + (per,))

    def readback_begin(self, vel_out: np.ndarray, pres_out: np.ndarray, layout: int = _lib.LAYOUT_SOA) -> None:
        """Starts an asynchronous copy of the current velocity (layout SOA:
        3N floats, XYZW: 4N, XYZ: 3N) and pressure (N) into the given host
        arrays (page-locked memory for a truly asynchronous copy); they are
        complete after readback_wait().  Keep the arrays alive until then."""
        n = self.n_cells
        per = {_lib.LAYOUT_SOA: 3, _lib.LAYOUT_XYZW: 4, _lib.LAYOUT_XYZ: 3}[layout]
        for a, size in ((vel_out, per * n), (pres_out, n)):
            if a.dtype != np.float32 or a.size != size or not a.flags.c_contiguous:
                raise ValueError("readback buffers must be contiguous float32 arrays of the field sizes")
        self._check(self._lib.wf_readback_begin(self._h, vel_out.ctypes.data, pres_out.ctypes.data, int(layout)))

    def readback_wait(self) -> None:
        self._check(self._lib.wf_readback_wait(self._h))

    def GetPresField(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n_cells, dtype=np.float32)
        elif out.dtype != np.float32 or out.size != self.n_cells or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array of the field's size")
        self._check(self._lib.wf_get_pres(self._h, _fptr(out)))
        return out.reshape(self.shape)

    def GetFlagField(self) -> np.ndarray:
        out = np.empty(self.n_cells, dtype=np.int32)
        self._check(self._lib.wf_get_flags(self._h, out.ctypes.data_as(POINTER(c_int32))))
        return out.reshape(self.shape)

    # snake_case aliases
    step = Step
    init_flags = InitFlags
    init_vel_pres_fields = InitVelPresFields
    set_fixed_value_vel_bnd_cond = SetFixedValueVelBndCond
    get_vel = GetVelField
    get_pres = GetPresField
    get_flags = GetFlagField

    # ---- extras ----
    def set_inflow_plane(self, plane_xyz: np.ndarray) -> None:
        """X0 inlet plane, shape (nz, ny, 3)."""
        a = np.ascontiguousarray(plane_xyz, dtype=np.float32).reshape(-1)
        if a.size != 3 * self.cfg.ny * self.cfg.nz:
            raise ValueError("inlet plane must be (nz, ny, 3)")
        self._check(self._lib.wf_set_inflow_plane(self._h, _fptr(a)))

    def get_state(self):
        vel = np.empty(3 * self.n_cells, dtype=np.float32)
        pres = np.empty(self.n_cells, dtype=np.float32)
        step = c_int64(0)
        self._check(self._lib.wf_get_state(self._h, _fptr(vel), _fptr(pres), byref(step)))
        return vel.reshape((3,) + self.shape), pres.reshape(self.shape), step.value

    def set_state(self, vel: np.ndarray, pres: np.ndarray, step: int = 0) -> None:
        v = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1)
        p = np.ascontiguousarray(pres, dtype=np.float32).reshape(-1)
        self._check(self._lib.wf_set_state(self._h, _fptr(v), _fptr(p), int(step)))

    def field_size(self, field: int):
        pts, comps = c_size_t(0), c_int(0)
        self._check(self._lib.wf_field_size(self._h, field, byref(pts), byref(comps)))
        return pts.value, comps.value

    def get_field(self, field: int) -> np.ndarray:
        pts, comps = self.field_size(field)
        out = np.empty(pts * comps, dtype=np.float32)
        self._check(self._lib.wf_get_field(self._h, field, _fptr(out)))
        return out.reshape((comps, pts)) if comps > 1 else out

    def set_field(self, field: int, data: np.ndarray) -> None:
        pts, comps = self.field_size(field)
        a = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
        if a.size != pts * comps:
            raise ValueError(f"field {field} needs {pts * comps} floats")
        self._check(self._lib.wf_set_field(self._h, field, _fptr(a)))

    def device_fields(self) -> WfDeviceFields:
        d = WfDeviceFields()
        self._check(self._lib.wf_get_device_fields(self._h, byref(d)))
        return d

    def residuals(self):
        v, p, m = c_float(0), c_float(0), c_float(0)
        self._check(self._lib.wf_residuals(self._h, byref(v), byref(p), byref(m)))
        return v.value, p.value, m.value

    def mass_imbalance(self) -> float:
        m = c_double(0)
        self._check(self._lib.wf_mass_imbalance(self._h, byref(m)))
        return m.value

    def check_finite(self) -> None:
        self._check(self._lib.wf_check_finite(self._h))

    def last_step_ms(self) -> float:
        ms = c_float(0)
        self._check(self._lib.wf_last_step_ms(self._h, byref(ms)))
        return ms.value

    def kernel_launches(self) -> int:
        n = c_int64(0)
        self._check(self._lib.wf_kernel_launches(self._h, byref(n)))
        return n.value

    def step_async(self, n_steps: int = 1) -> None:
        """Enqueues n_steps steps without waiting for them (wf_step_async)."""
        self._check(self._lib.wf_step_async(self._h, int(n_steps)))

    def sync(self) -> None:
        """Waits for every step and copy enqueued on the solver's stream."""
        self._check(self._lib.wf_sync(self._h))

    def step_phases(self) -> dict:
        """One step enqueued kernel by kernel with a CUDA event between its
        phases (wf_step_phases): {phase name: device ms}.  The fields end as
        after Step(1)."""
        out = (c_float * _lib.PHASE_COUNT)()
        self._check(self._lib.wf_step_phases(self._h, out))
        return {n: float(out[i]) for i, n in enumerate(_lib.PHASE_NAMES)}

    def time_kernel(self, kernel: int, reps: int = 20, flush_l2: bool = True):
        """(ms per launch, algorithmic bytes per launch, sweeps per launch)."""
        ms, by, sw = c_float(0), c_double(0), c_int(0)
        self._check(self._lib.wf_time_kernel(self._h, kernel, reps, int(flush_l2), byref(ms), byref(by), byref(sw)))
        return ms.value, by.value, sw.value

    @property
    def stream_ptr(self) -> int:
        return int(self.device_fields().stream or 0)

    def set_blocking(self, pres_k: int, vel_k: int) -> None:
        self._check(self._lib.wf_set_blocking(self._h, int(pres_k), int(vel_k)))

    def get_blocking(self):
        p, v = c_int(0), c_int(0)
        self._check(self._lib.wf_get_blocking(self._h, byref(p), byref(v)))
        return p.value, v.value

    def set_tiles(self, pres_rows: int, vel_block=(32, 4, 2)) -> None:
        """Tile shapes of the Jacobi kernels (wf_set_tiles): pressure
        multi-sweep tile rows (32 or 16) and the momentum sweep's block."""
        bx, by, bz = (int(v) for v in vel_block)
        self._check(self._lib.wf_set_tiles(self._h, int(pres_rows), bx, by, bz))

    def get_tiles(self):
        p, x, y, z = c_int(0), c_int(0), c_int(0), c_int(0)
        self._check(self._lib.wf_get_tiles(self._h, byref(p), byref(x), byref(y), byref(z)))
        return p.value, (x.value, y.value, z.value)

    # ---- per-kernel operations ----
    def op(self, name: str, *args) -> None:
        fn = getattr(self._lib, f"wf_op_{name}")
        self._check(fn(self._h, *[int(a) for a in args]))

    def op_residual(self, which: str) -> float:
        out = c_float(0)
        fn = getattr(self._lib, f"wf_op_{which}_residual")
        self._check(fn(self._h, byref(out)))
        return out.value


class FieldExporter:
    """Velocity/pressure frames appended to a netCDF file while the solver
    runs (wf_export_*; the file layout of the reference's
    NcFlowFieldExporter).  ``frame(t)`` queues the solver's current fields;
    ``close()`` drains the queue and finalises the file."""

    def __init__(self, solver: FvmSolverCuda, path: str, save_vel: bool = True, save_pres: bool = True,
                 ring: int = 3):
        self._lib = _lib.load()
        self.solver = solver
        e = c_void_p()
        st = self._lib.wf_export_open(solver._h, str(path).encode(), int(save_vel), int(save_pres), int(ring),
                                      byref(e))
        if st != _lib.WF_OK:
            raise WindFvmError(st, f"wf_export_open: {self._lib.wf_last_error(solver._h).decode()}")
        self._e = e

    def _check(self, st):
        if st != _lib.WF_OK:
            raise WindFvmError(st, self._lib.wf_export_last_error(self._e).decode() or
                               self._lib.wf_strerror(st).decode())

    def frame(self, phys_time: float) -> None:
        self._check(self._lib.wf_export_frame(self._e, float(phys_time)))

    def frames_written(self) -> int:
        n = c_int64(0)
        self._check(self._lib.wf_export_frames_written(self._e, byref(n)))
        return n.value

    def close(self) -> None:
        if getattr(self, "_e", None):
            e, self._e = self._e, None
            st = self._lib.wf_export_close(e)
            if st != _lib.WF_OK:
                raise WindFvmError(st, "wf_export_close failed")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchSolver:
    """Several FvmSolverCuda handles stepped together by one graph launch per
    step (wf_batch_*).  The handles stay usable on their own."""

    def __init__(self, solvers):
        self._lib = _lib.load()
        self.solvers = list(solvers)
        arr = (c_void_p * len(self.solvers))(*[s._h for s in self.solvers])
        b = c_void_p()
        st = self._lib.wf_batch_create(arr, len(self.solvers), byref(b))
        if st != _lib.WF_OK:
            raise WindFvmError(st, "wf_batch_create failed")
        self._b = b

    def _check(self, st):
        if st != _lib.WF_OK:
            raise WindFvmError(st, self._lib.wf_batch_last_error(self._b).decode())

    def step(self, n_steps: int = 1) -> None:
        self._check(self._lib.wf_batch_step(self._b, int(n_steps)))

    def last_step_ms(self) -> float:
        ms = c_float(0)
        self._check(self._lib.wf_batch_last_step_ms(self._b, byref(ms)))
        return ms.value

    def set_width(self, width: int) -> None:
        self._check(self._lib.wf_batch_set_width(self._b, int(width)))

    def set_mode(self, mode: int) -> None:
        """_lib.BATCH_GRAPHS (child graphs) or _lib.BATCH_PERSISTENT (one
        persistent launch per Jacobi loop over all cases)."""
        self._check(self._lib.wf_batch_set_mode(self._b, int(mode)))

    def get_mode(self) -> int:
        m = c_int(0)
        self._check(self._lib.wf_batch_get_mode(self._b, byref(m)))
        return m.value

    def set_barrier_timeout(self, ms: float) -> None:
        self._check(self._lib.wf_batch_set_barrier_timeout(self._b, float(ms)))

    def prepare_graphs(self) -> None:
        """Captures the batch graphs of every buffer-role state ahead of time
        (wf_batch_prepare_graphs); runs no step."""
        self._check(self._lib.wf_batch_prepare_graphs(self._b))

    def kernel_launches(self) -> int:
        n = c_int64(0)
        self._check(self._lib.wf_batch_kernel_launches(self._b, byref(n)))
        return n.value

    @property
    def n_cells(self) -> int:
        return sum(s.n_cells for s in self.solvers)

    def close(self):
        if getattr(self, "_b", None):
            self._lib.wf_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Reference-style name for the solver class.
FvmSolverGpu = FvmSolverCuda
