"""Discrete adjoint of the fixed-iteration step (wf_adj_* in include/windfvm.h).

``AdjointSolver`` wraps one ``FvmSolverCuda`` handle: vector-Jacobian
products of one step (cut after the momentum predictor, the SIMPLE
correction or the whole step) and the gradient of the pedestrian-comfort
objective with respect to the log-inflow parameters and the drag field of a
soft building mask over a window of steps.
``WindObjective`` exposes that gradient (inflow parameters and soft building
heights) as a ``torch.autograd.Function``.

The reference has no derivatives; the operations differentiated are the ones
of ``FvmSolverGpu.Step`` (Assets/Code/FvmSolver/FvmSolverGpu.cs:1050-1121)
with turbulence off.  All compute runs in libwindfvm.so on the GPU.
"""
from __future__ import annotations

from ctypes import POINTER, byref, c_double, c_float, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import WfObjective, WindFvmError
from .soft_mask import SoftBuildings
from .solver import FvmSolverCuda

PHASE_PREDICTOR, PHASE_SIMPLE, PHASE_FULL = 1, 2, 3


@dataclass
class Objective:
    """Mean |u|^2 over the fluid cells of the patch x0<=x<x1, z0<=z<z1 at
    height index y, averaged over the last ``window`` steps."""
    x0: int
    x1: int
    z0: int
    z1: int
    y: int
    window: int

    def to_c(self) -> WfObjective:
        return WfObjective(self.x0, self.x1, self.z0, self.z1, self.y, self.window)

    def evaluate(self, vel: np.ndarray, flags: np.ndarray) -> float:
        """One step's term (before the 1/window factor) from a (3, nz, ny, nx)
        velocity and (nz, ny, nx) flags, in float64."""
        u = np.asarray(vel, dtype=np.float64)[:, self.z0:self.z1, self.y, self.x0:self.x1]
        m = np.asarray(flags)[self.z0:self.z1, self.y, self.x0:self.x1] == _lib.CELL_FLUID
        area = (self.x1 - self.x0) * (self.z1 - self.z0)
        return float((u ** 2).sum(axis=0)[m].sum() / area)


class AdjointSolver:
    """Adjoint handle on one solver (wf_adj_create).  The solver must stay
    alive while this object is used."""

    def __init__(self, solver: FvmSolverCuda):
        self._lib = _lib.load()
        self.solver = solver
        a = c_void_p()
        st = self._lib.wf_adj_create(solver._h, byref(a))
        if st != _lib.WF_OK:
            raise WindFvmError(st, f"wf_adj_create: {self._lib.wf_strerror(st).decode()}")
        self._a = a
        self.plane_sizes = [solver.field_size(_lib.FIELD_BND_X0 + f)[0] for f in range(6)]

    def _check(self, st: int):
        if st != _lib.WF_OK:
            raise WindFvmError(st, self._lib.wf_adj_last_error(self._a).decode() or
                               self._lib.wf_strerror(st).decode())

    def close(self):
        if getattr(self, "_a", None):
            self._lib.wf_adj_destroy(self._a)
            self._a = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_max_tapes(self, max_tapes: int) -> None:
        """Caps the step tapes a gradient keeps on the device (0: as many as
        fit); longer checkpoint segments are reversed in sub-blocks."""
        self._check(self._lib.wf_adj_set_max_tapes(self._a, int(max_tapes)))

    def set_segment_policy(self, shorten: bool) -> None:
        """True (default): when a checkpoint segment's tapes do not fit,
        shorten the segments to the tapes that fit (each step recomputed
        once); False: keep the interval and reverse in sub-blocks from stored
        segment states (each step recomputed twice)."""
        self._check(self._lib.wf_adj_set_segment_policy(self._a, int(bool(shorten))))

    def step_forward(self, phases: int = PHASE_FULL):
        """State after one step from the solver's current state, cut after
        ``phases`` parts; the solver does not advance.  Returns (u (3, N), p (N))."""
        n = self.solver.n_cells
        u = np.empty((3, n), dtype=np.float32)
        p = np.empty(n, dtype=np.float32)
        self._check(self._lib.wf_adj_step_forward(self._a, int(phases), u.ctypes.data, p.ctypes.data))
        return u, p

    def step_vjp(self, ubar: np.ndarray, pbar: np.ndarray, phases: int = PHASE_FULL):
        """Adjoints of the step input (u, p), of the six boundary planes and of
        the drag field for output adjoints (ubar (3, N), pbar (N)).  Returns
        (ubar_in, pbar_in, planes, dragbar) with planes[f] of shape
        (3, points of plane f)."""
        n = self.solver.n_cells
        ub = np.ascontiguousarray(ubar, dtype=np.float32).reshape(3, n)
        pb = np.ascontiguousarray(pbar, dtype=np.float32).reshape(n)
        ui = np.empty((3, n), dtype=np.float32)
        pi = np.empty(n, dtype=np.float32)
        g = np.empty(3 * sum(self.plane_sizes), dtype=np.float32)
        db = np.empty(n, dtype=np.float32)
        self._check(self._lib.wf_adj_step_vjp(self._a, int(phases), ub.ctypes.data, pb.ctypes.data, ui.ctypes.data,
                                              pi.ctypes.data, g.ctypes.data, db.ctypes.data))
        planes, o = [], 0
        for s in self.plane_sizes:
            planes.append(g[o:o + 3 * s].reshape(3, s))
            o += 3 * s
        return ui, pi, planes, db

    def gradient(self, objective: Objective, n_steps: int, checkpoint_every: int = 1, include_init: bool = True,
                 soft: SoftBuildings | None = None):
        """Advances the solver ``n_steps`` steps and returns a dict with the
        objective J, dJ/du*, dJ/dz0, dJ/dchi (the drag field, (N,)), the
        device times of the forward pass and of the whole call (ms) and, when
        ``soft`` describes the solver's drag field, dJ/dh per building."""
        J, gu, gz = c_double(0), c_double(0), c_double(0)
        tf, tt = c_float(0), c_float(0)
        dd = np.empty(self.solver.n_cells, dtype=np.float32)
        obj = objective.to_c()
        self._check(self._lib.wf_adj_gradient(self._a, byref(obj), int(n_steps), int(checkpoint_every),
                                              int(bool(include_init)), byref(J), byref(gu), byref(gz), dd.ctypes.data,
                                              byref(tf), byref(tt)))
        out = {"J": J.value, "dJ_dustar": gu.value, "dJ_dz0": gz.value, "dJ_ddrag": dd, "ms_forward": tf.value,
               "ms_total": tt.value}
        if soft is not None:
            c = self.solver.cfg
            out["dJ_dheights"] = soft.height_gradient(dd, c.nx, c.ny, c.nz)
        return out


def _torch():
    import torch
    return torch


class WindObjective:
    """``torch.autograd.Function`` of the pedestrian-comfort objective J(u*,
    z0[, h_1..h_n]):

        J = WindObjective.apply(params, make_solver, objective, n_steps,
                                checkpoint_every, soft)

    ``params`` is a float64 tensor [u*, z0] or, with a SoftBuildings ``soft``,
    [u*, z0, h_1, ..., h_n]; ``make_solver(ustar, z0, soft_or_None)`` returns
    a freshly initialised FvmSolverCuda (flags set, fields at the inflow
    profile, drag field from the soft buildings).  The backward pass returns
    dJ/dparams from the discrete adjoint."""

    _fn = None

    @classmethod
    def _function(cls):
        if cls._fn is None:
            torch = _torch()

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, params, make_solver, objective, n_steps, checkpoint_every, soft):
                    v = [float(x) for x in params.detach().cpu().tolist()]
                    sb = soft.with_heights(v[2:]) if soft is not None else None
                    solver = make_solver(v[0], v[1], sb)
                    try:
                        with AdjointSolver(solver) as adj:
                            r = adj.gradient(objective, n_steps, checkpoint_every, include_init=True, soft=sb)
                    finally:
                        solver.close()
                    g = [r["dJ_dustar"], r["dJ_dz0"]]
                    if sb is not None:
                        g += list(r["dJ_dheights"])
                    ctx.save_for_backward(torch.tensor(g, dtype=params.dtype, device=params.device))
                    return torch.tensor(r["J"], dtype=params.dtype, device=params.device)

                @staticmethod
                def backward(ctx, gJ):
                    (g,) = ctx.saved_tensors
                    return gJ * g, None, None, None, None, None

            cls._fn = _Fn
        return cls._fn

    @classmethod
    def apply(cls, params, make_solver, objective: Objective, n_steps: int, checkpoint_every: int = 1,
              soft: SoftBuildings | None = None):
        return cls._function().apply(params, make_solver, objective, n_steps, checkpoint_every, soft)
