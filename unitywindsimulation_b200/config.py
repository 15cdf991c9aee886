"""Solver configuration: the ``wf_config`` struct and its defaults.

``default_config()`` mirrors ``wf_config_default`` (FluidSimConfig.cs:113-178
defaults + the canonical urban boundary set of the reference's
AijBuilding0.asset) so configurations can be built without loading the CUDA
library.
"""
from __future__ import annotations

import ctypes

from ._lib import (BND_FIXED_VALUE, BND_SYMMETRY, BND_ZERO_GRAD, FACE_X0, FACE_XN, FACE_Y0, FACE_YN, FACE_Z0,
                   FACE_ZN, INFLOW_CONSTANT, SOLVER_SIMPLE, TURB_NONE, WfConfig)


def default_config(**overrides) -> WfConfig:
    c = WfConfig()
    c.struct_size = ctypes.sizeof(WfConfig)
    c.nx, c.ny, c.nz = 100, 50, 100
    c.dx = 0.1
    c.dt = 0.1
    c.mu = 0.005
    c.den = 1.0
    vel = {FACE_X0: BND_FIXED_VALUE, FACE_XN: BND_ZERO_GRAD, FACE_Y0: BND_FIXED_VALUE, FACE_YN: BND_SYMMETRY,
           FACE_Z0: BND_SYMMETRY, FACE_ZN: BND_SYMMETRY}
    pres = {FACE_X0: BND_ZERO_GRAD, FACE_XN: BND_FIXED_VALUE, FACE_Y0: BND_ZERO_GRAD, FACE_YN: BND_SYMMETRY,
            FACE_Z0: BND_SYMMETRY, FACE_ZN: BND_SYMMETRY}
    for f in range(6):
        c.vel_bc[f] = vel[f]
        c.pres_bc[f] = pres[f]
    c.solver_type = SOLVER_SIMPLE
    c.piso_correctors = 2
    c.turbulence = TURB_NONE
    c.cs = 0.15
    c.vel_iters = 50
    c.pres_iters = 400
    c.inflow_type = INFLOW_CONSTANT
    c.wind_speed = 10.0
    c.inflow_ustar = 0.0
    c.inflow_z0 = 1.0
    c.inflow_kappa = 0.4
    c.inflow_href = 10.0
    c.calc_residual = 0
    c.vel_res_interval = 10
    c.pres_res_interval = 20
    c.vel_tol = 1e-15
    c.pres_tol = 1e-3
    c.compat_flags = 0
    c.check_finite = 0
    c.use_graph = 1
    return apply(c, **overrides)


def apply(c: WfConfig, **overrides) -> WfConfig:
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise KeyError(f"wf_config has no field {k!r}")
        cur = getattr(c, k)
        if hasattr(cur, "__len__"):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(c, k, v)
    return c
