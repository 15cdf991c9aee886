"""Generates tests/golden/ref_kernels.npz with the reference's own kernels.

    python tests/golden/make_ref_golden.py [reference_root]

oracle/ref_kernels.py translates the reference's compute shaders
(Assets/Resources/Shaders: FvmColl, PisoColl, LES, WallFunc, Utils,
InitShaderColl) into C++ and oracle/ref_driver.cpp replays FvmSolverGpu's
dispatch sequence with them on the CPU in FP32.  Each case below is built
through the solver API alone (constructor set-up, InitFlags, Step, and the
background-flow initialisation), so the same function drives the oracle and
the CUDA library in the tests.  The fixture holds the velocity
(velFieldLastTime) and pressure of every case after its steps, bit for bit
as the reference's kernels produce them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from unitywindsimulation_b200 import _lib, cases  # noqa: E402

FIXTURE = os.path.join(HERE, "ref_kernels.npz")
STEPS = 3
NESTED_POS = (1.0, 2.0, 0.5)
NESTED_POS_BG = (0.0, 2.5, 0.0)
NESTED_ROT_DEG = 30.0


def case_config(piso=True, les=True, log=True, compat=0, normalise=False, seed=0, nx=20, ny=10, nz=12):
    """Seeded 20 x 10 x 12 case with two buildings that the reference's own
    set-up can express: log inflow with the constants FvmSolverGpu hard-codes
    (kappa 0.4, z0 1 m, href 10 m, FvmSolverGpu.cs:817-819) or a constant
    inflow; optionally every pressure boundary zero-gradient, which turns on
    the pressure normalisation (FvmSolverGpu.cs:1425-1436)."""
    c = cases.small_case(nx, ny, nz, piso=piso, les=les, seed=seed, nv=8, np_=12, inflow_log=log, compat=compat)
    cfg = c.cfg
    if log:
        cfg.inflow_ustar = 0.0
        cfg.inflow_kappa, cfg.inflow_z0, cfg.inflow_href = 0.4, 1.0, 10.0
        cfg.wind_speed = 3.0
        ustar = 0.4 * 3.0 / np.log((10.0 + 1.0) / 1.0)
        cfg.dt = cases.cfl_dt(float(cases.log_profile((ny - 0.5) * cfg.dx, ustar, 1.0, 0.4)), cfg.dx)
    if normalise:
        for f in range(6):
            cfg.pres_bc[f] = _lib.BND_ZERO_GRAD
    return cfg, c.flags


CASES = {
    "les_simple_log": dict(piso=False, les=True, log=True, seed=0),
    "les_piso_log": dict(piso=True, les=True, log=True, seed=1),
    "laminar_simple_const_normalised": dict(piso=False, les=False, log=False, normalise=True, seed=2),
    "les_piso_rfloat": dict(piso=True, les=True, log=True, seed=3, compat=_lib.COMPAT_RFLOAT_FACE_EDDY_VIS),
}
NESTED_BG = "laminar_simple_const_normalised"


def run_case(make_solver, name):
    """make_solver(cfg) -> solver with InitFlags/Step/get_field.  Returns the
    solver after the case's steps."""
    cfg, flags = case_config(**CASES[name])
    s = make_solver(cfg)
    s.InitFlags(flags)
    s.Step(STEPS)
    return s


def run_nested(make_solver, bg):
    """Foreground 16 x 8 x 12 (dx 0.25) initialised from `bg` rotated by 30
    degrees.  The background's velField and velFieldLastTime textures are
    made equal first: the reference samples whichever of the two the
    controller captured (FvmSolverController.cs:201), the newest level or
    the one before it depending on how many steps have run since."""
    bg.set_field(_lib.FIELD_VEL, np.asarray(bg.get_field(_lib.FIELD_VEL_LAST_TIME), dtype=np.float32))
    cfg = cases.default_config(nx=16, ny=8, nz=12, dx=0.25, dt=0.02, mu=1e-3, inflow_type=_lib.INFLOW_CONSTANT,
                               wind_speed=2.0, vel_iters=5, pres_iters=8)
    s = make_solver(cfg)
    s.InitVelPresFieldsFromBackGroundFlow(bg, NESTED_POS, NESTED_POS_BG, NESTED_ROT_DEG)
    return s


def outputs(s):
    u = np.asarray(s.get_field(_lib.FIELD_VEL_LAST_TIME), dtype=np.float32)
    p = np.asarray(s.get_field(_lib.FIELD_PRES), dtype=np.float32)
    return u, p


def all_outputs(make_solver):
    out = {}
    for name in CASES:
        s = run_case(make_solver, name)
        out[name + "_u"], out[name + "_p"] = outputs(s)
        if name == NESTED_BG:
            n = run_nested(make_solver, s)
            out["nested_u"], out["nested_p"] = outputs(n)
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WINDFVM_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_ref_golden.py <reference checkout root> (or set WINDFVM_REFERENCE_ROOT)")
    from oracle.binding import RefSolver, build_ref
    build_ref(root)
    out = all_outputs(RefSolver)
    np.savez_compressed(FIXTURE, **out)
    print("wrote", FIXTURE, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
