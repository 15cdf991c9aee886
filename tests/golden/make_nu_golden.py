"""Generates tests/golden/nonuniform_ref.npz with the reference's own
non-uniform-grid kernels.

    python tests/golden/make_nu_golden.py [reference_root]

oracle/ref_kernels.py translates FvmCollNonUniform.compute and
InitShaderColl.compute into C++ and oracle/ref_driver.cpp replays the
reference's SIMPLE step on the non-uniform collocated grid (gridType
CollNonUniform) with them, in FP32 on the CPU.  Each case is built through
the solver API alone (constructor set-up, face positions, field and inlet
initialisation, InitFlags, Step), so the same function drives the reference
kernels and the CUDA library in the tests.  The fixture holds, after every
step, the new velocity (velFieldLastTime) and the pressure, and after the
last step also the face-flux texture and that step's momentum and
pressure-equation coefficients (D, b, Dp, bp) and velocity correction, bit
for bit as the reference's kernels produce them.
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

FIXTURE = os.path.join(HERE, "nonuniform_ref.npz")
STEPS = 3
CASES = {
    "const_tunnel": dict(log_inflow=False, seed=0),
    "log_urban_normalised": dict(log_inflow=True, seed=1),
    # nx = 15: the one-cell-per-thread sweeps (no four-cell quads in a row)
    "const_tunnel_odd_nx": dict(log_inflow=False, seed=2, nx=15, x_split=(7, 4)),
    # Smagorinsky LES on the non-uniform grid: wall function and LES terms
    # with the constant dx, face eddy viscosities interpolated with the mesh
    # weights in the momentum kernels (useLES)
    "log_urban_les": dict(log_inflow=True, seed=3, les=True),
    "const_tunnel_les": dict(log_inflow=False, seed=4, les=True),
}
# Fields recorded after each step, and after the last one: (name, field id).
STEP_FIELDS = (("vel", _lib.FIELD_VEL_LAST_TIME), ("pres", _lib.FIELD_PRES))
LAST_FIELDS = (("D", _lib.FIELD_D), ("b", _lib.FIELD_B), ("Dp", _lib.FIELD_DP), ("bp", _lib.FIELD_BP),
               ("vel_correct", _lib.FIELD_VEL_CORRECT))


def make_case(name):
    return cases.small_nonuniform_case(**CASES[name])


def run_case(make_solver, name, record):
    """make_solver(cfg) -> solver with the FvmSolver API plus get_field and
    get_face_flux.  record(step, key, array) receives the fields after each
    step and the initial state (step 0: vel, pres, inlet plane)."""
    case = make_case(name)
    s = make_solver(case.cfg)
    cases.apply_case(s, case)
    record(0, "vel", np.asarray(s.get_field(_lib.FIELD_VEL_LAST_TIME), dtype=np.float32))
    record(0, "pres", np.asarray(s.get_field(_lib.FIELD_PRES), dtype=np.float32))
    record(0, "inlet", np.asarray(s.get_field(_lib.FIELD_BND_X0), dtype=np.float32))
    for k in range(1, STEPS + 1):
        s.Step(1)
        for key, fid in STEP_FIELDS + (LAST_FIELDS if k == STEPS else ()):
            record(k, key, np.asarray(s.get_field(fid), dtype=np.float32))
        if k == STEPS:
            record(k, "flux", np.asarray(s.get_face_flux(), dtype=np.float32))
    return s


def main(reference_root):
    from oracle import binding

    binding.build_ref(reference_root)
    out = {}
    for name in CASES:
        def rec(step, key, a, name=name):
            out[f"{name}/{step}/{key}"] = a
        run_case(lambda cfg: binding.RefSolver(cfg), name, rec)
    np.savez_compressed(FIXTURE, **out)
    print(FIXTURE, len(out), "arrays")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WINDFVM_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_nu_golden.py <reference checkout root> (or set WINDFVM_REFERENCE_ROOT)")
    main(root)
