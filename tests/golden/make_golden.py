"""Generates the golden fixtures of tests/golden/ with the FP64 oracle.

    python tests/golden/make_golden.py

The reference ships no test data for this path, so these fixtures pin the
oracle (FP64 instance) and the CUDA library against regressions; they are
not outputs of the reference itself.

aij_building.json: the reference's own validation case
(Assets/Code/Config/AijBuilding0.asset: 80 x 40 x 40 cells of 1 m, dt 0.04,
SIMPLE, Smagorinsky 0.18, log inflow at 10 m/s with kappa 0.4, z0 1 m,
href 10 m, the box x 20..24, y 0..8, z 18..22) with the iteration counts cut
to 20 momentum and 60 pressure sweeps and 2 steps, sampled along the lines of
the reference's OpenFOAM comparison (OpenFOAMSetting/system/sampleDict:
centre line y = 19.5 m and near-ground lines y = 4.5, 1.5, 0.5 m at z = 19.5 m,
vertical lines at x = 25.5, 30.5, 40.5 m) plus per-z-plane sums.

small_piso.npz: full velocity and pressure of a 24 x 12 x 16 PISO + LES case
(cases.small_case(seed=0)) after 2 steps.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from unitywindsimulation_b200 import cases  # noqa: E402

AIJ_STEPS = 2
SMALL_STEPS = 2


def aij_case():
    return cases.aij_building(nv=20, np_=60, steps=AIJ_STEPS)


def small_case():
    return cases.small_case(seed=0)


def sample_aij(u, p):
    """u: (3, nz, ny, nx), p: (nz, ny, nx) -> dict of sample lines (cell
    centres of the sampleDict lines) and per-plane sums."""
    out = {}
    zc = 19  # z = 19.5 m
    for name, y in (("Ux_Centerline", 19), ("Ux_Ground_y4_Centerline", 4), ("Ux_Ground_y1_Centerline", 1),
                    ("Ux_Ground_y0_Centerline", 0)):
        out[name] = {"u": u[:, zc, y, :].tolist(), "p": p[zc, y, :].tolist()}
    for x in (25, 30, 40):
        out[f"sampleYAxis_x{x}_zCenter"] = {"u": u[:, zc, :, x].tolist(), "p": p[zc, :, x].tolist()}
    out["plane_sums"] = {"u": u.sum(axis=(2, 3)).tolist(), "p": p.sum(axis=(1, 2)).tolist()}
    out["norms"] = {"u_l2": float(np.linalg.norm(u)), "p_l2": float(np.linalg.norm(p))}
    return out


def run_aij(solver_cls, **kw):
    c = aij_case()
    s = solver_cls(c.cfg, **kw)
    s.InitFlags(c.flags)
    s.Step(AIJ_STEPS)
    return sample_aij(np.asarray(s.GetVelField(), np.float64), np.asarray(s.GetPresField(), np.float64))


def run_small(solver_cls, **kw):
    c = small_case()
    s = solver_cls(c.cfg, **kw)
    s.InitFlags(c.flags)
    s.Step(SMALL_STEPS)
    return np.asarray(s.GetVelField(), np.float64), np.asarray(s.GetPresField(), np.float64)


def main():
    from oracle import OracleSolver
    aij = run_aij(OracleSolver, precision=64)
    with open(os.path.join(HERE, "aij_building.json"), "w") as f:
        json.dump(aij, f)
    u, p = run_small(OracleSolver, precision=64)
    np.savez_compressed(os.path.join(HERE, "small_piso.npz"), u=u.astype(np.float32), p=p.astype(np.float32),
                        u64_norm=np.linalg.norm(u), p64_norm=np.linalg.norm(p))
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
