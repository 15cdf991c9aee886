"""Generates tests/golden/adjoint_street_fd.npz: FP64 central differences of
the pedestrian-level objective on the full adjoint workload.

Workload (cases.adjoint_street): 128 x 64(up) x 96 cells of 0.5 m, 12 soft
buildings with continuous heights, PISO laminar, nV=50 nP=30 nC=2, a 200-step
window; objective = mean |u|^2 over the 32 x 32 street patch at y index 3
(1.5-2.0 m), averaged over the last 100 steps.  The FP64 oracle runs the
window from the set-up state for the base parameters and for each
parameter moved by +-1e-4: u*, z0 and the three buildings whose heights
matter most in this layout (indices in HEIGHTS).  About 30 minutes on 8
host cores.

    python tests/golden/make_adjoint_fd.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIXTURE = os.path.join(HERE, "adjoint_street_fd.npz")
FD_EPS = 1e-4
HEIGHTS = (10, 9, 2)


def objective(case, obj, n_steps, ustar, z0, heights):
    """J of the window, FP64 oracle, from the set-up state with inflow
    (u*, z0) and building heights `heights`."""
    from oracle import OracleSolver
    from unitywindsimulation_b200 import cases

    cfg = case.cfg.copy()
    cfg.inflow_ustar, cfg.inflow_z0 = ustar, z0
    c = cases.Case(case.name, cfg, case.flags, case.inlet, case.steps, case.seed, case.buildings,
                   case.soft.with_heights(heights))
    o = OracleSolver(cfg, 64)
    cases.apply_case(o, c)
    flags = o.GetFlagField()
    J = 0.0
    for n in range(n_steps):
        o.Step(1)
        if n + 1 > n_steps - obj.window:
            J += obj.evaluate(o.GetVelField(), flags) / obj.window
    o.close()
    return J


def main():
    from unitywindsimulation_b200 import cases
    from unitywindsimulation_b200.adjoint import Objective

    case = cases.adjoint_street()
    obj = Objective(**cases.ADJOINT_STREET_OBJECTIVE)
    n = case.steps
    us, z0 = case.cfg.inflow_ustar, case.cfg.inflow_z0
    h0 = case.soft.heights.copy()

    def J(u=us, z=z0, h=h0):
        t0 = time.perf_counter()
        v = objective(case, obj, n, u, z, h)
        print(f"J(u*={u:.6f}, z0={z:.6f}) = {v:.15g} ({time.perf_counter() - t0:.0f} s)", flush=True)
        return v

    J0 = J()
    fd_u = (J(u=us + FD_EPS) - J(u=us - FD_EPS)) / (2 * FD_EPS)
    fd_z = (J(z=z0 + FD_EPS) - J(z=z0 - FD_EPS)) / (2 * FD_EPS)
    fd_h = []
    for i in HEIGHTS:
        hp, hm = h0.copy(), h0.copy()
        hp[i] += FD_EPS
        hm[i] -= FD_EPS
        fd_h.append((J(h=hp) - J(h=hm)) / (2 * FD_EPS))
    np.savez_compressed(FIXTURE, J=J0, dJ_dustar=fd_u, dJ_dz0=fd_z, heights=np.array(HEIGHTS),
                        dJ_dheights=np.array(fd_h), eps=FD_EPS, steps=n, window=obj.window)
    print(FIXTURE, J0, fd_u, fd_z, fd_h)


if __name__ == "__main__":
    main()
