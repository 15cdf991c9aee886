"""Generates tests/golden/urban_block_trajectory.npz: the FP32 oracle (bit-
identical to the reference's kernels step by step) run from the urban-block
set-up state (256 x 96(up) x 192 cells, seeded buildings and inlet, PISO +
LES, nV=50 nP=40 nC=2) until max|u| passes 20 x its initial value, with
(max |u|, mean 0.5|u|^2, max |p|) over fluid cells after every step.  About
20 minutes on 8 host cores.

    python tests/golden/make_trajectory.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIXTURE = os.path.join(HERE, "urban_block_trajectory.npz")
MAX_STEPS = 500
BLOWUP = 20.0


def main():
    from oracle.trajectory import STAT_NAMES, run
    from unitywindsimulation_b200 import cases

    case = cases.urban_block()
    rows, status, u0 = run(case, "oracle32", MAX_STEPS, blowup=BLOWUP, log=sys.stdout)
    np.savez_compressed(FIXTURE, rows=rows, status=status, u0=u0, solver="oracle32", workload=case.name,
                        stat_names=np.array(STAT_NAMES), blowup=BLOWUP)
    print(FIXTURE, len(rows), status)


if __name__ == "__main__":
    main()
