"""Long runs of a workload on the host cores, one statistics row per step.

Test infrastructure (like the rest of oracle/): it runs the FP32 or FP64
oracle, or the reference's own kernels (oracle/_ref/, where built), from the
workload's set-up state and records after every step the largest velocity
magnitude over fluid cells, the mean kinetic energy 0.5|u|^2 over fluid cells
and the largest |p|.  A run stops at the first non-finite value or once
max|u| passes `blowup` times its initial value.  The rows say where the
reference's arithmetic (the FP32 oracle is bit-identical to the reference's
kernels step by step) leaves the bounded range; the GPU tests compare the
CUDA library's rows with them.

    python -m oracle.trajectory --workload urban_block --solver oracle32 --steps 500 --out traj.npz
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

STAT_NAMES = ("max_u", "mean_ke", "max_p")


def step_stats(vel_soa: np.ndarray, pres: np.ndarray, fluid: np.ndarray) -> np.ndarray:
    """(max |u|, mean 0.5|u|^2, max |p|) over the fluid cells, in FP64."""
    u = np.asarray(vel_soa, dtype=np.float64).reshape(3, -1)[:, fluid]
    mag2 = (u * u).sum(axis=0)
    p = np.asarray(pres, dtype=np.float64).reshape(-1)[fluid]
    return np.array([np.sqrt(mag2.max()), 0.5 * mag2.mean(), np.abs(p).max()])


def save_state(s, path):
    """Every field the reference's step reads (velocity textures, pressure,
    eddy and face viscosities, boundary planes), FP32."""
    from oracle.binding import REF_STATE_FIELDS
    np.savez_compressed(path, **{str(f): np.asarray(s.get_field(f), dtype=np.float32) for f in REF_STATE_FIELDS})


def load_state(s, path):
    d = np.load(path)
    for k in d.files:
        s.set_field(int(k), np.asarray(d[k], dtype=np.float64))


def make_solver(case, which: str, threads: int):
    """The workload's set-up state in the chosen host solver."""
    from oracle import OracleSolver
    from oracle.binding import RefSolver, ref_available
    from unitywindsimulation_b200 import cases

    prec = 64 if which == "oracle64" else 32
    o = OracleSolver(case.cfg, prec, threads=threads)
    cases.apply_case(o, case)
    if which != "reference":
        return o
    if not ref_available():
        raise RuntimeError("the reference's kernels are not built (make -C oracle ref REFERENCE_ROOT=...)")
    r = RefSolver(case.cfg, construct=False)
    r.copy_state_from(o)
    o.close()
    return r


def run(case, which: str, steps: int, threads: int = 0, blowup: float = 20.0, log=None, start=None,
        save_at=None):
    """Steps the workload up to `steps` times; returns (rows, status, u0)
    where rows[k] are the statistics after step k+1 and status is "bounded",
    "blowup" or "nonfinite".  `start` = the path of a saved state that
    replaces the set-up state (load_state); `save_at` = (step, path) writes the
    state after that step (every field a step reads) to an .npz file."""
    s = make_solver(case, which, threads or (os.cpu_count() or 1))
    if start is not None:
        load_state(s, start)
    fluid = np.asarray(case.flags).reshape(-1) == 0
    u0 = step_stats(s.GetVelField(), s.GetPresField(), fluid)[0]
    rows, status = [], "bounded"
    for k in range(steps):
        t0 = time.perf_counter()
        s.Step(1)
        st = step_stats(s.GetVelField(), s.GetPresField(), fluid)
        rows.append(st)
        if save_at is not None and k + 1 == save_at[0]:
            save_state(s, save_at[1])
        if log:
            print(f"{which} step {k + 1}: max|u| {st[0]:.4g} mean ke {st[1]:.4g} max|p| {st[2]:.4g} "
                  f"({time.perf_counter() - t0:.1f} s)", file=log, flush=True)
        if not np.all(np.isfinite(st)):
            status = "nonfinite"
            break
        if st[0] > blowup * u0:
            status = "blowup"
            break
    s.close()
    return np.array(rows), status, u0


def main(argv=None):
    from unitywindsimulation_b200 import cases

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="urban_block", choices=sorted(cases.WORKLOADS))
    ap.add_argument("--solver", default="oracle32", choices=["oracle32", "oracle64", "reference"])
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--blowup", type=float, default=20.0)
    ap.add_argument("--out", required=True)
    ap.add_argument("--start", help="state file (save_state) to start from instead of the set-up state")
    ap.add_argument("--save-step", type=int, help="write the state after this step to --save-path")
    ap.add_argument("--save-path")
    a = ap.parse_args(argv)
    case = cases.WORKLOADS[a.workload]()
    save_at = (a.save_step, a.save_path) if a.save_step else None
    rows, status, u0 = run(case, a.solver, a.steps, a.threads, a.blowup, log=sys.stdout, start=a.start,
                           save_at=save_at)
    np.savez_compressed(a.out, rows=rows, status=status, u0=u0, solver=a.solver, workload=a.workload,
                        stat_names=np.array(STAT_NAMES))
    print(f"{a.solver} {a.workload}: {len(rows)} steps, {status}")


if __name__ == "__main__":
    main()
