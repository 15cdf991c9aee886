#!/usr/bin/env python
"""Throughput benchmark of the plain PISO + LES time step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl windfvm|reference]

A step is one complete time step (wall function, LES, momentum predictor with
50 Jacobi sweeps, Rhie-Chow pressure correction with 40 sweeps, 2 PISO
correctors with 40 sweeps each) of the urban-block workload: 256 x 96(up) x
192 cells of 0.5 m, 48 seeded buildings, log-law inflow u* = 0.6 m/s, z0 =
0.3 m with a 5 % inlet perturbation (synthetic, seeded; the reference ships
no dataset).  The metric is Mcell-steps/s = cells x steps / s / 1e6.

Multi-GPU: replicas only -- every rank steps its own copy of the workload,
there is no data-path collective; value = all ranks' cell-steps / max rank
time.  Rank 0 prints one JSON line.

--impl reference times the reference's algorithm on the host cores: its
compute shaders, translated to C++ and dispatched in FvmSolverGpu's order
(oracle/_ref/, built where the reference checkout is present), or, where those
are not built, its CPU restatement (oracle/, FP32); both run OpenMP over all
cores.  The C# host under Unity/D3D cannot run on this machine.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s"
B_ALG_FIXED = 287  # compulsory bytes per cell-step of the non-iterative kernels
# Wall-clock bound of the reference arm (warm-up and timed steps together):
# at 9-16 s per urban-block step on 16 host cores, 25 steps fit.
REFERENCE_BUDGET_S = 900.0
# Timed steps of each form in the batched sections.
BATCH_STEPS = 30


def b_alg(nv: int, np_: int, nc: int) -> int:
    """Algorithmic bytes per cell-step of the reference kernel sequence (each
    kernel reads each input once and writes each output once; vector 12 B,
    scalar 4 B, flag 1 B)."""
    return B_ALG_FIXED + 77 * nv + 29 * np_ + nc * (123 + 33 * np_)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="windfvm", choices=["windfvm", "reference"])
    ap.add_argument("--workload", default="urban_block")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-nonuniform", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=3)
    ap.add_argument("--cpu-table", action="store_true",
                    help="print the host-core baselines of every workload (no GPU) and exit")
    ap.add_argument("--kernels", action="store_true",
                    help="step the workload --steps times and time its two Jacobi kernels, nothing else "
                         "(the target program of an ncu capture); prints one JSON line")
    ap.add_argument("--adjoint", action="store_true",
                    help="with --kernels: also run the objective gradient over --steps steps")
    ap.add_argument("--vel-k", type=int, default=0,
                    help="with --kernels: momentum sweeps per pass (1 or 2; 0: the library's default)")
    return ap.parse_args()


def dist_env():
    from unitywindsimulation_b200.replicas import env_ranks
    return env_ranks()


def make_case(name: str):
    from unitywindsimulation_b200 import cases
    return cases.WORKLOADS[name]()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(kernel: str):
    """DRAM bytes per cell of one launch of `kernel`, from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)
        return d[kernel]
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), p[5], p[6], p[7], p[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = []
        for i, name in enumerate(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]):
            if any(r[2 + i].lower() == "active" for r in rows):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def host_state(case):
    """The workload's set-up state on the host cores, ready to step: the
    reference's own kernels where they are built (oracle/_ref/: its compute
    shaders translated to C++, dispatched in FvmSolverGpu's order), kind
    "reference", else the FP32 oracle, kind "port".  The state (flags, inflow
    plane, initial fields) is set up by the oracle in both cases: the
    workload's friction-velocity inflow and perturbed inlet plane have no
    set-up kernel in the reference."""
    from oracle import OracleSolver
    from oracle.binding import RefSolver, ref_available
    cores = os.cpu_count() or 1
    o = OracleSolver(case.cfg, 32, threads=cores)
    o.InitFlags(case.flags)
    if case.inlet is not None:
        o.set_inflow_plane(case.inlet)
    if ref_available():
        s = RefSolver(case.cfg, construct=False)
        s.copy_state_from(o)
        o.close()
        return s, cores, "reference", "the reference's own kernels (FvmColl/PisoColl/LES/WallFunc compute " \
                                      "shaders compiled as C++, FP32, OpenMP over z)"
    return o, cores, "port", "the FP32 oracle (C++ restatement, OpenMP over z)"


def host_step_sampler(case, max_steps: int, budget_s: float):
    """Times whole steps of the workload on all host cores until `max_steps`
    steps or `budget_s` seconds (at least one step), from the state of
    host_state()."""
    s, cores, kind, what = host_state(case)
    done, t0 = 0, time.perf_counter()
    while done < max(1, max_steps):
        s.Step(1)
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    s.close()
    return case.n_cells * done / dt / 1e6, dt, done, cores, kind, what


def _host_rate(make, cases_, max_steps: int, budget_s: float):
    """Mcell-steps/s of whole steps over a list of cases on the host cores
    (each case stepped until max_steps or its share of the budget)."""
    cells_steps, secs = 0, 0.0
    for c in cases_:
        s = make(c)
        done, t0 = 0, time.perf_counter()
        while done < max_steps:
            s.Step(1)
            done += 1
            if time.perf_counter() - t0 >= budget_s / len(cases_):
                break
        secs += time.perf_counter() - t0
        cells_steps += c.n_cells * done
        s.close()
    return cells_steps / secs / 1e6


def cpu_table(max_steps: int = 2, budget_s: float = 20.0):
    """The CPU baselines of every workload on the host cores: the reference's
    own kernels (FP32, where oracle/_ref/ is built) and the oracle in FP32 and
    FP64.  The reference kernels take the oracle's set-up state; they have no
    drag field, so the soft-mask workloads run without it there."""
    from oracle import OracleSolver
    from oracle.binding import RefSolver, ref_available
    from unitywindsimulation_b200 import cases

    cores = os.cpu_count() or 1
    work = {
        "cfg1 plain_cube": [cases.plain_cube()],
        "cfg2 urban_block": [cases.urban_block()],
        "cfg3 batch_directions (16 cases)": cases.batch_directions(),
        "cfg4 adjoint_street (forward)": [cases.adjoint_street()],
        "cfg5 adjoint_batch (one direction)": cases.adjoint_batch()[:1],
    }

    def oracle(prec):
        def make(c):
            o = OracleSolver(c.cfg, prec, threads=cores)
            cases.apply_case(o, c)
            return o
        return make

    def reference(c):
        o = OracleSolver(c.cfg, 32, threads=cores)
        cases.apply_case(o, c)
        r = RefSolver(c.cfg, construct=False)
        r.copy_state_from(o)
        o.close()
        return r

    rows = {}
    for name, cs in work.items():
        row = {"cells": sum(c.n_cells for c in cs)}
        if ref_available():
            row["reference_kernels_f32"] = _host_rate(reference, cs, max_steps, budget_s)
        row["oracle_f32"] = _host_rate(oracle(32), cs, max_steps, budget_s)
        row["oracle_f64"] = _host_rate(oracle(64), cs, max_steps, budget_s)
        rows[name] = row
        print(json.dumps({name: row}), flush=True)
    return {"unit": METRIC, "cores": cores, "max_steps": max_steps, "budget_s": budget_s, "rows": rows}


def cpu_baseline(case, steps: int):
    """Bounded CPU sample of the same workload (about 10-30 s of host work)."""
    v, dt, done, cores, kind, what = host_step_sampler(case, steps, 10.0)
    return {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"{done} full steps of {case.name} ({case.n_cells} cells, {dt:.1f} s) with {what}, "
                      f"{cores} threads"}


def batched_section(steps: int, local: int, small: bool = False, group=None):
    """Batched form on 16 cases: the direction sweep (uneven grids 96..192 x
    48..80(up) x 96..160, wind rotated by 22.5 degree steps), or with
    small=True 16 small grids (about 0.1 M cells each).  The same cases are
    stepped one after another (plain form) and together (batched form), both
    after autotuning the blocking depths and tiles per grid size and with
    every step graph captured before timing.  The batched form is timed in
    both modes over `steps` steps: child graphs (one parent graph launch per
    step, autotuned chain width) and persistent loops (one cooperative launch
    per Jacobi loop over all cases); the faster is the batched figure.
    Device time from CUDA events.  Under torchrun the cases are dealt to the
    ranks (replicas.deal: largest first onto the least-loaded rank); each
    rank steps its share, and the whole-job rates are all cases' cell-steps
    over the slowest rank's time (barrier and max over ranks around each
    timed form)."""
    from unitywindsimulation_b200 import FvmSolverCuda, _lib, autotune, cases
    from unitywindsimulation_b200.replicas import LocalGroup, deal
    from unitywindsimulation_b200.solver import BatchSolver

    group = group or LocalGroup()
    all_cs = cases.batch_small() if small else cases.batch_directions()
    mine = deal([c.n_cells for c in all_cs], group.world)[group.rank]
    cs = [all_cs[i] for i in mine]
    solvers = [FvmSolverCuda(c.cfg, device=local) for c in cs]
    for s, c in zip(solvers, cs):
        cases.apply_case(s, c)
    cache = os.path.join(tempfile.gettempdir(), f"windfvm_autotune_rank{group.rank}.json")  # one file per process
    tuned = []
    for s in solvers:
        s.Step(1)
        tuned.append(autotune.tune(s, cache, reps=3))
    cells = sum(c.n_cells for c in all_cs)
    for s in solvers:
        s.Step(2)
        s.prepare_graphs()  # every step graph captured before timing
    group.barrier()
    plain_ms = 0.0
    for s in solvers:
        s.Step(steps)
        plain_ms += s.last_step_ms()
    plain_ms = group.max_over_ranks(plain_ms)
    b = BatchSolver(solvers)
    width = autotune.tune_batch(b, steps=2, modes=(_lib.BATCH_GRAPHS,))
    modes = {}
    for name, mode in (("graphs", _lib.BATCH_GRAPHS), ("persistent", _lib.BATCH_PERSISTENT)):
        b.set_mode(mode)
        if mode == _lib.BATCH_GRAPHS:
            b.set_width(width["width"])
        b.step(1)
        b.prepare_graphs()
        group.barrier()
        l0 = b.kernel_launches()
        b.step(steps)
        ms = group.max_over_ranks(b.last_step_ms())
        modes[name] = {"mcell_steps_s": cells * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps,
                       "gpu_launches": b.kernel_launches() - l0}
    b.close()
    for s in solvers:
        s.close()
    plain = cells * steps / (plain_ms / 1e3) / 1e6
    best = max(modes, key=lambda k: modes[k]["mcell_steps_s"])
    batched = modes[best]["mcell_steps_s"]
    name = "batch_small" if small else "batch_directions"
    return {"workload": f"{name}: {len(all_cs)} cases, {cells} cells total, grids "
                        f"{min(c.n_cells for c in all_cs)}..{max(c.n_cells for c in all_cs)} cells, nV=50 nP=30 nC=2",
            "ranks": group.world, "cases_rank0": mine if group.rank == 0 else None,
            "plain_mcell_steps_s": plain, "batched_mcell_steps_s": batched, "batched_over_plain": batched / plain,
            "batched_mode": best, "modes": modes, "steps": steps, "gpu_launches": modes[best]["gpu_launches"],
            "tuned": sorted({(t["pres_k"], t["pres_rows"], t["vel_k"], tuple(t["vel_block"])) for t in tuned}),
            "width": width}


def adjoint_section(local: int):
    """Differentiated form on the adjoint workload (128 x 64(up) x 96 cells,
    12 soft buildings, PISO, turbulence off): the objective's gradient with
    respect to (u*, z0, 12 building heights) over a 200-step window,
    checkpoints every 20 steps, objective over the last 100 steps.  Cost
    against the plain forward of the same 200 steps (device time, CUDA
    events)."""
    from unitywindsimulation_b200 import FvmSolverCuda, cases
    from unitywindsimulation_b200.adjoint import AdjointSolver, Objective

    case = cases.adjoint_street()
    steps = case.steps
    obj = Objective(**cases.ADJOINT_STREET_OBJECTIVE)
    g = FvmSolverCuda(case.cfg, device=local)
    cases.apply_case(g, case)
    g.Step(3)
    g.prepare_graphs()
    g.Step(steps)
    fwd_ms = g.last_step_ms()
    g.close()
    g = FvmSolverCuda(case.cfg, device=local)
    cases.apply_case(g, case)
    with AdjointSolver(g) as adj:
        r = adj.gradient(obj, steps, cases.ADJOINT_STREET_CHECKPOINT, soft=case.soft)
    g.close()
    return {"workload": f"adjoint_street: {case.n_cells} cells, 12 soft buildings, PISO laminar, nV=50 nP=30 nC=2, "
                        f"{steps}-step window, checkpoints every {cases.ADJOINT_STREET_CHECKPOINT}, objective over "
                        f"the last {obj.window} steps",
            "forward_ms": fwd_ms, "gradient_ms": r["ms_total"], "gradient_forward_pass_ms": r["ms_forward"],
            "adjoint_over_forward": r["ms_total"] / fwd_ms, "J": r["J"], "dJ_dustar": r["dJ_dustar"],
            "dJ_dz0": r["dJ_dz0"], "dJ_dheights": [float(x) for x in r["dJ_dheights"]]}


def adjoint_scale_section(local: int, directions: int = 1):
    """Adjoint at scale on the batched-adjoint workload (256 x 96(up) x 256
    cells, 64 soft buildings, nP = 40, 400-step window, checkpoints every
    25 steps): the gradient of `directions` of its wind directions (a bounded
    sample of the 8; each direction is an independent case), each against
    its own plain forward over the same 400 steps (device time, CUDA
    events)."""
    from unitywindsimulation_b200 import FvmSolverCuda, cases
    from unitywindsimulation_b200.adjoint import AdjointSolver, Objective

    cs = cases.adjoint_batch()[:directions]
    obj = Objective(**cases.ADJOINT_BATCH_OBJECTIVE)
    rows = []
    for c in cs:
        g = FvmSolverCuda(c.cfg, device=local)
        cases.apply_case(g, c)
        g.Step(3)
        g.prepare_graphs()
        g.Step(c.steps)
        fwd = g.last_step_ms()
        g.close()
        g = FvmSolverCuda(c.cfg, device=local)
        cases.apply_case(g, c)
        with AdjointSolver(g) as adj:
            r = adj.gradient(obj, c.steps, cases.ADJOINT_BATCH_CHECKPOINT, soft=c.soft)
        g.close()
        rows.append({"case": c.name, "forward_ms": fwd, "gradient_ms": r["ms_total"],
                     "adjoint_over_forward": r["ms_total"] / fwd, "J": r["J"]})
    c = cs[0]
    return {"workload": f"adjoint_batch: {directions} of 8 directions, {c.cfg.nx}x{c.cfg.ny}(up)x{c.cfg.nz} "
                        f"cells each, 64 soft buildings, PISO laminar with viscosity {c.cfg.mu} m^2/s, "
                        f"nV={c.cfg.vel_iters} nP={c.cfg.pres_iters} nC={c.cfg.piso_correctors}, {c.steps}-step window, "
                        f"checkpoints every {cases.ADJOINT_BATCH_CHECKPOINT}",
            "directions": rows,
            "adjoint_over_forward": sum(r["gradient_ms"] for r in rows) / sum(r["forward_ms"] for r in rows)}


def b_alg_nonuniform(nv: int, np_: int) -> int:
    """Compulsory bytes per cell-step of the non-uniform SIMPLE step
    (FvmCollNonUniform.compute; vector 12 B, scalar 4 B, flag 1 B): momentum
    pre-compute 53 (u_T, p, face fluxes, flag in; D, b out), sweep 61 per
    iteration (iterate, face fluxes, D, b, flag in; iterate out), pressure
    pre-compute 49 (u, p, D, flag in; fluxes, Dp, bp out), sweep 29 per
    iteration (p', D, Dp, bp, flag in; p' out), apply-p 13, apply-u 53,
    zero-p' 8, end copy 24."""
    return 53 + 61 * nv + 49 + 29 * np_ + 13 + 53 + 8 + 24


def nonuniform_section(local: int, steps: int, cpu: bool):
    """The non-uniform grid (gridType CollNonUniform) on the reference's own
    configuration for it, WindTunnelBoxConfig: 100 x 50(up) x 100 cells on
    the InitMeshBuffers mesh, SIMPLE, laminar, nV=800 nP=2000.  Device time
    of graph-replayed steps (CUDA events).  The fields (about 50 MB) stay in
    L2, so the algorithmic-byte rate may exceed the HBM copy peak.  With
    cpu=True one full step of the reference's own kernels (where built) on
    the host cores is timed beside it."""
    from unitywindsimulation_b200 import FvmSolverCuda, cases

    case = cases.wind_tunnel()
    c = case.cfg
    s = FvmSolverCuda(c, device=local)
    cases.apply_case(s, case)
    s.Step(1)
    s.prepare_graphs()
    l0 = s.kernel_launches()
    s.Step(steps)
    ms = s.last_step_ms() / steps
    launches = (s.kernel_launches() - l0) // steps
    s.close()
    rate = case.n_cells / (ms / 1e3) / 1e6
    b = b_alg_nonuniform(c.vel_iters, c.pres_iters)
    peak, src = measured_peaks()
    out = {"workload": f"wind_tunnel: {c.nx}x{c.ny}(up)x{c.nz} cells on the reference's non-uniform mesh "
                       f"(25 + 50 + 25 cells in x and z, ratio 1.08), SIMPLE laminar, nV={c.vel_iters} "
                       f"nP={c.pres_iters}, one box",
           "mcell_steps_s": rate, "ms_per_step": ms, "steps": steps, "gpu_launches_per_step": launches,
           "b_alg_bytes_per_cell_step": b, "alg_gbs": rate * b / 1e3, "alg_frac_of_hbm_peak": rate * b / 1e3 / peak,
           "peak_source": f"hbm_gbs of {src}", "l2": "fields resident in L2 (about 50 MB)"}
    if cpu:
        from oracle.binding import RefSolver, ref_available
        if ref_available():
            # A full step is 2800 sweeps (about a minute on 16 cores): time one
            # step with a tenth of each loop's sweeps and one without sweeps,
            # and take fixed part + 10 x the sweep part.
            def one_step(nv, np_):
                cs = cases.wind_tunnel(nv=nv, np_=np_)
                r = RefSolver(cs.cfg)
                cases.apply_case(r, cs)
                t0 = time.perf_counter()
                r.Step(1)
                dt = time.perf_counter() - t0
                r.close()
                return dt
            t_tenth = one_step(c.vel_iters // 10, c.pres_iters // 10)
            t_fixed = one_step(0, 0)
            t_full = t_fixed + 10.0 * (t_tenth - t_fixed)
            cores = os.cpu_count() or 1
            out["cpu_baseline"] = {"value": case.n_cells / t_full / 1e6, "unit": METRIC, "cores": cores,
                                   "kind": "reference",
                                   "sample": f"wind_tunnel with the reference's own FvmCollNonUniform kernels "
                                             f"compiled as C++ (FP32, {cores} threads): one step with "
                                             f"nV={c.vel_iters // 10} nP={c.pres_iters // 10} ({t_tenth:.1f} s) and "
                                             f"one without sweeps ({t_fixed:.1f} s); full step = fixed part + 10 x "
                                             f"the sweep part = {t_full:.1f} s"}
    return out


def run_reference(args):
    """The reference arm: W untimed and then K timed whole steps of the
    workload on the host cores (host_state), rank 0 only.  The line reports
    the steps and warm-up steps it ran; a run that would pass
    REFERENCE_BUDGET_S stops early and says so."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    case = make_case(args.workload)
    s, cores, kind, what = host_state(case)
    t_start = time.perf_counter()
    warm = 0
    for _ in range(args.warmup):
        s.Step(1)
        warm += 1
    done, t0 = 0, time.perf_counter()
    per_step = (t0 - t_start) / warm if warm else 0.0
    while done < max(1, args.steps):
        if done and time.perf_counter() - t_start + per_step > REFERENCE_BUDGET_S:
            break
        t1 = time.perf_counter()
        s.Step(1)
        per_step = time.perf_counter() - t1
        done += 1
    dt = time.perf_counter() - t0
    s.close()
    v = case.n_cells * done / dt / 1e6
    cut = "" if done == max(1, args.steps) else f"; stopped after {done} of {args.steps} steps at the " \
                                                f"{REFERENCE_BUDGET_S:.0f} s budget"
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": done, "warmup": warm, "ms_per_step": dt * 1e3 / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(case),
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": kind,
                         "sample": f"{warm} untimed and {done} timed full steps of {case.name} ({dt:.1f} s timed) "
                                   f"with {what}, {cores} threads; the reference's host (C# under Unity, "
                                   f"D3D dispatch) cannot run here{cut}"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(case):
    c = case.cfg
    ws = 4 * case.n_cells * (3 * 8 + 6 + 6 + 9 + 5 + 0.25)
    return {"workload": f"{case.name} {c.nx}x{c.ny}(up)x{c.nz} cells, PISO+LES, nV={c.vel_iters} "
                        f"nP={c.pres_iters} nC={c.piso_correctors}",
            "cells": case.n_cells, "grid_ref_order": [c.nx, c.ny, c.nz], "dx": c.dx, "dt": c.dt,
            "vel_iters": c.vel_iters, "pres_iters": c.pres_iters, "piso_correctors": c.piso_correctors,
            "b_alg_bytes_per_cell_step": b_alg(c.vel_iters, c.pres_iters, c.piso_correctors),
            "l2": f"inputs larger than L2: {ws / 1e6:.0f} MB of fields vs 126 MB L2",
            "parallelism": "replicas", "seed": case.seed}


def run_windfvm(args):
    import numpy as np
    import torch

    from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases

    from unitywindsimulation_b200.replicas import ReplicaGroup, whole_job_rate

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    group = ReplicaGroup("nccl")

    case = make_case(args.workload)
    cfg = case.cfg
    N = case.n_cells
    solver = FvmSolverCuda(cfg, device=local)
    cases.apply_case(solver, case)

    def barrier():
        group.barrier()
        torch.cuda.synchronize()

    max_over_ranks = group.max_over_ranks

    # ---- device-resident throughput ----
    solver.Step(args.warmup)
    solver.prepare_graphs()  # captures only; no step runs
    barrier()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    smi_index = int(vis.split(",")[local]) if vis and vis.split(",")[local].isdigit() else local
    clk = ClockSampler(smi_index)
    clk.start()
    l0 = solver.kernel_launches()
    solver.Step(args.steps)
    ms = solver.last_step_ms()
    launches = solver.kernel_launches() - l0
    clocks = clk.stop()
    barrier()
    ms_max = max_over_ranks(ms)
    value = whole_job_rate(N, args.steps, ms_max, world)
    solver.check_finite()
    # one more step, outside the timed region, traced phase by phase (no
    # graph replay) to show where a step's time goes
    phases = solver.step_phases()

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        inlet = case.inlet if case.inlet is not None else np.zeros((cfg.nz, cfg.ny, 3), np.float32)
        h_in = torch.empty(inlet.size, dtype=torch.float32, pin_memory=True)
        h_in.numpy()[:] = inlet.reshape(-1)
        h_vel = torch.empty(3 * N, dtype=torch.float32, pin_memory=True)
        h_pres = torch.empty(N, dtype=torch.float32, pin_memory=True)
        stream = torch.cuda.ExternalStream(solver.stream_ptr)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        # one untimed iteration: first use of the readback path allocates
        # its snapshot buffer and copy stream
        solver.set_inflow_plane(h_in.numpy())
        solver.Step(1)
        solver.readback_begin(h_vel.numpy(), h_pres.numpy())
        solver.readback_wait()
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            # enqueue this step's inlet upload and the step without waiting
            # for the GPU; then wait for the previous step's fields, which
            # reached the host while the GPU ran on
            solver.set_inflow_plane(h_in.numpy())
            solver.step_async(1)
            solver.readback_wait()
            solver.readback_begin(h_vel.numpy(), h_pres.numpy())
        solver.readback_wait()
        e1.record(stream)
        e1.synchronize()
        barrier()
        e_ms = max_over_ranks(e0.elapsed_time(e1))
        e2e = {"value": whole_job_rate(N, args.steps, e_ms, world), "unit": METRIC,
               "h2d_bytes_per_step": int(inlet.size * 4), "d2h_bytes_per_step": int(4 * N * 4),
               "api": "set_inflow_plane + step_async + readback_begin/readback_wait of velocity and pressure "
                      "(every step's inlet uploaded and its fields copied to pinned host buffers while the GPU "
                      "runs the next step)"}

    # ---- roofline of the dominant kernel ----
    # The four-sweep pressure wavefront (k_pres_tma4: TMA-staged tiles, 30
    # launches per step) and the momentum sweep (50 launches) share the
    # step's kernel time about equally; the roofline object is the pressure
    # wavefront, the momentum sweep's figures ride beside it.  Achieved =
    # algorithmic bytes of the launch's sweeps over its CUDA-event time;
    # traffic = DRAM bytes of one launch (ncu), below the algorithmic bytes
    # because the wavefront keeps 4 sweeps on chip.
    peak, peak_kind = measured_peaks()
    v_ms, v_bytes, v_sweeps = solver.time_kernel(_lib.KERNEL_VEL_SWEEP, reps=20, flush_l2=True)
    k_ms, k_bytes, k_sweeps = solver.time_kernel(_lib.KERNEL_PRES_SWEEP, reps=20, flush_l2=True)
    v_gbs = v_bytes / (v_ms / 1e3) / 1e9
    k_gbs = k_bytes / (k_ms / 1e3) / 1e9
    tv, tp = committed_traffic("vel_sweep"), committed_traffic("pres_sweep")
    roofline = {"bound": "hbm", "achieved": k_gbs, "peak": peak, "unit": "GB/s", "frac": k_gbs / peak,
                "traffic": (tp * N) if tp is not None else None,
                "kernel": "k_pres_tma4: pressure Jacobi wavefront, 4 sweeps per launch, tiles staged by TMA "
                          "(cp.async.bulk.tensor onto mbarriers)", "ms_per_launch": k_ms,
                "sweeps_per_launch": k_sweeps, "alg_bytes_per_launch": k_bytes,
                "peak_source": f"hbm_gbs of {peak_kind}"}
    vel_kernel = {"kernel": "momentum Jacobi sweep (four cells per thread)", "ms_per_launch": v_ms,
                  "sweeps_per_launch": v_sweeps, "alg_bytes_per_launch": v_bytes, "achieved_gbs": v_gbs,
                  "frac": v_gbs / peak, "traffic": (tv * N) if tv is not None else None}
    step_gbs = value / world * b_alg(cfg.vel_iters, cfg.pres_iters, cfg.piso_correctors) / 1e3

    solver.close()
    batched = batched_small = None
    if not args.no_batched:
        # the independent cases are dealt to the ranks (replicas.deal)
        batched = batched_section(BATCH_STEPS, local, group=group)
        batched_small = batched_section(BATCH_STEPS, local, small=True, group=group)

    adjoint = adjoint_scale = None
    if world == 1 and not args.no_adjoint:
        adjoint = adjoint_section(local)
        adjoint_scale = adjoint_scale_section(local)

    nonuniform = None
    if world == 1 and not args.no_nonuniform:
        nonuniform = nonuniform_section(local, 3, cpu=rank == 0 and not args.no_cpu_baseline)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case, args.cpu_sample_steps)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(case),
            "e2e": e2e, "gpu_launches": launches * world, "clocks": clocks, "roofline": roofline,
            "cpu_baseline": cpu,
            "step_alg_gbs": step_gbs, "step_alg_frac": step_gbs / peak,
            "step_phases_ms": phases,
            "vel_sweep_kernel": vel_kernel,
            "batched": batched,
            "batched_small_cases": batched_small,
            "adjoint": adjoint,
            "adjoint_scale": adjoint_scale,
            "nonuniform": nonuniform,
        }
        print(json.dumps(line), flush=True)
    group.close()
    return 0


def run_kernels(args):
    """A short run of the workload: --steps graph-replayed steps, then the
    two Jacobi kernels timed alone (CUDA events, cold L2), optionally the
    objective gradient over --steps steps.  Meant as the program an ncu
    capture (`ncu -k regex:<kernel> -s <n> -c <m>`) runs."""
    from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
    from unitywindsimulation_b200.adjoint import AdjointSolver, Objective

    case = make_case(args.workload)
    s = FvmSolverCuda(case.cfg)
    cases.apply_case(s, case)
    if args.vel_k:
        s.set_blocking(s.get_blocking()[0], args.vel_k)
    s.Step(args.steps)
    out = {"workload": args.workload, "cells": case.n_cells, "step_ms": s.last_step_ms() / max(args.steps, 1),
           "blocking": list(s.get_blocking())}
    if case.faces is None:
        for name, k in (("pres_sweep", _lib.KERNEL_PRES_SWEEP), ("vel_sweep", _lib.KERNEL_VEL_SWEEP)):
            ms, by, sw = s.time_kernel(k, reps=2, flush_l2=True)
            out[name] = {"ms_per_launch": ms, "sweeps_per_launch": sw, "alg_gbs": by / (ms / 1e3) / 1e9}
    s.close()
    if args.adjoint:
        s = FvmSolverCuda(case.cfg)
        cases.apply_case(s, case)
        nx, nz = case.cfg.nx, case.cfg.nz
        obj = Objective(x0=nx // 4, x1=3 * nx // 4, z0=nz // 4, z1=3 * nz // 4, y=min(3, case.cfg.ny - 1), window=1)
        with AdjointSolver(s) as adj:
            r = adj.gradient(obj, args.steps, args.steps, soft=case.soft)
        out["adjoint"] = {"gradient_ms": r["ms_total"], "forward_pass_ms": r["ms_forward"], "J": r["J"]}
        s.close()
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.kernels:
        return run_kernels(args)
    if args.cpu_table:
        print(json.dumps(cpu_table()), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_windfvm(args)


if __name__ == "__main__":
    sys.exit(main())
