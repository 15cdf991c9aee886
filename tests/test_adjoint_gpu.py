"""Discrete adjoint of the step (GPU tests).

The adjoint is checked against central finite differences of the FP64
oracle, which restates the forward step independently:

* dot-product tests of one step cut after the momentum predictor, after the
  SIMPLE correction and after the PISO correctors: <ubar, du/dx . dx> from
  the oracle's differences against <J^T ubar, dx> from the adjoint, for
  random directions in the velocity, the pressure and the inlet plane;
* the gradient of the pedestrian-comfort objective over a window of steps
  with respect to the log-inflow parameters (u*, z0) and the heights of
  soft buildings, with checkpoints and recomputation, against FP64
  differences with step 1e-4.

Bound: 1e-3 relative, as for the objective gradient.
"""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from unitywindsimulation_b200.adjoint import (PHASE_FULL, PHASE_PREDICTOR, PHASE_SIMPLE, AdjointSolver,
                                              Objective, WindObjective)
from oracle import OracleSolver

pytestmark = pytest.mark.gpu

ADJ_TOL = 1e-3
FD_EPS = 1e-4


def adj_case(piso=True, seed=5, nx=24, ny=12, nz=16):
    return cases.small_case(nx, ny, nz, piso=piso, les=False, seed=seed, nv=6, np_=8)


def developed_solver(case, steps=3):
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    g.Step(steps)
    return g


def oracle_phase(case, g, u, p, phases, bnd_x0=None, drag=None):
    """One step of the FP64 oracle from state (u, p), cut after `phases`
    parts, with the GPU solver's boundary planes (X0 replaced by bnd_x0) and
    the case's drag field (replaced by drag)."""
    o = OracleSolver(case.cfg, 64)
    cases.apply_case(o, case)
    for f in range(_lib.FIELD_BND_X0, _lib.FIELD_BND_ZN + 1):
        o.set_field(f, np.asarray(g.get_field(f), dtype=np.float64))
    if bnd_x0 is not None:
        o.set_field(_lib.FIELD_BND_X0, bnd_x0)
    if drag is not None:
        o.set_field(_lib.FIELD_DRAG, drag)
    for f in (_lib.FIELD_VEL, _lib.FIELD_VEL_LAST_TIME, _lib.FIELD_VEL_LAST_ITER):
        o.set_field(f, u)
    o.set_field(_lib.FIELD_PRES, p)
    n = u.shape[1]
    o.set_field(_lib.FIELD_PRES_CORRECT, np.zeros(n))
    o.set_field(_lib.FIELD_PRES_CORRECT_LAST_ITER, np.zeros(n))
    c = case.cfg
    o.op("vel_precompute")
    o.op("vel_sweeps", c.vel_iters)
    if phases >= PHASE_SIMPLE:
        o.op("pres_precompute")
        o.op("pres_sweeps", c.pres_iters)
        o.op("apply_pres")
        o.op("apply_vel")
        o.op("zero_pres_correct")
    if phases >= PHASE_FULL and c.solver_type == _lib.SOLVER_PISO:
        for _ in range(c.piso_correctors):
            o.op("piso", c.pres_iters)
    out = o.get_field(_lib.FIELD_VEL).reshape(3, n), o.get_field(_lib.FIELD_PRES).reshape(n)
    o.close()
    return out


def drag_of(case):
    c = case.cfg
    if case.soft is None:
        return np.zeros(c.nx * c.ny * c.nz)
    return case.soft.drag(c.nx, c.ny, c.nz, np.float64).reshape(-1)


@pytest.fixture(scope="module", params=["flags", "soft"])
def setup(built, request):
    case = adj_case() if request.param == "flags" else cases.small_soft_case(seed=3)
    g = developed_solver(case)
    adj = AdjointSolver(g)
    u0, p0, _ = g.get_state()
    n = g.n_cells
    yield case, g, adj, np.asarray(u0, np.float64).reshape(3, n), np.asarray(p0, np.float64).reshape(n)
    adj.close()
    g.close()


def test_tape_matches_step(setup):
    """The recorded forward step equals the solver's own step (fast kernels)."""
    case, g, adj, u0, p0 = setup
    u1, p1 = adj.step_forward(PHASE_FULL)
    h = FvmSolverCuda(case.cfg)
    cases.apply_case(h, case)
    h.set_state(u0.astype(np.float32), p0.astype(np.float32))
    h.Step(1)
    u2, p2, _ = h.get_state()
    h.close()
    n = g.n_cells
    np.testing.assert_allclose(u1, np.asarray(u2).reshape(3, n), rtol=0, atol=1e-5 * np.abs(u2).max())
    np.testing.assert_allclose(p1, np.asarray(p2).reshape(n), rtol=0, atol=1e-5 * np.abs(p2).max() + 1e-7)


@pytest.mark.parametrize("phases", [PHASE_PREDICTOR, PHASE_SIMPLE, PHASE_FULL])
@pytest.mark.parametrize("direction", ["vel", "pres", "inlet", "drag"])
def test_step_vjp_dot_product(setup, phases, direction):
    case, g, adj, u0, p0 = setup
    n = g.n_cells
    rng = np.random.default_rng(100 + 10 * phases + len(direction))
    ubar = rng.standard_normal((3, n))
    pbar = rng.standard_normal(n)
    ui, pi, planes, dragbar = adj.step_vjp(ubar, pbar, phases)
    x0 = np.asarray(g.get_field(_lib.FIELD_BND_X0), dtype=np.float64)
    chi = drag_of(case)
    du = np.zeros_like(u0)
    dp = np.zeros_like(p0)
    dg = np.zeros_like(x0)
    dchi = np.zeros_like(chi)
    if direction == "vel":
        du = rng.standard_normal(u0.shape) * 0.5
        ad = float((ui.astype(np.float64) * du).sum())
    elif direction == "pres":
        dp = rng.standard_normal(p0.shape) * max(1e-3, np.abs(p0).max())
        ad = float((pi.astype(np.float64) * dp).sum())
    elif direction == "inlet":
        dg = rng.standard_normal(x0.shape) * 0.5
        ad = float((planes[_lib.FACE_X0].astype(np.float64) * dg.reshape(planes[0].shape)).sum())
    else:
        dchi = rng.uniform(0.0, 1.0, chi.shape) / case.cfg.dt
        ad = float((dragbar.astype(np.float64) * dchi).sum())

    def J(s):
        u, p = oracle_phase(case, g, u0 + s * du, p0 + s * dp, phases, x0 + s * dg, chi + s * dchi)
        return float((ubar * u).sum() + (pbar * p).sum())

    fd = (J(FD_EPS) - J(-FD_EPS)) / (2 * FD_EPS)
    assert abs(fd - ad) <= ADJ_TOL * abs(fd), f"phase {phases} {direction}: adjoint {ad} vs FD {fd}"


def _oracle_objective(case, obj, n_steps, ustar, z0, heights=None):
    cfg = case.cfg.copy()
    cfg.inflow_ustar, cfg.inflow_z0 = ustar, z0
    o = OracleSolver(cfg, 64)
    c = case if heights is None else cases.Case(case.name, cfg, case.flags, case.inlet, case.steps, case.seed,
                                                case.buildings, case.soft.with_heights(heights))
    cases.apply_case(o, c)
    flags = o.GetFlagField()
    J = 0.0
    for n in range(n_steps):
        o.Step(1)
        if n + 1 > n_steps - obj.window:
            J += obj.evaluate(o.GetVelField(), flags) / obj.window
    o.close()
    return J


@pytest.mark.parametrize("piso", [True, False])
def test_inflow_gradient_vs_fd(built, piso):
    case = adj_case(piso=piso, seed=6)
    obj = Objective(x0=6, x1=22, z0=2, z1=14, y=1, window=3)
    n_steps = 6
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    with AdjointSolver(g) as adj:
        r = adj.gradient(obj, n_steps, checkpoint_every=2, include_init=True)
    g.close()
    us, z0 = case.cfg.inflow_ustar, case.cfg.inflow_z0
    J0 = _oracle_objective(case, obj, n_steps, us, z0)
    assert abs(r["J"] - J0) <= 1e-4 * abs(J0)  # FP32 forward against FP64
    fu = (_oracle_objective(case, obj, n_steps, us + FD_EPS, z0)
          - _oracle_objective(case, obj, n_steps, us - FD_EPS, z0)) / (2 * FD_EPS)
    fz = (_oracle_objective(case, obj, n_steps, us, z0 + FD_EPS)
          - _oracle_objective(case, obj, n_steps, us, z0 - FD_EPS)) / (2 * FD_EPS)
    assert abs(r["dJ_dustar"] - fu) <= ADJ_TOL * abs(fu), (r, fu)
    assert abs(r["dJ_dz0"] - fz) <= ADJ_TOL * abs(fz), (r, fz)


@pytest.mark.parametrize("piso", [True, False])
def test_soft_height_gradient_vs_fd(built, piso):
    case = cases.small_soft_case(piso=piso, seed=4)
    obj = Objective(x0=4, x1=20, z0=2, z1=14, y=1, window=3)
    n_steps = 6
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    with AdjointSolver(g) as adj:
        r = adj.gradient(obj, n_steps, checkpoint_every=2, soft=case.soft)
    g.close()
    us, z0 = case.cfg.inflow_ustar, case.cfg.inflow_z0
    h0 = case.soft.heights
    for i in range(h0.size):
        hp, hm = h0.copy(), h0.copy()
        hp[i] += FD_EPS
        hm[i] -= FD_EPS
        fd = (_oracle_objective(case, obj, n_steps, us, z0, hp)
              - _oracle_objective(case, obj, n_steps, us, z0, hm)) / (2 * FD_EPS)
        ad = r["dJ_dheights"][i]
        assert abs(ad - fd) <= ADJ_TOL * abs(fd), (i, ad, fd)
    fu = (_oracle_objective(case, obj, n_steps, us + FD_EPS, z0, h0)
          - _oracle_objective(case, obj, n_steps, us - FD_EPS, z0, h0)) / (2 * FD_EPS)
    assert abs(r["dJ_dustar"] - fu) <= ADJ_TOL * abs(fu), (r["dJ_dustar"], fu)


def test_checkpoint_interval_does_not_change_gradient(built):
    case = adj_case(seed=7)
    obj = Objective(x0=6, x1=22, z0=2, z1=14, y=1, window=2)
    out = []
    for every in (1, 3, 5):
        g = FvmSolverCuda(case.cfg)
        cases.apply_case(g, case)
        with AdjointSolver(g) as adj:
            out.append(adj.gradient(obj, 5, checkpoint_every=every))
        g.close()
    # recomputed states come from the one-sweep kernels, stored ones from the
    # blocked sweeps of the solver: equal up to FP32 rounding
    for r in out[1:]:
        assert r["J"] == pytest.approx(out[0]["J"], rel=1e-12)
        assert abs(r["dJ_dustar"] - out[0]["dJ_dustar"]) <= 1e-5 * abs(out[0]["dJ_dustar"])
        assert abs(r["dJ_dz0"] - out[0]["dJ_dz0"]) <= 1e-5 * abs(out[0]["dJ_dz0"])


def test_tape_cap_does_not_change_gradient(built):
    """Tape caps below the window: the taped tail is shorter, and segments
    longer than the cap are either shortened or reversed in sub-blocks from
    stored segment states; the gradient is the same."""
    case = cases.small_soft_case(seed=9)
    obj = Objective(x0=4, x1=20, z0=2, z1=14, y=1, window=3)
    out = []
    for cap, shorten in ((0, True), (2, True), (1, True), (2, False), (1, False)):
        g = FvmSolverCuda(case.cfg)
        cases.apply_case(g, case)
        with AdjointSolver(g) as adj:
            adj.set_max_tapes(cap)
            adj.set_segment_policy(shorten)
            out.append(adj.gradient(obj, 7, checkpoint_every=5, soft=case.soft))
        g.close()
    for r in out[1:]:
        assert r["J"] == pytest.approx(out[0]["J"], rel=1e-12)
        assert r["dJ_dustar"] == pytest.approx(out[0]["dJ_dustar"], rel=1e-5)
        np.testing.assert_allclose(r["dJ_dheights"], out[0]["dJ_dheights"], rtol=1e-4,
                                   atol=1e-6 * np.abs(out[0]["dJ_dheights"]).max())


def test_autograd_function(built):
    torch = pytest.importorskip("torch")
    case = cases.small_soft_case(seed=8)
    obj = Objective(x0=4, x1=20, z0=2, z1=14, y=1, window=2)

    def make(us, z0, soft):
        cfg = case.cfg.copy()
        cfg.inflow_ustar, cfg.inflow_z0 = us, z0
        c = cases.Case(case.name, cfg, case.flags, None, 1, case.seed, [], soft)
        s = FvmSolverCuda(cfg)
        cases.apply_case(s, c)
        return s

    p0 = [case.cfg.inflow_ustar, case.cfg.inflow_z0] + list(case.soft.heights)
    params = torch.tensor(p0, dtype=torch.float64, requires_grad=True)
    J = WindObjective.apply(params, make, obj, 4, 2, case.soft)
    J.backward()
    s = make(case.cfg.inflow_ustar, case.cfg.inflow_z0, case.soft)
    with AdjointSolver(s) as adj:
        r = adj.gradient(obj, 4, 2, soft=case.soft)
    s.close()
    # the adjoint scatters with float atomics: equal up to summation order
    assert J.item() == pytest.approx(r["J"], rel=1e-9)
    ref = [r["dJ_dustar"], r["dJ_dz0"]] + list(r["dJ_dheights"])
    np.testing.assert_allclose(params.grad.numpy(), ref, rtol=1e-5)


def test_unsupported_configurations(built):
    les = cases.small_case(16, 8, 12, les=True, seed=1)
    g = FvmSolverCuda(les.cfg)
    with pytest.raises(_lib.WindFvmError) as e:
        AdjointSolver(g)
    assert e.value.status == _lib.WF_ERR_UNSUPPORTED
    g.close()
