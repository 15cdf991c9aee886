"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests, fixtures or golden vectors for this path and its
own code cannot run here, so the oracle is pinned by closed-form answers and
physical invariants, and by the agreement of its FP32 and FP64 instances.
"""
import math

import numpy as np
import pytest

from unitywindsimulation_b200 import _lib, cases
from unitywindsimulation_b200.config import default_config
from oracle import OracleSolver, log_law_wall_func

from helpers import rel_l2


def _open_box(**kw):
    c = default_config(nx=16, ny=10, nz=12, dx=0.5, dt=0.05, mu=1.5e-5, den=1.0,
                       solver_type=_lib.SOLVER_PISO, turbulence=_lib.TURB_SMAGORINSKY, cs=0.12,
                       vel_iters=6, pres_iters=10)
    return default_config(**{**c.as_dict(), **kw}) if kw else c


def test_quiescent_box_stays_zero(built):
    """Zero inflow, no obstacles: every field stays exactly zero."""
    cfg = _open_box(inflow_type=_lib.INFLOW_CONSTANT, wind_speed=0.0)
    o = OracleSolver(cfg, 32)
    o.Step(3)
    assert np.all(o.GetVelField() == 0.0)
    assert np.all(o.GetPresField() == 0.0)


def test_free_stream_preserved(built):
    """Uniform inflow through an empty channel with slip walls stays uniform:
    no gradients, so no eddy viscosity, no pressure correction."""
    cfg = _open_box(inflow_type=_lib.INFLOW_CONSTANT, wind_speed=2.0)
    for f in (_lib.FACE_Y0, _lib.FACE_YN, _lib.FACE_Z0, _lib.FACE_ZN):
        cfg.vel_bc[f] = _lib.BND_SYMMETRY
        cfg.pres_bc[f] = _lib.BND_SYMMETRY
    for prec in (32, 64):
        o = OracleSolver(cfg, prec)
        o.Step(3)
        u = o.GetVelField()
        assert np.max(np.abs(u[0] - 2.0)) < 1e-5
        assert np.max(np.abs(u[1:])) < 1e-5
        assert np.max(np.abs(o.GetPresField())) < 1e-3


def _bisect_utau(uP, C, kappa=0.41):
    lo, hi = 1e-12, 10.0
    f = lambda t: t * math.log(C * t) - kappa * uP
    # f is increasing for t > 1/(e C); bracket above that
    lo = max(lo, 1.0 / (math.e * C))
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


@pytest.mark.parametrize("uP", [1e-3, 0.01, 0.1, 0.5, 1.0, 3.0, 8.0, 20.0])
def test_log_law_wall_function_closed_form(built, uP):
    """LogLawWallFunc (WallFunc.compute:77-123): the 10-step Newton solve of
    u_tau ln(C u_tau) = kappa u_P, C = 9.8 (dx/2) / nu, gives the eddy
    viscosity of the exact root."""
    dx, nu, den = 0.5, 1.5e-5, 1.0
    C = 9.8 * (dx / 2.0) / nu
    ut = _bisect_utau(uP, C)
    exact = max(ut * ut * den / ((uP / (dx / 2.0)) * den) - nu, 0.0)
    got64 = log_law_wall_func(uP, dx, nu, den, 64)
    got32 = log_law_wall_func(uP, dx, nu, den, 32)
    assert abs(got64 - exact) <= 1e-9 + 1e-8 * exact
    assert abs(got32 - exact) <= 1e-7 + 1e-4 * exact


def test_log_law_cutoff(built):
    assert log_law_wall_func(5e-6, 0.5, 1.5e-5, 1.0, 32) == 0.0
    assert log_law_wall_func(-2.0, 0.5, 1.5e-5, 1.0, 64) == log_law_wall_func(2.0, 0.5, 1.5e-5, 1.0, 64)


def test_smagorinsky_linear_shear(built):
    """u = (gamma y, 0, 0): nu_t = (Cs dx)^2 gamma in the interior
    (CSCalEddyVis, LES.compute:268-324)."""
    cfg = _open_box(cs=0.17)
    gamma = 0.8
    o = OracleSolver(cfg, 64)
    nz, ny, nx = o.shape
    y = (np.arange(ny) + 0.5) * cfg.dx
    u = np.zeros((3, nz, ny, nx))
    u[0] = gamma * y[None, :, None]
    o.set_field(_lib.FIELD_VEL_LAST_TIME, u)
    o.op("eddy_vis")
    nut = o.get_field(_lib.FIELD_EDDY_VIS).reshape(o.shape)
    expect = (0.17 * cfg.dx) ** 2 * gamma
    inner = nut[1:-1, 1:-1, 1:-1]
    assert np.allclose(inner, expect, rtol=1e-6, atol=0)


def test_pressure_operator_symmetric(built):
    """<A x, y> = <x, A y> for the off-diagonal pressure stencil (face
    coefficients shared by the two cells of a face).  The operator is read
    through one Jacobi sweep with a zero right-hand side: p_out = -Dp^-1 A p_in."""
    case = cases.small_case(seed=3)
    o = OracleSolver(case.cfg, 64)
    o.InitFlags(case.flags)
    o.Step(1)
    o.op("vel_precompute")
    o.op("pres_precompute")
    Dp = o.get_field(_lib.FIELD_DP)
    o.set_field(_lib.FIELD_BP, np.zeros_like(Dp))
    fluid = case.flags.reshape(-1) == 0
    rng = np.random.default_rng(0)

    def apply(x):
        o.set_field(_lib.FIELD_PRES_CORRECT_LAST_ITER, x)
        o.set_field(_lib.FIELD_PRES_CORRECT, np.zeros_like(x))
        o.op("pres_sweeps", 1)
        out = o.get_field(_lib.FIELD_PRES_CORRECT)
        return np.where(fluid, -Dp * out, 0.0)

    x = np.where(fluid, rng.standard_normal(Dp.size), 0.0)
    y = np.where(fluid, rng.standard_normal(Dp.size), 0.0)
    ax, ay = apply(x), apply(y)
    lhs, rhs = float(ax @ y), float(x @ ay)
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)


def test_velocity_correction_reduces_divergence(built):
    """SIMPLE's correction lowers the face-flux imbalance of the predicted
    velocity (CSApplyVelCorrectionDivergenceTheorem)."""
    case = cases.small_case(seed=4, np_=200)
    o = OracleSolver(case.cfg, 64)
    o.InitFlags(case.flags)
    o.Step(1)
    probe = OracleSolver(case.cfg, 64)
    probe.InitFlags(case.flags)
    o.op("wallfunc"); o.op("eddy_vis"); o.op("les_term")
    o.op("vel_precompute"); o.op("vel_sweeps", case.cfg.vel_iters)
    probe.set_field(_lib.FIELD_VEL_LAST_TIME, o.get_field(_lib.FIELD_VEL))
    before = probe.mass_imbalance()
    o.op("pres_precompute"); o.op("pres_sweeps", case.cfg.pres_iters); o.op("apply_pres"); o.op("apply_vel")
    probe.set_field(_lib.FIELD_VEL_LAST_TIME, o.get_field(_lib.FIELD_VEL))
    after = probe.mass_imbalance()
    assert after < 0.75 * before, (before, after)


@pytest.mark.parametrize("kw", [dict(piso=True, les=True), dict(piso=False, les=False),
                                dict(piso=True, les=True, compat=_lib.COMPAT_RFLOAT_FACE_EDDY_VIS)])
def test_fp32_tracks_fp64(built, kw):
    """The FP32 instance stays within 1e-5 relative L2 of FP64 over 3 steps."""
    case = cases.small_case(seed=5, **kw)
    outs = []
    for prec in (32, 64):
        o = OracleSolver(case.cfg, prec)
        o.InitFlags(case.flags)
        o.Step(3)
        outs.append((o.GetVelField(), o.GetPresField()))
    assert rel_l2(outs[0][0], outs[1][0]) < 1e-5
    assert rel_l2(outs[0][1], outs[1][1]) < 1e-5


def test_solid_cells_keep_zero_velocity(built):
    case = cases.small_case(seed=6)
    o = OracleSolver(case.cfg, 32)
    o.InitFlags(case.flags)
    o.Step(2)
    u = o.GetVelField()
    assert np.all(u[:, case.flags == 1] == 0.0)


def test_rfloat_compat_drops_y_and_z_wall_viscosity(built):
    """Q1: with the RFloat face texture only the x-normal (W face) wall
    viscosity reaches the momentum equation."""
    base = cases.small_case(seed=7)
    res = []
    for compat in (0, _lib.COMPAT_RFLOAT_FACE_EDDY_VIS):
        base.cfg.compat_flags = compat
        o = OracleSolver(base.cfg, 64)
        o.InitFlags(base.flags)
        o.Step(1)
        o.op("wallfunc"); o.op("eddy_vis"); o.op("les_term"); o.op("vel_precompute")
        res.append(o.get_field(_lib.FIELD_D))
    assert not np.allclose(res[0], res[1])


def test_init_profile_modes(built):
    """Q2: the interior log profile starts at y = j dx (zero in the bottom
    row), the inlet at (j + 1/2) dx; the compat flag aligns both."""
    case = cases.small_case(seed=8)
    o = OracleSolver(case.cfg, 64)
    u = o.GetVelField()
    assert np.all(u[0, :, 0, :] == 0.0)
    case.cfg.compat_flags = _lib.COMPAT_INIT_PROFILE_CELL_CENTRE
    o2 = OracleSolver(case.cfg, 64)
    u2 = o2.GetVelField()
    inlet = o2.get_field(_lib.FIELD_BND_X0)[0].reshape(case.cfg.nz, case.cfg.ny)
    np.testing.assert_allclose(u2[0, :, :, 0], inlet, rtol=1e-12)


def test_normalization_reads_reference_first(built):
    """Q4: CSPresNormalization subtracts the value the reference cell held
    before the dispatch from every non-solid cell, the reference cell included."""
    case = cases.small_case(seed=9)
    o = OracleSolver(case.cfg, 64)
    o.InitFlags(case.flags)
    rng = np.random.default_rng(1)
    p = rng.standard_normal(o.n_cells)
    o.set_field(_lib.FIELD_PRES, p)
    o.op("normalize")
    nz, ny, nx = o.shape
    ref = p.reshape(o.shape)[2, ny // 2, 2]
    got = o.get_field(_lib.FIELD_PRES)
    solid = case.flags.reshape(-1) == 1
    np.testing.assert_allclose(got[~solid], p[~solid] - ref, rtol=0, atol=1e-14)
    np.testing.assert_array_equal(got[solid], p[solid])


def _d_split_mask(cfg, shape):
    """Cells with a domain-boundary face under a symmetry velocity condition
    (the sweeps' d_split rule)."""
    nz, ny, nx = shape
    sym = [cfg.vel_bc[f] == _lib.BND_SYMMETRY for f in range(6)]
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    m = np.zeros(shape, dtype=bool)
    m |= sym[_lib.FACE_X0] & (x == 0)
    m |= sym[_lib.FACE_XN] & (x == nx - 1)
    m |= sym[_lib.FACE_Y0] & (y == 0)
    m |= sym[_lib.FACE_YN] & (y == ny - 1)
    m |= sym[_lib.FACE_Z0] & (z == 0)
    m |= sym[_lib.FACE_ZN] & (z == nz - 1)
    return m.reshape(-1)


@pytest.mark.parametrize("bcs", ["canonical", "all_symmetry", "no_symmetry"])
def test_momentum_diagonal_components_equal_off_symmetry(built, bcs):
    """The momentum diagonal D (CSVelPredictPreCompute, FvmColl.compute:
    1292-1859) has three bit-identical components in every cell without a
    symmetry domain face; the momentum sweeps read one component of 1/D there.
    FP32 oracle after a few steps, so D carries advection, LES and wall terms."""
    case = cases.small_case(seed=5, buildings=3)
    cfg = case.cfg
    if bcs == "all_symmetry":
        for f in (_lib.FACE_X0, _lib.FACE_XN, _lib.FACE_Y0, _lib.FACE_YN, _lib.FACE_Z0, _lib.FACE_ZN):
            if f != _lib.FACE_X0:
                cfg.vel_bc[f] = _lib.BND_SYMMETRY
    elif bcs == "no_symmetry":
        for f in (_lib.FACE_YN, _lib.FACE_Z0, _lib.FACE_ZN):
            cfg.vel_bc[f] = _lib.BND_ZERO_GRAD
    o = OracleSolver(cfg, 32)
    o.InitFlags(case.flags)
    o.Step(3)
    o.op("wallfunc"); o.op("eddy_vis"); o.op("les_term"); o.op("vel_precompute")
    D = np.asarray(o.get_field(_lib.FIELD_D), dtype=np.float32).reshape(3, -1)
    split = _d_split_mask(cfg, o.shape)
    fluid = case.flags.reshape(-1) == 0
    keep = fluid & ~split
    assert keep.sum() > 0
    assert np.array_equal(D[0][keep].view(np.uint32), D[1][keep].view(np.uint32))
    assert np.array_equal(D[0][keep].view(np.uint32), D[2][keep].view(np.uint32))
    if bcs != "no_symmetry":
        # the rule is needed: some symmetry cell has components that differ
        s = fluid & split
        assert np.any(D[0][s] != D[1][s]) or np.any(D[0][s] != D[2][s])
