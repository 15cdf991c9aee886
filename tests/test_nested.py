"""Initialisation from a background domain (InitVelPresFieldsFromBackGroundFlow).

CPU tests pin the oracle's restatement of CSInitVelPresFieldsFromBGFlowRotate
(InitShaderColl.compute:185-226) on fields whose trilinear samples are known
in closed form; the GPU test holds the library to the FP32 oracle.
"""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from oracle import OracleSolver

from helpers import REL_TOL, rel_l2


def _pair(nx, ny, nz, dx=0.5, nbx=None, nby=None, nbz=None, dxb=None, precision=64):
    c = cases.small_case(nx, ny, nz, les=False, seed=1, buildings=0).cfg
    cb = c.copy()
    cb.nx, cb.ny, cb.nz = nbx or nx, nby or ny, nbz or nz
    cb.dx = dxb or dx
    c.dx = dx
    return OracleSolver(c, precision), OracleSolver(cb, precision), c, cb


def _set_bg(bg, cb, fx):
    """Background velocity (all three components) and pressure from a
    function of the cell indices (z, y, x)."""
    z, y, x = np.meshgrid(np.arange(cb.nz), np.arange(cb.ny), np.arange(cb.nx), indexing="ij")
    f = fx(z, y, x).astype(np.float64).reshape(-1)
    vel = np.stack([f, 2 * f, -f])
    for fid in (_lib.FIELD_VEL, _lib.FIELD_VEL_LAST_TIME, _lib.FIELD_VEL_LAST_ITER):
        bg.set_field(fid, vel)
    bg.set_field(_lib.FIELD_PRES, 3 * f)


@pytest.mark.parametrize("nx", [16, 17])
def test_identity_placement_half_cell_offset(built, nx):
    """Same grid, same centre, no rotation: a cell samples the background at
    texel coordinate index + (0 if the size is odd else -0.5), clamped."""
    fg, bg, c, cb = _pair(nx, 8, 10)
    _set_bg(bg, cb, lambda z, y, x: 0.25 * x + 1.0)
    fg.InitVelPresFieldsFromBackGroundFlow(bg)
    u = fg.GetVelField()[0][0, 0, :]
    x = np.arange(nx)
    t = x if nx % 2 else np.maximum(x - 0.5, 0.0)
    np.testing.assert_allclose(u, 0.25 * t + 1.0, rtol=0, atol=1e-12)
    np.testing.assert_allclose(fg.GetPresField()[0, 0, :], 3 * (0.25 * t + 1.0), atol=1e-12)
    np.testing.assert_allclose(fg.GetVelField()[2][0, 0, :], -(0.25 * t + 1.0), atol=1e-12)
    assert not np.any(fg.get_field(_lib.FIELD_VEL_CORRECT))


def test_rotation_maps_offsets(built):
    """Rotation acts on the offset between the domain centres: at 90 degrees
    an offset of d along x samples the background d further along z (the
    cell offsets themselves rotate back, R(-theta) R(theta) = 1)."""
    fg, bg, c, cb = _pair(8, 6, 16, nbz=32)
    _set_bg(bg, cb, lambda z, y, x: 0.5 * z)
    d = 3.0  # metres = 6 cells at dx = 0.5
    fg.InitVelPresFieldsFromBackGroundFlow(bg, pos=(d, 0.0, 0.0), rot_deg=90.0)
    u = fg.GetVelField()[0][:, 2, 3]
    z = np.arange(16)
    # fg cell z sits at (z - 8) dx + 6 cells from the background centre (16)
    t = (z - 8) + 6 + 16 - 0.5
    np.testing.assert_allclose(u, 0.5 * np.clip(t, 0, 31), atol=1e-6)


def test_scaled_grids_and_clamping(built):
    """A coarse background (dx twice as large) and a domain that reaches past
    its edge: samples clamp to the edge texel."""
    fg, bg, c, cb = _pair(16, 8, 8, dx=0.5, nbx=6, nby=8, nbz=8, dxb=1.0)
    _set_bg(bg, cb, lambda z, y, x: x * 1.0)
    fg.InitVelPresFieldsFromBackGroundFlow(bg)
    u = fg.GetVelField()[0][4, 4, :]
    x = np.arange(16)
    # position (x - 8) * 0.5 m; background texel coordinate = pos / 1.0 + 3 - 0.5
    t = np.clip((x - 8) * 0.5 + 3 - 0.5, 0, 5)
    np.testing.assert_allclose(u, t, atol=1e-12)


@pytest.mark.gpu
def test_init_from_background_matches_oracle(built):
    bgc = cases.small_case(32, 16, 24, les=True, seed=3)
    fgc = cases.small_case(20, 12, 16, les=True, seed=4)
    gb, gf = FvmSolverCuda(bgc.cfg), FvmSolverCuda(fgc.cfg)
    ob, of = OracleSolver(bgc.cfg, 32), OracleSolver(fgc.cfg, 32)
    cases.apply_case(gb, bgc)
    cases.apply_case(gf, fgc)
    gb.Step(3)
    vel, pres, _ = gb.get_state()
    cases.apply_case(ob, bgc)
    cases.apply_case(of, fgc)
    for fid in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_VEL, _lib.FIELD_VEL_LAST_ITER):
        ob.set_field(fid, np.asarray(vel, np.float64).reshape(3, -1))
    ob.set_field(_lib.FIELD_PRES, np.asarray(pres, np.float64).reshape(-1))
    args = dict(pos=(1.3, 0.2, -0.7), pos_background=(0.4, 0.0, 0.5), rot_deg=30.0)
    gf.InitVelPresFieldsFromBackGroundFlow(gb, **args)
    of.InitVelPresFieldsFromBackGroundFlow(ob, **args)
    for fid in (_lib.FIELD_VEL, _lib.FIELD_VEL_LAST_TIME, _lib.FIELD_VEL_LAST_ITER, _lib.FIELD_PRES):
        assert rel_l2(gf.get_field(fid), of.get_field(fid)) <= REL_TOL, _lib.FIELD_NAMES[fid]
    assert not np.any(gf.get_field(_lib.FIELD_VEL_CORRECT))
    # the initialised domain steps like any other: one step against the oracle
    gf.Step(1)
    of.Step(1)
    assert rel_l2(gf.GetVelField(), of.GetVelField()) <= REL_TOL
    assert rel_l2(gf.GetPresField(), of.GetPresField()) <= REL_TOL
    # the background is untouched
    v2, p2, _ = gb.get_state()
    np.testing.assert_array_equal(v2, vel)
    with pytest.raises(_lib.WindFvmError):
        gf.InitVelPresFieldsFromBackGroundFlow(gf)
