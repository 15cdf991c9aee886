"""Non-uniform collocated grid (gridType CollNonUniform).

Parity is pinned on the reference's own kernels: FvmCollNonUniform.compute
and InitShaderColl.compute translated to C++ (oracle/ref_kernels.py) and
replayed in FvmSolverGpu's order (oracle/ref_driver.cpp), recorded in
tests/golden/nonuniform_ref.npz by tests/golden/make_nu_golden.py.  The
oracle's restatement must reproduce every recorded field bit for bit in
FP32 and within 1e-5 in FP64; the CUDA library must match every recorded
field within REL_TOL = 1e-5 relative L2 per field and step.  The mesh generator restates InitMeshBuffers
(FvmSolverGpu.cs:682-788).
"""
import os
import sys

import numpy as np
import pytest

from unitywindsimulation_b200 import _lib, cases

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_nu_golden as G  # noqa: E402

from helpers import REL_TOL, rel_l2  # noqa: E402

FIXTURE = np.load(G.FIXTURE)


# ---- mesh (CPU) -------------------------------------------------------------

def test_wind_tunnel_mesh_follows_init_mesh_buffers():
    """WindTunnelBoxConfig: 25 cells growing by 1.08 towards x0 (largest at
    the boundary), 50 cells of dx = 1, then 25 cells growing away from the
    core; y uniform."""
    fx = cases.stretched_faces(100, 1.0, 50, 25)
    d = np.diff(fx.astype(np.float64))
    assert fx[0] == 0.0 and np.all(d > 0)
    sizes = np.empty(25, dtype=np.float32)
    sizes[0] = 1.0
    for i in range(1, 25):
        sizes[i] = np.float32(sizes[i - 1] * np.float32(1.08))
    np.testing.assert_allclose(d[:25], sizes[::-1], rtol=0, atol=4e-5)  # differences of FP32 sums
    np.testing.assert_allclose(d[25:75], 1.0, rtol=0, atol=4e-5)
    np.testing.assert_allclose(d[75:], sizes, rtol=0, atol=4e-5)
    fy = cases.stretched_faces(50, 1.0, 50, 0)
    assert np.array_equal(fy, np.arange(51, dtype=np.float32))


def test_mesh_upper_side_reuses_lower_sizes():
    """The upper side takes the lower side's sizes (FvmSolverGpu.cs:758-762):
    a longer upper side has no sizes to take."""
    f = cases.stretched_faces(10, 0.5, 6, 3)
    d = np.diff(f)
    assert np.allclose(d[:3], [0.5 * 1.08 ** 2, 0.5 * 1.08, 0.5], rtol=1e-6)
    assert np.allclose(d[9:], [0.5], rtol=1e-6)
    with pytest.raises(ValueError):
        cases.stretched_faces(10, 0.5, 4, 2)  # 4 upper cells, 2 lower sizes


def test_fixture_covers_cases():
    for name in G.CASES:
        assert f"{name}/0/vel" in FIXTURE.files
        for k in range(1, G.STEPS + 1):
            for key in ("vel", "pres") + (("flux",) if k == G.STEPS else ()):
                a = FIXTURE[f"{name}/{k}/{key}"]
                assert np.isfinite(a).all() and np.abs(a).max() > 0.01, (name, k, key)
        for key, _ in G.LAST_FIELDS:
            assert np.isfinite(FIXTURE[f"{name}/{G.STEPS}/{key}"]).all()


def _oracle_outputs(precision, names=None):
    from oracle import OracleSolver
    out = {}
    for name in (names or G.CASES):
        def rec(step, key, a, name=name):
            out[f"{name}/{step}/{key}"] = np.asarray(a)
        G.run_case(lambda cfg: OracleSolver(cfg, precision), name, rec)
    return out


def test_oracle_fp32_bit_identical_to_reference_kernels(built):
    """The oracle's C++ restatement of FvmCollNonUniform.compute (FP32, no
    contraction) reproduces the reference's own kernels bit for bit."""
    out = _oracle_outputs(32)
    assert set(out) == set(FIXTURE.files)
    for k, a in out.items():
        assert np.array_equal(a.astype(np.float32), FIXTURE[k]), (k, float(np.abs(a - FIXTURE[k]).max()))


# Recorded fields that are small differences of large terms: bp (the
# divergence of the predicted velocity) and the velocity correction.  The
# reference's own FP32 arithmetic departs from FP64 by up to about 2e-5
# there (LES cases); other fields by less than 1e-5.
CANCELLING = ("/bp", "/vel_correct")


def _fp64_bound(k):
    return 5e-5 if k.endswith(CANCELLING) else 1e-5


def test_oracle_fp64_within_fp32_rounding_of_reference_kernels(built):
    out = _oracle_outputs(64)
    for k, a in out.items():
        assert rel_l2(a, FIXTURE[k]) <= _fp64_bound(k), (k, rel_l2(a, FIXTURE[k]))


def test_reference_kernels_reproduce_fixture():
    """Where the translated kernels are built (the reference checkout is
    present), they reproduce the committed fixture bit for bit."""
    from oracle.binding import RefSolver, ref_available
    if not ref_available():
        pytest.skip("reference kernels not built (oracle/_ref)")
    for name in G.CASES:
        got = {}

        def rec(step, key, a):
            got[f"{name}/{step}/{key}"] = a
        G.run_case(lambda cfg: RefSolver(cfg), name, rec)
        for k, a in got.items():
            assert np.array_equal(a, FIXTURE[k]), k


def test_reference_kernels_reject_piso():
    from oracle.binding import RefSolver, ref_available
    if not ref_available():
        pytest.skip("reference kernels not built (oracle/_ref)")
    case = cases.small_nonuniform_case()
    cfg = case.cfg.copy()
    cfg.solver_type = _lib.SOLVER_PISO
    r = RefSolver(cfg)
    with pytest.raises(RuntimeError):
        r.set_face_positions(*case.faces)


# ---- CUDA library against the fixture (GPU) --------------------------------

def _cuda(**over):
    from unitywindsimulation_b200.solver import FvmSolverCuda

    def make(cfg):
        c = cfg.copy()
        for k, v in over.items():
            setattr(c, k, v)
        return FvmSolverCuda(c)
    return make


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(G.CASES))
def test_cuda_matches_reference_kernels(name):
    got = {}

    def rec(step, key, a):
        got[f"{name}/{step}/{key}"] = a
    G.run_case(_cuda(), name, rec)
    assert set(got) == {k for k in FIXTURE.files if k.startswith(name + "/")}
    # the cancelling fields: held to max(REL_TOL, 2 x the reference's own
    # FP32 departure from FP64 on the same field)
    ref64 = _oracle_outputs(64, names=[name]) if any(k.endswith(CANCELLING) for k in got) else {}
    for k, a in got.items():
        err = rel_l2(a, FIXTURE[k])
        tol = REL_TOL
        if k.endswith(CANCELLING):
            tol = max(REL_TOL, 2.0 * rel_l2(FIXTURE[k], ref64[k]))
        assert err <= tol, (k, err, tol)


@pytest.mark.gpu
def test_graph_replay_equals_eager_steps():
    name = "const_tunnel"
    outs = []
    for graph in (1, 0):
        got = {}

        def rec(step, key, a):
            got[f"{step}/{key}"] = a
        G.run_case(_cuda(use_graph=graph), name, rec)
        outs.append(got)
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.gpu
def test_residual_path_runs_the_same_sweeps():
    """calc_residual with tolerances no sweep reaches: the loop with residual
    reads gives the same fields as the plain loop."""
    name = "log_urban_normalised"
    outs = []
    for resid in (0, 1):
        got = {}

        def rec(step, key, a):
            got[f"{step}/{key}"] = a
        over = dict(calc_residual=resid)
        if resid:
            over.update(vel_tol=0.0, pres_tol=0.0, vel_res_interval=3, pres_res_interval=5)
        G.run_case(_cuda(**over), name, rec)
        outs.append(got)
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.gpu
def test_unsupported_combinations_are_refused():
    from unitywindsimulation_b200.solver import FvmSolverCuda
    from unitywindsimulation_b200._lib import WindFvmError
    case = cases.small_nonuniform_case()
    # PISO: the reference has no PISO shader for this grid (FvmSolverGpu.cs:493-496)
    cfg = case.cfg.copy()
    cfg.solver_type = _lib.SOLVER_PISO
    s = FvmSolverCuda(cfg)
    with pytest.raises(WindFvmError) as e:
        s.set_face_positions(*case.faces)
    assert e.value.status == _lib.WF_ERR_UNSUPPORTED
    # LES runs on this grid, as in the reference
    cfg = case.cfg.copy()
    cfg.turbulence = _lib.TURB_SMAGORINSKY
    FvmSolverCuda(cfg).set_face_positions(*case.faces)
    s = FvmSolverCuda(case.cfg)
    with pytest.raises(WindFvmError):
        s.set_face_positions(case.faces[0][::-1].copy(), case.faces[1], case.faces[2])  # decreasing
    s.set_face_positions(*case.faces)
    from unitywindsimulation_b200.adjoint import AdjointSolver
    with pytest.raises(WindFvmError):
        AdjointSolver(s)
    s.set_face_positions(None, None, None)  # back to the uniform grid
    s.Step(1)


@pytest.mark.gpu
def test_four_cell_sweeps_equal_one_cell_sweeps(monkeypatch):
    """The four-cells-per-thread momentum and pressure sweeps (nx % 4 == 0)
    give the same fields, bit for bit, as the one-cell sweeps (WF_VEC4=0)."""
    name = "const_tunnel"
    outs = []
    for vec4 in ("1", "0"):
        monkeypatch.setenv("WF_VEC4", vec4)
        got = {}

        def rec(step, key, a):
            got[f"{step}/{key}"] = a
        G.run_case(_cuda(), name, rec)
        outs.append(got)
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.gpu
def test_chained_launches_equal_plain_stream_order(monkeypatch):
    """Programmatic dependent launch of the sweep chains (default) gives the
    same fields, bit for bit, as plain stream order (WF_PDL=0), with and
    without graph replay."""
    name = "log_urban_normalised"
    outs = []
    for pdl, graph in (("1", 1), ("0", 1), ("1", 0)):
        monkeypatch.setenv("WF_PDL", pdl)
        got = {}

        def rec(step, key, a):
            got[f"{step}/{key}"] = a
        G.run_case(_cuda(use_graph=graph), name, rec)
        outs.append(got)
    for other in outs[1:]:
        for k in outs[0]:
            assert np.array_equal(outs[0][k], other[k]), k


@pytest.mark.parametrize("name", list(G.CASES))
def test_momentum_diagonal_components_equal_off_symmetry(built, name):
    """On the non-uniform grid too, the three components of D
    (CSVelPredictPreCompute, FvmCollNonUniform.compute:111-721) are
    bit-identical outside cells with a symmetry domain face, which the
    momentum sweeps rely on when they read one component of 1/D there
    (FP32 oracle after 3 steps)."""
    from oracle import OracleSolver
    from test_oracle import _d_split_mask
    case = G.make_case(name)
    o = OracleSolver(case.cfg, 32)
    cases.apply_case(o, case)
    o.Step(3)
    D = np.asarray(o.get_field(_lib.FIELD_D), dtype=np.float32).reshape(3, -1)
    keep = (case.flags.reshape(-1) == 0) & ~_d_split_mask(case.cfg, o.shape)
    assert keep.sum() > 0
    assert np.array_equal(D[0][keep].view(np.uint32), D[1][keep].view(np.uint32))
    assert np.array_equal(D[0][keep].view(np.uint32), D[2][keep].view(np.uint32))


@pytest.mark.gpu
def test_checkpoint_with_face_flux_resumes_exactly():
    """wf_get_state / wf_set_state plus the face-flux texture restore a
    non-uniform handle exactly: two more steps from the checkpoint on a
    fresh handle give the fields of two more steps on the original."""
    from unitywindsimulation_b200.solver import FvmSolverCuda
    case = G.make_case("log_urban_normalised")
    a = FvmSolverCuda(case.cfg)
    cases.apply_case(a, case)
    a.Step(2)
    vel, pres, step = a.get_state()
    flux = a.get_face_flux()
    b = FvmSolverCuda(case.cfg)
    cases.apply_case(b, case)
    b.set_state(vel, pres, step)
    b.set_face_flux(flux)
    a.Step(2)
    b.Step(2)
    for f in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES):
        assert np.array_equal(a.get_field(f), b.get_field(f)), f
    assert np.array_equal(a.get_face_flux(), b.get_face_flux())


@pytest.mark.gpu
def test_traced_step_equals_plain_step():
    """wf_step_phases on a non-uniform handle leaves the same fields as a
    plain step."""
    from unitywindsimulation_b200.solver import FvmSolverCuda
    case = G.make_case("const_tunnel")
    a, b = FvmSolverCuda(case.cfg), FvmSolverCuda(case.cfg)
    for s in (a, b):
        cases.apply_case(s, case)
    a.Step(2)
    b.Step(1)
    ms = b.step_phases()
    assert all(v >= 0.0 for v in ms.values())
    for f in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES):
        assert np.array_equal(a.get_field(f), b.get_field(f)), f
