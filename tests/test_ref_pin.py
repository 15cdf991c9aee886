"""Parity pinned on the reference's own kernels.

tests/golden/ref_kernels.npz holds the outputs of the reference's compute
shaders (translated to C++ by oracle/ref_kernels.py and dispatched in
FvmSolverGpu's order by oracle/ref_driver.cpp; generated by
tests/golden/make_ref_golden.py).  The FP32 oracle must reproduce them bit
for bit, the FP64 oracle within FP32 rounding, and the CUDA library within
REL_TOL = 1e-5 relative L2 per field (the per-field bound of the FP32
kernels, which fuse multiply-adds and reorder sums).  Where the translated
kernels have been built (oracle/_ref/, only where the reference checkout is
present) they are also compared with the oracle live, field by field.
"""
import os
import sys

import numpy as np
import pytest

from unitywindsimulation_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_ref_golden as G  # noqa: E402

from helpers import REL_TOL, rel_l2  # noqa: E402

FIXTURE = np.load(G.FIXTURE)
KEYS = sorted(FIXTURE.files)


def _oracle(precision):
    from oracle import OracleSolver
    return lambda cfg: OracleSolver(cfg, precision=precision)


def test_fixture_covers_every_case():
    expect = {f"{n}_{q}" for n in list(G.CASES) + ["nested"] for q in ("u", "p")}
    assert set(KEYS) == expect
    for k in KEYS:
        assert np.isfinite(FIXTURE[k]).all() and np.abs(FIXTURE[k]).max() > 0.1, k


def test_oracle_fp32_bit_identical_to_reference_kernels(built):
    out = G.all_outputs(_oracle(32))
    for k in KEYS:
        assert np.array_equal(out[k], FIXTURE[k]), (k, float(np.abs(out[k] - FIXTURE[k]).max()))


def test_oracle_fp64_within_fp32_rounding_of_reference_kernels(built):
    out = G.all_outputs(_oracle(64))
    for k in KEYS:
        assert rel_l2(out[k], FIXTURE[k]) <= 1e-5, k


# ---- live comparison with the translated kernels (where they are built) ----

def _ref():
    from oracle.binding import ref_available
    if not ref_available():
        pytest.skip("reference kernels not built (make -C oracle ref, needs the reference checkout)")
    from oracle.binding import RefSolver
    return RefSolver


def test_reference_kernels_reproduce_fixture(built):
    out = G.all_outputs(_ref())
    for k in KEYS:
        assert np.array_equal(out[k], FIXTURE[k]), k


def _all_fields_equal(o, r, label, skip=()):
    for f in range(_lib.FIELD_BND_ZN + 1):
        if f in skip:
            continue
        a = np.asarray(o.get_field(f), dtype=np.float32)
        b = r.get_field(f)
        assert np.array_equal(a, b), (label, _lib.FIELD_NAMES[f], float(np.abs(a - b).max()))
    assert np.array_equal(np.asarray(o.GetFlagField()), r.GetFlagField()), label


@pytest.mark.parametrize("kw", [
    dict(piso=True, les=True, log=True, seed=10),
    dict(piso=False, les=True, log=False, seed=11),
    dict(piso=True, les=False, log=True, normalise=True, seed=12),
    dict(piso=False, les=True, log=True, seed=13, compat=_lib.COMPAT_RFLOAT_FACE_EDDY_VIS),
], ids=["piso_les_log", "simple_les_const", "piso_laminar_normalised", "simple_les_rfloat"])
def test_every_field_matches_reference_kernels_each_step(built, kw):
    """Every texture of the step (intermediates included: D, b, the pressure
    coefficients, AodU, eddy viscosities, the correction fields, the
    velField/velFieldLastIter roles) after construction, InitFlags and each
    of three steps.  Under WF_COMPAT_RFLOAT_FACE_EDDY_VIS the oracle keeps
    all three face channels and drops y and z when it reads them, while the
    texture drops them when written, so that field is compared as read."""
    from oracle import OracleSolver
    Ref = _ref()
    cfg, flags = G.case_config(**kw)
    o, r = OracleSolver(cfg, precision=32), Ref(cfg)
    rfloat = bool(cfg.compat_flags & _lib.COMPAT_RFLOAT_FACE_EDDY_VIS)

    def check(label):
        if rfloat:
            a = np.asarray(o.get_field(_lib.FIELD_FACE_EDDY_VIS), dtype=np.float32)
            b = r.get_field(_lib.FIELD_FACE_EDDY_VIS)
            assert np.array_equal(a[0], b[0]) and not b[1:].any(), label
            _all_fields_equal(o, r, label, skip=(_lib.FIELD_FACE_EDDY_VIS,))
        else:
            _all_fields_equal(o, r, label)

    check("construct")
    o.InitFlags(flags)
    r.InitFlags(flags)
    check("flags")
    for step in range(3):
        o.Step(1)
        r.Step(1)
        check(f"step {step}")


def test_aij_validation_case_matches_reference_kernels(built):
    """The reference's AIJ case (80 x 40 x 40, SIMPLE + Smagorinsky, log
    inflow, the hard-coded box), set up and stepped twice with cut iteration
    counts, every field bit-identical."""
    from oracle import OracleSolver
    from unitywindsimulation_b200 import cases
    Ref = _ref()
    c = cases.aij_building(nv=10, np_=20)
    o, r = OracleSolver(c.cfg, precision=32), Ref(c.cfg)
    o.InitFlags(c.flags)
    r.InitFlags(c.flags)
    o.Step(2)
    r.Step(2)
    _all_fields_equal(o, r, "aij")


@pytest.mark.parametrize("rot", [0.0, 30.0, -75.0, 180.0])
def test_background_init_matches_reference_kernels(built, rot):
    from oracle import OracleSolver
    Ref = _ref()
    cfg, _ = G.case_config(piso=False, les=False, log=False, seed=20)
    rng = np.random.default_rng(21)
    n = cfg.nx * cfg.ny * cfg.nz
    v = rng.standard_normal((3, n)).astype(np.float32)
    p = rng.standard_normal(n).astype(np.float32)
    bgs = OracleSolver(cfg, precision=32), Ref(cfg)
    for b in bgs:
        b.set_field(_lib.FIELD_VEL, v)
        b.set_field(_lib.FIELD_VEL_LAST_TIME, v)
        b.set_field(_lib.FIELD_PRES, p)
    fcfg = G.case_config(piso=False, les=False, log=False, seed=22, nx=16, ny=8, nz=12)[0]
    fcfg.dx = 0.25
    o, r = OracleSolver(fcfg, precision=32), Ref(fcfg)
    o.InitVelPresFieldsFromBackGroundFlow(bgs[0], (1.0, 2.0, 0.5), (0.0, 2.5, 0.0), rot)
    r.InitVelPresFieldsFromBackGroundFlow(bgs[1], (1.0, 2.0, 0.5), (0.0, 2.5, 0.0), rot)
    _all_fields_equal(o, r, f"rot {rot}")


def test_reinit_and_boundary_calls_match_reference_kernels(built):
    from oracle import OracleSolver
    Ref = _ref()
    for log in (False, True):
        cfg, flags = G.case_config(piso=True, les=True, log=log, seed=30)
        o, r = OracleSolver(cfg, precision=32), Ref(cfg)
        for s in (o, r):
            s.InitFlags(flags)
            s.Step(1)
            s.SetFixedValueVelBndCond(4.5)
            s.InitVelPresFields()
            s.Step(1)
        _all_fields_equal(o, r, f"log={log}")


# ---- the CUDA library against the reference kernels' fixture ----------------

@pytest.mark.gpu
def test_cuda_library_matches_reference_kernel_fixture(built):
    from unitywindsimulation_b200 import FvmSolverCuda
    out = G.all_outputs(lambda cfg: FvmSolverCuda(cfg))
    errs = {k: rel_l2(out[k], FIXTURE[k]) for k in KEYS}
    bad = {k: e for k, e in errs.items() if not e <= REL_TOL}
    assert not bad, f"above {REL_TOL}: {bad} (all: {errs})"
