"""Per-phase device timing of one step (wf_step_phases): the phases cover the
step, and the traced step leaves the same fields as a plain step."""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [dict(piso=True, les=True, seed=0), dict(piso=False, les=False, seed=1)],
                         ids=["piso_les", "simple_laminar"])
def test_traced_step_equals_plain_step(built, kw):
    case = cases.small_case(nx=48, ny=24, nz=32, **kw)
    a, b = FvmSolverCuda(case.cfg), FvmSolverCuda(case.cfg)
    for s in (a, b):
        cases.apply_case(s, case)
        s.Step(2)
    ph = a.step_phases()
    b.Step(1)
    for f in (_lib.FIELD_VEL_LAST_TIME, _lib.FIELD_PRES, _lib.FIELD_VEL_CORRECT):
        assert np.array_equal(a.get_field(f), b.get_field(f)), _lib.FIELD_NAMES[f]
    assert set(ph) == set(_lib.PHASE_NAMES)
    assert all(v >= 0.0 for v in ph.values())
    assert ph["vel_sweeps"] > 0.0 and ph["pres_sweeps"] > 0.0
    if kw["piso"]:
        assert ph["piso"] > 0.0
    # both continue identically
    a.Step(1)
    b.Step(1)
    assert np.array_equal(a.get_field(_lib.FIELD_VEL_LAST_TIME), b.get_field(_lib.FIELD_VEL_LAST_TIME))
    a.close()
    b.close()


def test_phase_times_add_up_to_a_step(built):
    case = cases.small_case(nx=64, ny=32, nz=48, seed=2)
    s = FvmSolverCuda(case.cfg)
    cases.apply_case(s, case)
    s.Step(3)
    ph = s.step_phases()
    total = sum(ph.values())
    s.Step(5)
    plain = s.last_step_ms() / 5
    # the traced step is enqueued without graph replay: the same kernels plus
    # launch gaps, so it takes at least about as long as a replayed step
    assert total > plain / 3
    assert ph["vel_sweeps"] + ph["pres_sweeps"] + ph["piso"] > 0.3 * total
    s.close()
