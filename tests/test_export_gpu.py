"""Field export (wf_export_*): frames written while the solver runs, read
back with an independent netCDF reader (scipy.io.netcdf_file)."""
import numpy as np
import pytest

from unitywindsimulation_b200 import FvmSolverCuda, _lib, cases
from unitywindsimulation_b200.solver import FieldExporter

pytestmark = pytest.mark.gpu

netcdf = pytest.importorskip("scipy.io").netcdf_file


def _solver(seed=2):
    case = cases.small_case(24, 12, 16, seed=seed)
    g = FvmSolverCuda(case.cfg)
    cases.apply_case(g, case)
    return case, g


@pytest.mark.parametrize("ring", [1, 3])
def test_export_frames_match_fields(built, tmp_path, ring):
    case, g = _solver()
    c = case.cfg
    path = tmp_path / "flow.nc"
    frames = []
    with FieldExporter(g, path, ring=ring) as ex:
        for k in range(5):
            g.Step(1)
            t = (k + 1) * c.dt
            ex.frame(t)
            frames.append((t, g.GetVelField(layout=_lib.LAYOUT_XYZW), g.GetPresField()))
    f = netcdf(str(path), "r", mmap=False)
    assert f.version_byte == 2
    assert f.gridLayoutType == b"Collocated"
    assert np.float32(f.dt) == np.float32(c.dt)
    assert f.dimensions["velX"] == c.nx and f.dimensions["velY"] == c.ny and f.dimensions["velZ"] == c.nz
    assert f.dimensions["velVec"] == 4 and f.dimensions["time"] is None
    np.testing.assert_array_equal(f.variables["velX"][:], ((np.arange(c.nx) + 0.5) * np.float32(c.dx)).astype(np.float32))
    np.testing.assert_array_equal(f.variables["presZ"][:], ((np.arange(c.nz) + 0.5) * np.float32(c.dx)).astype(np.float32))
    vel = f.variables["velField"][:]
    pres = f.variables["presField"][:]
    times = f.variables["time"][:]
    assert vel.shape == (5, c.nz, c.ny, c.nx, 4) and pres.shape == (5, c.nz, c.ny, c.nx)
    for k, (t, v, p) in enumerate(frames):
        assert times[k] == np.float32(t)
        np.testing.assert_array_equal(vel[k], np.asarray(v).reshape(c.nz, c.ny, c.nx, 4))
        np.testing.assert_array_equal(pres[k], np.asarray(p).reshape(c.nz, c.ny, c.nx))
    f.close()
    g.close()


def test_export_single_field(built, tmp_path):
    case, g = _solver(3)
    g.Step(2)
    path = tmp_path / "pres.nc"
    with FieldExporter(g, path, save_vel=False) as ex:
        ex.frame(0.5)
    f = netcdf(str(path), "r", mmap=False)
    assert "velField" not in f.variables
    np.testing.assert_array_equal(f.variables["presField"][0], g.GetPresField())
    f.close()
    g.close()


def test_export_bad_path(built, tmp_path):
    case, g = _solver(4)
    with pytest.raises(_lib.WindFvmError) as e:
        FieldExporter(g, tmp_path / "missing_dir" / "x.nc")
    assert e.value.status == _lib.WF_ERR_IO
    g.close()


@pytest.mark.parametrize("layout", [_lib.LAYOUT_SOA, _lib.LAYOUT_XYZW])
def test_async_readback_overlaps_next_step(built, layout):
    """readback_begin snapshots the state it is called on: a step launched
    before readback_wait does not change what arrives on the host."""
    case, g = _solver(5)
    n = g.n_cells
    per = 4 if layout == _lib.LAYOUT_XYZW else 3
    vel = np.empty(per * n, np.float32)
    pres = np.empty(n, np.float32)
    g.Step(2)
    want_v = g.GetVelField(layout=layout).reshape(-1).copy()
    want_p = g.GetPresField().reshape(-1).copy()
    g.readback_begin(vel, pres, layout)
    g.Step(1)
    g.readback_wait()
    np.testing.assert_array_equal(vel, want_v)
    np.testing.assert_array_equal(pres, want_p)
    g.readback_begin(vel, pres, layout)
    g.readback_wait()
    np.testing.assert_array_equal(vel, g.GetVelField(layout=layout).reshape(-1))
    g.close()
