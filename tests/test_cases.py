"""Case generator: flag layout, seeds, margins, isolated cells (no GPU)."""
import numpy as np
import pytest

from unitywindsimulation_b200 import cases


def test_plain_cube_layout():
    c = cases.plain_cube()
    assert (c.cfg.nx, c.cfg.ny, c.cfg.nz) == (64, 32, 48)
    assert c.flags.shape == (48, 32, 64)
    flat = c.flags.reshape(-1)
    # reference index z*nx*ny + y*nx + x (InitShaderColl.compute:353)
    nx, ny = 64, 32
    for (x, y, z) in [(12, 0, 20), (19, 7, 27), (15, 3, 24)]:
        assert flat[z * nx * ny + y * nx + x] == 1
    for (x, y, z) in [(11, 0, 20), (20, 0, 20), (12, 8, 20), (12, 0, 28)]:
        assert flat[z * nx * ny + y * nx + x] == 0
    assert flat.sum() == 8 * 8 * 8
    # dt from CFL 0.5 at the top-cell inlet velocity
    umax = 0.5 / 0.41 * np.log((31.5 * 0.5 + 0.1) / 0.1)
    assert abs(c.cfg.dt - 0.5 * 0.5 / umax) < 1e-6


def test_urban_block_seeded_and_valid():
    a = cases.urban_block(seed=2)
    b = cases.urban_block(seed=2)
    c = cases.urban_block(seed=3)
    np.testing.assert_array_equal(a.flags, b.flags)
    np.testing.assert_array_equal(a.inlet, b.inlet)
    assert not np.array_equal(a.flags, c.flags)
    assert len(a.buildings) == 48
    nz, ny, nx = a.flags.shape
    assert (nx, ny, nz) == (256, 96, 192)
    m = cases.MARGIN
    assert a.flags[:, :, :m].sum() == 0 and a.flags[:, :, nx - m:].sum() == 0
    assert a.flags[:m].sum() == 0 and a.flags[nz - m:].sum() == 0
    for (x0, x1, z0, z1, h) in a.buildings:
        assert 6 <= x1 - x0 <= 16 and 6 <= z1 - z0 <= 16 and 4 <= h <= 40
    assert cases.isolated_fluid_count(a.flags) == 0
    # 5 % perturbation: the x velocity varies across the inlet, others zero
    assert a.inlet[:, :, 1:].max() == 0
    rel = a.inlet[:, :, 0] / cases.inlet_plane(ny, nz, 0.5, 0.6, 0.3)[:, :, 0]
    assert 0.02 < rel.std() < 0.08


def test_buildings_do_not_overlap():
    a = cases.urban_block(seed=5)
    occ = np.zeros((192, 256), dtype=int)
    for (x0, x1, z0, z1, h) in a.buildings:
        occ[z0:z1, x0:x1] += 1
    assert occ.max() == 1


def test_batch_directions():
    cs = cases.batch_directions(seed=3)
    assert len(cs) == 16
    sizes = {(c.cfg.nx, c.cfg.ny, c.cfg.nz) for c in cs}
    assert len(sizes) > 4
    for c in cs:
        assert 96 <= c.cfg.nx <= 192 and 48 <= c.cfg.ny <= 80 and 96 <= c.cfg.nz <= 160
        assert cases.isolated_fluid_count(c.flags) == 0
        assert c.flags.sum() > 0


def test_rotation_changes_footprint_not_volume_much():
    blds = [(40, 56, 40, 56, 10)]
    f0 = cases.rasterise_boxes(96, 32, 96, blds, angle_deg=0.0)
    f45 = cases.rasterise_boxes(96, 32, 96, blds, angle_deg=45.0)
    assert not np.array_equal(f0, f45)
    assert abs(int(f45.sum()) - int(f0.sum())) < 0.15 * f0.sum()


def test_isolated_fluid_cells_removed():
    f = np.ones((5, 5, 5), dtype=np.int32)
    f[2, 2, 2] = 0  # fluid pocket inside a solid
    f[0, 0, 0] = 0
    g = cases.remove_isolated_fluid(f)
    assert g[2, 2, 2] == 1 and g[0, 0, 0] == 1
    f[2, 2, 3] = 0  # two connected fluid cells survive
    f[2, 2, 2] = 0
    g = cases.remove_isolated_fluid(f)
    assert g[2, 2, 2] == 0 and g[2, 2, 3] == 0


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_small_cases(seed):
    c = cases.small_case(seed=seed)
    assert cases.isolated_fluid_count(c.flags) == 0
    assert c.cfg.dt > 0


def test_autotune_cache_roundtrip(tmp_path):
    from unitywindsimulation_b200 import autotune
    p = str(tmp_path / "sub" / "t.json")
    assert autotune.load_cache(p) == {}
    autotune.save_cache(p, {"dev|8x8x8": {"pres_k": 3, "vel_k": 1}})
    assert autotune.load_cache(p)["dev|8x8x8"]["pres_k"] == 3
