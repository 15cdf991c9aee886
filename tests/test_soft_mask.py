"""Soft building mask (host-side, no GPU): drag field shape and the chain
rule from dJ/dchi to dJ/dh against numerical differences of the mask."""
import numpy as np

from unitywindsimulation_b200 import cases
from unitywindsimulation_b200.soft_mask import SoftBuildings


def test_drag_profile():
    sb = SoftBuildings([(2, 4, 1, 3)], [5.0], chi_max=100.0, width=1.0)
    d = sb.drag(8, 14, 6, np.float64)
    col = d[1, :, 2]
    assert col[0] > 98.0 and col[-1] < 0.1
    assert np.all(np.diff(col) < 0)
    assert abs(d[1, 4, 2] - 100.0 / (1.0 + np.exp(-0.5))) < 1e-9  # y_c = 4.5, h = 5
    assert not np.any(d[0]) and not np.any(d[:, :, 5])


def test_height_gradient_chain_rule():
    rng = np.random.default_rng(0)
    nx, ny, nz = 20, 12, 14
    sb = SoftBuildings([(2, 5, 1, 4), (8, 11, 6, 10), (14, 17, 2, 5)], [3.3, 6.1, 8.7], chi_max=400.0)
    w = rng.standard_normal((nz, ny, nx))
    g = sb.height_gradient(w, nx, ny, nz)
    for i in range(3):
        hp, hm = sb.heights.copy(), sb.heights.copy()
        hp[i] += 1e-5
        hm[i] -= 1e-5
        fd = ((w * sb.with_heights(hp).drag(nx, ny, nz, np.float64)).sum()
              - (w * sb.with_heights(hm).drag(nx, ny, nz, np.float64)).sum()) / 2e-5
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd))


def test_rotated_footprints_chain_rule():
    rng = np.random.default_rng(1)
    nx, ny, nz = 24, 10, 20
    sb = SoftBuildings([(4, 9, 3, 8), (13, 18, 10, 16)], [4.2, 6.7], chi_max=300.0, angle_deg=30.0)
    assert sb.footprint_mask(0, nx, nz).sum() > 10
    w = rng.standard_normal((nz, ny, nx))
    g = sb.height_gradient(w, nx, ny, nz)
    for i in range(2):
        hp, hm = sb.heights.copy(), sb.heights.copy()
        hp[i] += 1e-5
        hm[i] -= 1e-5
        fd = ((w * sb.with_heights(hp).drag(nx, ny, nz, np.float64)).sum()
              - (w * sb.with_heights(hm).drag(nx, ny, nz, np.float64)).sum()) / 2e-5
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd))


def test_adjoint_street_case():
    c = cases.adjoint_street()
    assert c.soft is not None and len(c.soft.footprints) == 12
    assert np.all((c.soft.heights >= 4) & (c.soft.heights <= 30))
    assert not np.any(c.flags)
    assert c.cfg.turbulence == 0
    fp = c.soft.footprints
    for i in range(len(fp)):
        for j in range(i + 1, len(fp)):
            a, b = fp[i], fp[j]
            assert a[1] <= b[0] or b[1] <= a[0] or a[3] <= b[2] or b[3] <= a[2]
