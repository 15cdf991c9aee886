"""GPU footprint rasteriser (wf_rasterise_boxes) against the NumPy case
generator: identical flags, integer-exact, for rotated footprints, the
boundary margin, heights rounded half to even and clipped at the top, and
overlapping boxes."""
import numpy as np
import pytest

from unitywindsimulation_b200 import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("angle", [0.0, 22.5, 45.0, 90.0, 157.5, 333.0])
def test_matches_numpy_generator(built, angle):
    rng = np.random.default_rng(11)
    blds = cases.street_lattice_buildings(rng, 160, 128, 24, 6, 14, 3, 40)
    blds += [(40, 60, 40, 55, 2.5), (50, 70, 45, 50, 3.5), (70, 75, 70, 75, 500), (10, 20, 10, 20, 0)]
    a = cases.rasterise_boxes(160, 48, 128, blds, angle_deg=angle, margin=10)
    b = cases.rasterise_boxes_gpu(160, 48, 128, blds, angle_deg=angle, margin=10)
    assert a.dtype == b.dtype and a.shape == b.shape
    assert np.array_equal(a, b), int((a != b).sum())
    assert a.sum() > 0


def test_no_boxes_and_tiny_grid(built):
    assert not cases.rasterise_boxes_gpu(8, 4, 6, [], angle_deg=10.0, margin=0).any()
    blds = [(0, 8, 0, 6, 3)]
    assert np.array_equal(cases.rasterise_boxes_gpu(8, 4, 6, blds, margin=0), cases.rasterise_boxes(8, 4, 6, blds, margin=0))


def test_direction_sweep_cases_reproduced(built):
    """The batched workload's flags (before isolated-fluid removal) for all
    16 directions."""
    rng = np.random.default_rng(3)
    blds = cases.street_lattice_buildings(rng, 144, 112, 20, 6, 14, 4, 30)
    for k in range(16):
        a = cases.rasterise_boxes(144, 64, 112, blds, angle_deg=22.5 * k)
        b = cases.rasterise_boxes_gpu(144, 64, 112, blds, angle_deg=22.5 * k)
        assert np.array_equal(a, b), k
