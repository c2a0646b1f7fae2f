"""Host logic of the storage-precision sweep (no GPU): surface heights from
the fill level and the comparison metrics."""
import numpy as np

from flowlb_b200 import cases
from flowlb_b200 import precision_sweep as P


def test_surface_height_interpolates_the_half_crossing():
    ny, nx = 20, 4
    phi = np.zeros((ny, nx))
    flags = np.full((ny, nx), cases.GAS, np.uint8)
    phi[:10, 0] = 1.0
    phi[10, 0] = 0.75          # crossing between y=10 (0.75) and y=11 (0)
    phi[:5, 1] = 1.0           # crossing between y=4 (1.0) and y=5 (0.0): 4.5 + 0.5
    phi[:3, 2] = 1.0
    phi[7, 2] = 0.6            # a droplet above: the topmost crossing counts
    phi[0, 3] = 0.4            # dry column
    flags[phi > 0] = cases.FLUID
    flags[0, 3] = cases.INTERFACE
    h = P.surface_heights(phi, flags)
    assert np.isclose(h[0], 10.5 + 0.25 / 0.75)
    assert np.isclose(h[1], 5.0)
    assert np.isclose(h[2], 7.5 + 0.1 / 0.6)
    assert h[3] == 0.0


def test_surface_height_ignores_solid_cells():
    phi = np.zeros((6, 1))
    phi[:, 0] = [1, 1, 1, 0.9, 0.9, 0.9]
    flags = np.full((6, 1), cases.FLUID, np.uint8)
    flags[3:, 0] = cases.WALL  # a solid roof holding stale fill levels
    assert np.isclose(P.surface_heights(phi, flags)[0], 3.0)


def test_compare_of_identical_fields_is_zero_and_detects_a_shift():
    rng = np.random.default_rng(3)
    nx, ny = 16, 12
    flags = np.full(nx * ny, cases.FLUID, np.uint8)
    flags[nx * 8:] = cases.GAS
    flags[nx * 7:nx * 8] = cases.INTERFACE
    u = rng.standard_normal(2 * nx * ny) * 0.01
    phi = np.where(flags == cases.FLUID, 1.0, np.where(flags == cases.INTERFACE, 0.5, 0.0))
    r = P.compare(u, phi, flags, u, phi, flags, nx, ny)
    assert r["velocity_l2"] == 0.0 and r["surface_error_cells"] == 0.0 and r["depth_error_cells"] == 0.0
    assert r["flag_mismatch_cells"] == 0
    u2 = u * 1.001
    phi2 = phi.copy()
    phi2[nx * 7:nx * 8] = 0.75
    r2 = P.compare(u2, phi2, flags, u, phi, flags, nx, ny)
    assert np.isclose(r2["velocity_l2"], 1e-3)
    assert np.isclose(r2["depth_error_cells"], 0.25)
    assert r2["surface_error_cells"] > 0
