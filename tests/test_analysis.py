"""Post-processing definitions (CPU): tip position, radius, velocity."""
import numpy as np

from microsim_b200 import analysis as A


def _disc(n, r, cx=0.0, cy=0.0, w=2.0):
    x, y = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    d = np.sqrt((x - cx) ** 2 + (y - cy) ** 2)
    return 0.5 * (1.0 - np.tanh((d - r) / w))


def test_tip_position_of_a_corner_disc():
    phi = _disc(64, 20.0)
    assert abs(A.tip_position(phi, 0) - 20.0) < 0.05
    assert abs(A.tip_position(phi, 1) - 20.0) < 0.05
    assert A.tip_position(np.zeros((8, 8)), 0) == -1.0


def test_tip_radius_of_a_disc_is_its_radius():
    phi = _disc(96, 30.0, w=1.0)
    assert abs(A.tip_radius(phi, 0, rows=8) - 30.0) / 30.0 < 0.05


def test_velocity_is_the_slope():
    t = np.arange(10.0)
    assert abs(A.velocity(t, 3.0 * t + 1.0) - 3.0) < 1e-12
    assert abs(A.velocity(t, np.r_[np.zeros(5), 2.0 * np.arange(5)], window=5) - 2.0) < 1e-12
