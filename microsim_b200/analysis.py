"""Post-processing of solidification fields: tip position, tip radius, velocity,
solute mass.

Restates, in numpy, the definitions of the reference's post-processing tools
(resources/PP_tools/tipradius.py: the phi = 0.5 contour of the solid, the point
farthest from the seed, a quadratic fit of the contour around it;
resources/PP_tools/frontvelocity.py: growth of the solid's extent between
snapshots divided by the time between them).  The reference uses scikit-image
contours; here the phi = 0.5 crossing is interpolated linearly between cell
centres along grid lines, which is what a marching-squares contour does on the
grid lines it crosses.

Fields are interior arrays phi[a][x][y] (the layout of include/gp_b200.h).
A dendrite seeded at the corner (0, 0) with mirror boundaries grows along +x and
+y; its tip along x lies on the row y = 0.
"""
from __future__ import annotations

import numpy as np


def crossing(profile: np.ndarray, level: float = 0.5) -> float:
    """Position of the last downward crossing of `level` along a 1-D profile
    (cell-centre coordinates), linearly interpolated; -1 if the profile never
    reaches the level."""
    above = np.nonzero(profile >= level)[0]
    if above.size == 0:
        return -1.0
    i = int(above[-1])
    if i + 1 >= profile.size:
        return float(i)
    a, b = float(profile[i]), float(profile[i + 1])
    if a == b:
        return float(i)
    return i + (a - level) / (a - b)


def tip_position(phi_solid: np.ndarray, axis: int = 0, line: int = 0, level: float = 0.5) -> float:
    """Tip of the solid along `axis` (0: x, on row y = line; 1: y, on column x = line)."""
    prof = phi_solid[:, line] if axis == 0 else phi_solid[line, :]
    return crossing(prof, level)


def tip_radius(phi_solid: np.ndarray, axis: int = 0, level: float = 0.5, rows: int = 6) -> float:
    """Radius of curvature at the tip along `axis`: the contour x(y) of the first
    `rows` grid lines next to the growth axis is fitted with x = x_tip - y^2/(2R)
    (the quadratic fit of tipradius.py, on the mirror-symmetric half dendrite)."""
    ys, xs = [], []
    for r in range(rows):
        prof = phi_solid[:, r] if axis == 0 else phi_solid[r, :]
        c = crossing(prof, level)
        if c < 0:
            break
        ys.append(float(r))
        xs.append(c)
    if len(ys) < 3:
        return float("nan")
    ys = np.array(ys)
    xs = np.array(xs)
    # mirror about the growth axis: y -> -y (the reference reflects the half dendrite the same way)
    Y = np.concatenate([-ys[:0:-1], ys])
    X = np.concatenate([xs[:0:-1], xs])
    a, b, c = np.polyfit(Y, X, 2)
    return float(-1.0 / (2.0 * a)) if a < 0 else float("inf")


def velocity(times: np.ndarray, positions: np.ndarray, window: int | None = None) -> float:
    """Growth velocity as the least-squares slope of position against time over
    the last `window` samples (all when None)."""
    t = np.asarray(times, dtype=np.float64)
    p = np.asarray(positions, dtype=np.float64)
    if window:
        t, p = t[-window:], p[-window:]
    return float(np.polyfit(t, p, 1)[0])


def solid_fraction(phi: np.ndarray, liquid: int = -1) -> float:
    """Mean of 1 - phi_liquid over the interior."""
    return float(1.0 - phi[liquid].mean())
