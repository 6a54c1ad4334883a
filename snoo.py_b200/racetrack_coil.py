"""Racetrack filament coils (``snoopy/racetrack_coil.py``).

A coil is 8 keypoints in the x-z plane: four straight segments kp7->kp0, kp1->kp2,
kp3->kp4, kp5->kp6 joined by quadratic B-spline arcs whose middle control point is
the intersection of the adjacent straight lines (``racetrack_coil.py:90-242``).  Each
turn is one copy of that loop at a height y.  ``compute_B`` evaluates Biot-Savart of
the segments through the drop-in ``fem_c.compute_B_line_segs_cpp`` (GPU).
"""

import numpy as np
from scipy.interpolate import BSpline


def compute_2D_line_intersection(intercept_1, slope_1, intercept_2, slope_2):
    """Intersection of two lines in 2-D (``racetrack_coil.py:14-42``)."""
    M = np.array([[slope_1[0], -slope_2[0]], [slope_1[1], -slope_2[1]]])
    b = np.array([intercept_2[0] - intercept_1[0], intercept_2[1] - intercept_1[1]])
    x_2 = np.linalg.solve(M, b)
    return slope_1 * x_2[0] + intercept_1


class RacetrackCoil:
    """Racetrack coil of filaments (``racetrack_coil.py:45-70``)."""

    def __init__(self, kp, y, rad, current=1.0):
        self.kp = np.asarray(kp, dtype=np.float64)
        self.y = np.asarray(y, dtype=np.float64)
        self.rad = float(rad)
        self.current = float(current)

    def compute_B(self, positions, disc_arc=5):
        """B at ``positions`` [M, 3] (``racetrack_coil.py:72-88``)."""
        from . import fem_c

        segs = self.get_segments(disc_arc=disc_arc)
        return fem_c.compute_B_line_segs_cpp(segs, positions, self.current, self.rad)

    def get_segments(self, disc_arc=5, enable_plot=False):
        """Segments [M, 6] (start xyz, end xyz), ``4*disc_arc + 4`` per turn."""
        kp = self.kp
        k = 2
        t = [0, 0, 0, 1, 1, 1]
        t_vec = np.linspace(0.0, 1.0, disc_arc + 1)
        segs_per_lvl = 4 * disc_arc + 4
        segs_base = np.zeros((segs_per_lvl, 6))

        def straight(row, a, b):
            segs_base[row, :3] = [kp[a, 0], 0.0, kp[a, 1]]
            segs_base[row, 3:] = [kp[b, 0], 0.0, kp[b, 1]]

        def arc(row0, a, b, prev_a, prev_b, next_a, next_b):
            ctrl = compute_2D_line_intersection(kp[prev_a, :], kp[prev_b, :] - kp[prev_a, :],
                                                kp[next_a, :], kp[next_b, :] - kp[next_a, :])
            cx = [kp[a, 0], ctrl[0], kp[b, 0]]
            cz = [kp[a, 1], ctrl[1], kp[b, 1]]
            sx = BSpline(t, cx, k)(t_vec)
            sz = BSpline(t, cz, k)(t_vec)
            for i in range(disc_arc):
                segs_base[row0 + i, :3] = [sx[i], 0.0, sz[i]]
                segs_base[row0 + i, 3:] = [sx[i + 1], 0.0, sz[i + 1]]

        straight(0, 7, 0)
        arc(1, 0, 1, 7, 0, 1, 2)
        straight(disc_arc + 1, 1, 2)
        arc(2 + disc_arc, 2, 3, 1, 2, 3, 4)
        straight(2 + 2 * disc_arc, 3, 4)
        arc(3 + 2 * disc_arc, 4, 5, 3, 4, 5, 6)
        straight(3 + 3 * disc_arc, 5, 6)
        arc(4 + 3 * disc_arc, 6, 7, 5, 6, 7, 0)

        out = []
        for yy in self.y:
            s = segs_base.copy()
            s[:, 1] = yy
            s[:, 4] = yy
            out.append(s)
        return np.concatenate(out, axis=0) if out else np.zeros((0, 6))

    def get_length(self, one_layer=True):
        segs = self.get_segments()
        lens = np.sqrt(((segs[:, 3:] - segs[:, :3]) ** 2).sum(axis=1))
        total = lens.sum()
        return total / len(self.y) if one_layer else total
