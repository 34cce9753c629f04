"""Detector pose and per-pattern source offset (oracle restatement of zebsdsolve `src/geometry.zig`).

x = R (row, col, 0) + t with R = R0(sample tilt, detector tilt) · Exp(rot) and
t = R (0.5 − pcy·rows, 0.5 − pcx·cols, pcz·rows) (geometry.zig:86-99).
"""
import math

import numpy as np

from . import rot


class Geometry:
    """geometry.zig:113-193"""

    def __init__(self, pc=(0.5, 0.5, 0.5), sample_tilt_deg=70.0, detector_tilt_deg=0.0, rot_vec=(0.0, 0.0, 0.0),
                 px_um=0.0, step_x_um=1.0, step_y_um=1.0):
        self.pc = np.array(pc, dtype=np.float64)
        self.sample_tilt_deg = float(sample_tilt_deg)
        self.detector_tilt_deg = float(detector_tilt_deg)
        self.rot = np.array(rot_vec, dtype=np.float64)
        self.px_um = float(px_um)
        self.step_x_um = float(step_x_um)
        self.step_y_um = float(step_y_um)

    def nominal(self):
        """geometry.zig:141-146"""
        a = math.radians(self.detector_tilt_deg - self.sample_tilt_deg)
        s, c = math.sin(a), math.cos(a)
        return np.array([[-s, 0, c], [0, 1, 0], [-c, 0, -s]], dtype=np.float64)

    def rotation(self):
        """geometry.zig:148-150"""
        return self.nominal() @ rot.to_mat(rot.so3_exp(self.rot))

    def translation(self, rows, cols):
        """geometry.zig:153-155"""
        return self.translation_for(self.pc, rows, cols)

    def translation_for(self, pc, rows, cols):
        """geometry.zig:159-161"""
        return self.rotation() @ np.array([0.5 - pc[1] * rows, 0.5 - pc[0] * cols, pc[2] * rows])

    @staticmethod
    def pc_of(R, t, rows, cols):
        """geometry.zig:171-174"""
        p = np.asarray(R).T @ np.asarray(t)
        return np.array([(0.5 - p[1]) / cols, (0.5 - p[0]) / rows, p[2] / rows])

    def pixel_angle(self, rows):
        """geometry.zig:178-180"""
        return 1.0 / max(self.pc[2] * rows, 1e-9)

    def scan_offset(self, row, col, ref_row, ref_col, x_sign, y_sign, binning):
        """geometry.zig:184-192"""
        if not (self.px_um > 0):
            return np.zeros(3)
        k = 1.0 / (self.px_um * binning)
        return np.array([y_sign * (row - ref_row) * self.step_y_um * k, x_sign * (col - ref_col) * self.step_x_um * k, 0.0])

    def position_for(self, row, col, ref_row, ref_col, x_sign, y_sign, binning, rows, cols):
        """geometry.zig:165-168 (no plane of source points)"""
        return self.translation(rows, cols) - self.scan_offset(row, col, ref_row, ref_col, x_sign, y_sign, binning)

    def frame(self):
        """engine.zig:1567-1578 — detector row direction c0, column direction c1, normal c2."""
        R = self.rotation()
        return R[:, 0].copy(), R[:, 1].copy(), R[:, 2].copy()


def mask_of(h, w, mask=True, mask_radius=1.0):
    """engine.zig:1444-1448 — mask centre (row, col) and squared radius (0: none)."""
    if not mask:
        return np.array([0.0, 0.0, 0.0])
    r = mask_radius * 0.5 * min(h, w)
    return np.array([0.5 * (h - 1), 0.5 * (w - 1), r * r])
