"""The plain-function API (python/zebsdsolve/api.py of the reference): one call per job, each
opening its own engine.

`scan` is an array of patterns shaped (rows, cols, h, w) or (n, h, w); `phases` are master
pattern files (ebsdsim .npz).  Keyword arguments naming a geometry field (pc, rot,
sample_tilt_deg, detector_tilt_deg, px_um, step_x_um, step_y_um) set the geometry; every other
keyword is a setting.
"""
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

GEOMETRY_FIELDS = ("pc", "rot", "sample_tilt_deg", "detector_tilt_deg", "px_um", "step_x_um", "step_y_um")


@dataclass
class Result:
    """Indexing results per map cell, with the geometry they were indexed under (api.py:22-47)."""

    quaternions: np.ndarray
    euler: np.ndarray
    ncc: np.ndarray
    nmi: np.ndarray
    phase: np.ndarray
    z: np.ndarray
    sweep: np.ndarray
    geometry: dict
    phases: list
    settings: dict
    fit: dict = field(default_factory=dict)


def _open(solver, scan, phases, kwargs):
    geo = {k: kwargs.pop(k) for k in list(kwargs) if k in GEOMETRY_FIELDS}
    roi = {k: kwargs.pop(k) for k in list(kwargs) if k in ("roi_x", "roi_y", "roi_w", "roi_h")}
    solver.configure(**kwargs)
    if isinstance(scan, (str, Path)) or (isinstance(scan, (list, tuple)) and scan and isinstance(scan[0], (str, Path))):
        solver.open(*([scan] if isinstance(scan, (str, Path)) else scan))
    else:
        solver.set_patterns(scan)
    if roi:
        solver.configure(**roi)
    if geo:
        solver.set_geometry(**geo)
    for p in [phases] if isinstance(phases, (str, Path)) else phases:
        solver.add_phase(p)


def load_patterns(scan, cells=None, processed=False, **settings):
    """Patterns of a scan file as float32 (n, h, w) (api.py:70-80): the given map cells
    (row-major indices; all of them by default), as stored or after the filters, at the size the
    `binning` setting reduces them to."""
    from . import Solver

    with Solver() as s:
        s.configure(**settings)
        s.open(*([scan] if isinstance(scan, (str, Path)) else scan))
        info = s.scan
        cells = range(info["rows"] * info["cols"]) if cells is None else cells
        return np.stack([s.pattern(int(c), processed) for c in cells])


def fit_pattern_center(scan, phases, **kwargs):
    """Fit the pattern centre by the voting search (api.py:83-93). Returns the fit's report (pc,
    score, start, …) with the last grid's votes under "scores", its axes under "axes" and the
    geometry it leaves under "geometry"."""
    from . import Solver

    s = Solver()
    try:
        _open(s, scan, phases, dict(kwargs))
        r = s.fit_pc()
        scores, x, y, z = s.pc_scores()
        r.update(scores=scores, axes=(x, y, z), geometry=s.geometry)
        return r
    finally:
        s.close()


def fit_plane(scan, phases, **kwargs):
    """Fit the plane of source points from the pattern centre as given (api.py:96-108). Returns the
    fit's report with the final "geometry" and the measured "points" (Solver.plane_points)."""
    from . import Solver

    s = Solver()
    try:
        _open(s, scan, phases, dict(kwargs))
        r = s.fit_plane()
        r.update(geometry=s.geometry, points=s.plane_points())
        return r
    finally:
        s.close()


def index(scan, phases, fit=None, progress=None, **kwargs):
    """Index a scan against candidate phases (api.py:111-132). fit: None indexes under the
    geometry as given; "geometry" first fits it by itself (Solver.fit_geometry: the vote for the
    pattern centre, then the plane of source points); "pc" fits the pattern centre by the vote."""
    from . import Solver

    if fit not in (None, "geometry", "pc"):
        raise ValueError('fit is None, "geometry" or "pc"')
    s = Solver()
    try:
        _open(s, scan, phases, dict(kwargs))
        report = {}
        if fit == "pc":
            report["pc"] = s.fit_pc()
        if fit == "geometry":
            report["geometry"] = s.fit_geometry()
        r = s.index(progress)
        return Result(geometry=s.geometry, phases=s.phases, settings=s.settings, fit=report, **r)
    finally:
        s.close()
