"""The reference's per-scan indexing schedule in FP64, from the oracle's pieces (test
infrastructure: the oracle that the parity tests and the bench's CPU leg run on a workload's own
patterns; nothing here is part of the product).

For one phase and one sweep without CLAHE, band pass or NLPAR (the configurations' settings):
  * the static background: the mean of `static_patterns` patterns on a lattice over the map
    (engine.zig:1325-1341 lattice, 1344-1424 average);
  * the master baked for the detector: the pixel's width on the master quantized in steps of 5 %
    (engine.zig:1674-1697), smoothed on the sphere by master_smooth of those pixels, then both
    sheets normalized together to mean 0 and variance 1 (engine.zig:1718-1788, prep.zig:215-237);
  * the gradient table of the baked sheets (prep.zig:253-260), the master's harmonics
    (master.zig:665-711), the phase's tables and the map-centre window's denominators
    (spherical.zig:204-241, 448-464);
  * per pattern: the filters (prep.zig:143-204), the coefficients (spherical.zig:319-361), the
    correlation volume times the denominators and its peak (spherical.zig:401-432), the
    Gauss–Newton refinement and NMI (detector.zig:178-202), and the record's orientation in the
    fundamental zone (engine.zig:2392-2419 with sym.zig:120-131).
"""
import math

import numpy as np

from . import detector as od
from . import geometry as og
from . import master as om
from . import prep as op
from . import spherical as osp
from . import sym as osym


def lattice(rows, cols, want):
    """engine.zig:1325-1341 — about `want` cells on a lattice over the map, row-major."""
    gy, gx = rows, cols
    if rows * cols > want:
        ratio = rows / cols
        gy = int(min(max(round(math.sqrt(want * ratio)), 1), rows))
        gx = int(min(max(want // gy, 1), cols))
    r = (2 * np.arange(gy) + 1) * rows // (2 * gy)
    c = (2 * np.arange(gx) + 1) * cols // (2 * gx)
    return (r[:, None] * cols + c[None, :]).reshape(-1).astype(np.int64)


def static_average(patterns, rows, cols, want=1024):
    """engine.zig:1344-1424 — the mean of the lattice's patterns (patterns: [rows·cols][h][w])."""
    cells = lattice(rows, cols, want)
    return np.asarray(patterns)[cells].astype(np.float64).mean(0)


def cell_positions(geo, rows, cols, cells, h, w, x_sign=1.0, y_sign=1.0, binning=1.0):
    """engine.zig:1601-1613 with geometry.zig:165-192 — each map cell's detector position
    (pixels): the map-centre cell's less the beam's travel from it (none without a pixel size)."""
    cells = np.asarray(cells, np.int64)
    return np.stack([geo.position_for(c // cols, c % cols, 0.5 * (rows - 1), 0.5 * (cols - 1), x_sign, y_sign, binning,
                                      h / binning, w / binning) for c in cells])


def pixel_angle(geo, h, binning=1.0, pixel_angle_deg=0.0):
    """engine.zig:1028-1035 — a detector pixel's angular width, radians."""
    if pixel_angle_deg > 0:
        return math.radians(pixel_angle_deg) * binning
    return 1.0 / max(geo.pc[2] * h, 1e-9) * binning


def bake(raw, side, angle, master_smooth=0.3):
    """engine.zig:1674-1788 without CLAHE and band pass — the sheets smoothed on the sphere by
    master_smooth detector pixels (the pixel's width on the master, sqrt(2π)/side per sheet pixel,
    quantized to powers of 1.05), then normalized together."""
    px = angle * side / math.sqrt(2 * math.pi)
    sheets = np.asarray(raw, np.float64).reshape(-1)
    if px > 0:
        q = int(math.floor(math.log(px) / math.log(1.05) + 0.5))
        smooth = master_smooth * 1.05 ** q
        if smooth > 0.05:
            sheets = od.sphere_blur(sheets, side, smooth)
    mean = sheets.mean()
    sd = math.sqrt(((sheets - mean) ** 2).mean())
    return (sheets - mean) / max(sd, 1e-30)


class Scan:
    """What a scan's indexing shares across its patterns (FP64, the oracle's)."""

    def __init__(self, raw_sheets, side, ops, geo, h, w, L, static_bg=None, dynamic="subtract", dynamic_sigma=0.15,
                 mask_radius=1.0, master_smooth=0.3, refine=True, refine_iters=8, refine_step_deg=2.0, nmi_bins=16,
                 baked=None):
        self.side, self.h, self.w, self.L = side, h, w, L
        self.geo = geo
        self.frame = geo.frame()
        self.mask = og.mask_of(h, w, True, mask_radius)
        self.static = None if static_bg is None else np.asarray(static_bg, np.float64)
        self.dynamic = dynamic
        self.sigma = dynamic_sigma * w if dynamic != "none" else 0.0
        self.refine_on, self.iters, self.max_step, self.nmi_bins = refine, refine_iters, math.radians(refine_step_deg), nmi_bins
        self.sheets = bake(raw_sheets, side, pixel_angle(geo, h), master_smooth) if baked is None else np.asarray(
            baked, np.float64).reshape(-1)
        m = om.Master(side, self.sheets.astype(np.float32), ops)
        m.measure_symmetry()
        self.rotations = np.asarray(m.rotations(), np.float64)
        self.grad = od.gradient_table(self.sheets, side)
        self.tb = osp.Tables(L)
        self.hm = om.Harmonics(m, self.sheets, L)
        self.pt = osp.PhaseTables(self.tb, self.hm, om.fold_of(self.hm.rules))
        t0 = geo.translation(h, w)
        walm, wst = osp.coefficients(self.tb, None, t0, self.frame, self.mask, flags=osp.FLAG_WINDOW, shape=(h, w))
        self.rden = osp.window_denominators(self.tb, self.pt, walm, wst[0])
        self.t0 = t0

    def index(self, raw, t=None):
        """One stored pattern [h][w] at detector position t (the map centre's by default): the
        record (q in the fundamental zone (w, x, y, z), NCC, NMI, last improving step) and the
        spherical peak (q, score)."""
        t = self.t0 if t is None else np.asarray(t, np.float64)
        pat = op.run(raw, static=self.static, dynamic=self.dynamic, dynamic_sigma=self.sigma, mask=self.mask)
        g, _ = osp.coefficients(self.tb, pat, t, self.frame, self.mask)
        vol = osp.correlation_volume(self.tb, self.pt, self.hm.f, g) * self.rden
        q, v0, _, _ = osp.peak(self.tb, self.pt, vol)
        iters = self.iters if self.refine_on else 0
        qb, best, step = od.refine(self.grad, self.side, self.frame, t, q, pat, self.mask, iters=iters,
                                   max_step=self.max_step)
        nmi = od.nmi(self.sheets, self.side, self.frame, t, qb, pat, self.mask, self.nmi_bins)
        return {"q": osym.to_fz(np.asarray(qb, np.float64), self.rotations), "ncc": float(best), "nmi": float(nmi), "step": float(step),
                "peak_q": np.asarray(q, np.float64), "peak_score": float(v0)}


_STATE = {}


def _init(scan):
    _STATE["scan"] = scan


def _one(job):
    raw, t = job
    return _STATE["scan"].index(raw, t)


def index_many(scan, raws, ts=None, workers=None, limit=1800.0):
    """Scan.index over the stored patterns `raws` (at detector positions `ts`, default the map
    centre's) in a spawn pool of `workers` processes (default: every core this process may use,
    at most 64), one thread each. One pattern per worker goes first, untimed (imports, caches).
    Returns (records, seconds of the timed map, workers); a map that takes more than `limit`
    seconds raises."""
    import multiprocessing as mp
    import os
    import time

    # one thread per worker: the workers' BLAS and FFT pools would otherwise each take every core
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS"):
        os.environ[k] = "1"
    raws = list(zip(raws, [None] * len(raws) if ts is None else list(ts)))
    workers = max(1, min(workers or len(os.sched_getaffinity(0)), 64, len(raws)))
    osp._wigner_blocks(scan.tb)  # built once here and shipped to the workers with the rest
    with mp.get_context("spawn").Pool(workers, initializer=_init, initargs=(scan,)) as pool:
        pool.map_async(_one, [raws[i % len(raws)] for i in range(workers)], chunksize=1).get(limit)
        t0 = time.perf_counter()
        out = pool.map_async(_one, raws, chunksize=1).get(limit)
        return out, time.perf_counter() - t0, workers
