"""The indexing engine: the reference's Engine (zebsdsolve src/engine.zig) for the spherical path,
driving the C-ABI kernels on one GPU.

State: the settings, the detector geometry, the scan (patterns on the host), the candidate phases
(masters, baked per pattern resolution on the device), the per-bandwidth tables, the chance
calibration and the per-cell results.  Indexing goes in batches of cells, each batch one pass of
the device path: upload → preprocess → sphere → spectrum → peaks → refine → NMI → records, one
readback (engine.zig:2005-2137).
"""
import ctypes
import json
import math

import numpy as np
import torch

from . import _native as N
from . import dictionary as DI
from .reduce import reduce_image
from . import master as M
from . import rotations as R
from .device import BandTables, PhaseBand, master_blur, ptr, stream_ptr
from .settings import Settings

FLAG_CENTER, FLAG_NORM, FLAG_WINDOW = 1, 2, 4


class EngineError(RuntimeError):
    pass


class Geometry:
    """geometry.zig:113-193 — one detector pose, per-cell beam offsets, and (after a plane fit)
    the plane of source points that replaces them: plane_kind 0 none, 1 affine, 2 projective;
    plane P (12, row-major 4 × 3) with P · (column, row, 1) = w · (PCx, PCy, PCz, 1)."""

    FIELDS = ("pc", "sample_tilt_deg", "detector_tilt_deg", "rot", "px_um", "step_x_um", "step_y_um")
    KINDS = ("none", "affine", "projective")

    def __init__(self):
        self.pc = np.array([0.5, 0.5, 0.5])
        self.sample_tilt_deg = 70.0
        self.detector_tilt_deg = 0.0
        self.rot = np.zeros(3)
        self.px_um = 0.0
        self.step_x_um = 1.0
        self.step_y_um = 1.0
        self.plane_kind = 0
        self.plane = np.zeros(12)

    def copy(self):
        g = Geometry()
        g.__dict__.update({k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        return g

    def as_dict(self):
        return {"pc": list(map(float, self.pc)), "sample_tilt_deg": self.sample_tilt_deg,
                "detector_tilt_deg": self.detector_tilt_deg, "rot": list(map(float, self.rot)), "px_um": self.px_um,
                "step_x_um": self.step_x_um, "step_y_um": self.step_y_um, "plane_kind": self.KINDS[self.plane_kind],
                "plane": [list(map(float, self.plane[3 * k:3 * k + 3])) for k in range(4)]}

    def set(self, **kw):
        for k, v in kw.items():
            if k in ("pc", "rot"):
                a = np.asarray(v, np.float64).reshape(3)
                setattr(self, k, a)
            elif k in self.FIELDS:
                setattr(self, k, float(v))
            elif k == "plane_kind":
                self.plane_kind = self.KINDS.index(v) if isinstance(v, str) else int(v)
            elif k == "plane":
                self.plane = np.asarray(v, np.float64).reshape(12).copy()
            else:
                raise EngineError(f"geometry has no field {k!r}")

    def given(self, kw, given):
        """exports.zig:131-155 — set_geometry's fields: a pattern centre set by hand (changed,
        with no other plane given) is one for the whole map again, the scan's steps saying how the
        beam went from it; the fields the caller changed are recorded in `given` (the geometry an
        automatic fit starts from)."""
        was = self.copy()
        self.set(**kw)
        pc_changed = not np.array_equal(self.pc, was.pc)
        if pc_changed and np.array_equal(self.plane, was.plane) and self.plane_kind == was.plane_kind:
            self.plane_kind = 0
        for k in self.FIELDS:
            a, b = getattr(self, k), getattr(was, k)
            if not np.array_equal(a, b):
                setattr(given, k, a.copy() if isinstance(a, np.ndarray) else a)

    def key(self):
        return (tuple(self.pc), self.sample_tilt_deg, self.detector_tilt_deg, tuple(self.rot), self.px_um,
                self.step_x_um, self.step_y_um, self.plane_kind, tuple(self.plane) if self.plane_kind else ())

    def nominal(self):
        """geometry.zig:141-146 — R0(sample tilt, detector tilt)."""
        a = math.radians(self.detector_tilt_deg - self.sample_tilt_deg)
        s, c = math.sin(a), math.cos(a)
        return np.array([[-s, 0, c], [0, 1, 0], [-c, 0, -s]])

    def rotation(self):
        """geometry.zig:141-150 — R0(sample tilt, detector tilt) · Exp(rot)."""
        return self.nominal() @ R.to_matrix(R.exp_map(self.rot))

    def translation(self, rows, cols, pc=None):
        """geometry.zig:153-161 — t in pixels for a pattern of rows × cols."""
        pc = self.pc if pc is None else pc
        return self.rotation() @ np.array([0.5 - pc[1] * rows, 0.5 - pc[0] * cols, pc[2] * rows])

    def scan_offsets(self, row, col, ref_row, ref_col, x_sign, y_sign, binning):
        """geometry.zig:184-192 — beam travel of cells from the reference cell, in pixels."""
        row = np.asarray(row, np.float64)
        col = np.asarray(col, np.float64)
        if not self.px_um > 0:
            return np.zeros(row.shape + (3,))
        k = 1.0 / (self.px_um * binning)
        return np.stack([y_sign * (row - ref_row) * self.step_y_um * k, x_sign * (col - ref_col) * self.step_x_um * k,
                         np.zeros_like(row)], -1)


class Phase:
    def __init__(self, master):
        self.master = master
        self.baked = None  # (key, sheets, grad4, value pairs, gradient pairs), all on the device
        self.bakes = {}    # the last few of them by smoothing key (detector sizes met before)
        self.quads = {}    # each bake's FP16 neighbourhood records (zeb_master_quads), by the same key

    def info(self, bands):
        m = self.master
        out = {"name": m.name, "side": m.side, "point_group": m.point_group, "space_group": m.space_group,
               "laue": R.LAUE_NAMES[m.laue], "rotations": len(m.rotations()), "voltage_kv": m.voltage_kv,
               "n_fold": 0, "mirror": False, "inversion": False}
        return out


class Engine:
    def __init__(self, device=None):
        if not torch.cuda.is_available():
            raise EngineError("no CUDA device: this engine runs only on the GPU")
        N.load()
        self.dev = torch.device(device or "cuda")
        self.set = Settings()
        self.geo = Geometry()
        self.patterns = None  # host array [rows, cols, h, w]
        self.pixel = None
        self.phases = []
        self.bands = {}
        self.avg = None
        self.chance_key = None
        self.chance_med = []
        self.chance_spread = []
        self.batch_stamp = 0
        self.events = []
        self.cancel = False
        self.res = None
        self.index_cells_list = None
        self.index_done = 0
        self.index_sweep = 0
        self.index_accepted = 0
        self.index_region = 0
        self._buf = {}
        self._batch_t = None  # bounding box of the last batch's detector positions
        self._spans = {}
        self.dicts = {}  # (phase, grid) → dictionary.Dictionary
        self._stage, self._stage_next = {}, {}  # page-locked staging rings of to_device
        self.tuned = {}  # what tune() chose for the way work is cut up (device_batch)
        self._pinned = None
        self._pin_buf = None  # the page-locked buffer behind _pinned, reused across scans
        self._index_calls = 0  # whole passes over the scan since set_patterns (whole_pinned)
        self._ring, self._ring_i = [], 0  # two page-locked slots a scan not pinned whole streams through
        self._last_fz = None  # the last index_cells' records in the fundamental zones, their Bunge angles
        self.pending_skip = 0  # batches whose readback is dropped (host-side fault injection)
        self.counts = {"submits": 0, "reads": 0, "waits": 0}  # device passes, readbacks, host waits
        self._full = False  # at_full: the stored size is the level being worked at
        self._resident = None  # the scan's filtered patterns a whole pass kept on the device (prepared)
        self._whole_pass = False  # an indexing run over the scan is under way (its batches are kept)
        self.geo_given = Geometry()  # the geometry as given (set_geometry), where a full fit starts
        self._nl_view = None  # what averaging with neighbours did to the last pattern looked at
        self._nl_report = False  # log what the averaging did to the next batch (an indexing run's first)
        self.pc_history = []  # the grids of the last pattern-centre vote (pcfit.run)
        self.plane_points = None  # the source points of the last plane fit
        self.fit = None  # the last fit's patterns: cells, orientations, phases, scores

    # ── plumbing ──

    def log(self, text):
        self.events.append({"kind": "log", "text": text})

    def buf(self, name, numel, dtype=torch.float32):
        t = self._buf.get(name)
        if t is None or t.numel() < numel or t.dtype != dtype:
            t = torch.empty(max(int(numel), 1), dtype=dtype, device=self.dev)
            self._buf[name] = t
        return t

    # ── scan ──

    def set_patterns(self, a):
        a = np.asarray(a)
        if a.ndim == 3:
            a = a[None]
        if a.ndim != 4:
            raise EngineError("patterns must be (rows, cols, h, w) or (n, h, w)")
        if a.dtype == np.uint8:
            self.pixel = 0
        elif a.dtype == np.uint16:
            self.pixel = 1
        else:
            a = a.astype(np.float32)
            self.pixel = 2
        if a.shape[2] < 4 or a.shape[3] < 4:
            raise EngineError("PatternTooSmall")
        self.patterns = np.ascontiguousarray(a)
        self.scan_source = None  # the file the patterns came from (Solver.open), if any
        self.convention = None  # the orientation convention the exports write in (None: the engine's own)
        self.told_no_background = False
        self._pinned = None
        self._index_calls = 0
        if self._resident is not None:
            self._resident["key"] = None  # (its buffer is kept for the next scan, as the page-locked one)
        rows, cols = a.shape[:2]
        self.avg = None
        self.chance_key = None
        self.res = {"quat": np.zeros((rows * cols, 4), np.float32), "ncc": np.zeros(rows * cols, np.float32),
                    "nmi": np.zeros(rows * cols, np.float32), "phase": np.full(rows * cols, -1, np.int32),
                    "z": np.zeros(rows * cols, np.float32), "sweep": np.full(rows * cols, -1, np.int32),
                    "settled": np.zeros(rows * cols, bool)}
        self.res["quat"][:, 0] = 1
        self.res["euler"] = np.zeros((rows * cols, 3), np.float32)  # Bunge angles of quat, kept as cells land

    def info(self):
        if self.patterns is None:
            raise EngineError("NoScan")
        rows, cols, h, w = self.patterns.shape
        return rows, cols, h, w

    # ── levels (engine.zig:990-1035): the patterns reduced by settings.binning, and as stored ──

    def factor(self):
        """The reduction of the level being worked at: settings.binning, or 1 inside at_full."""
        return 1.0 if self._full else float(self.set["binning"])

    def at_full(self):
        """A context in which everything that depends on the level (the pattern's size, the frame,
        the detector positions, the static background, the filters' widths, the master's bake,
        the chance calibration) is the stored size's (engine.zig Level.full)."""
        import contextlib

        @contextlib.contextmanager
        def ctx():
            was = self._full
            self._full = True
            try:
                yield
            finally:
                self._full = was

        return ctx()

    def stage_full(self, stage):
        """engine.zig:996-1003 — whether a stage ("search", "refine", "score") works at the stored
        size: never when nothing is reduced; settings.full_resolution "scores" puts the scores
        there, "refine" the refinement and the scores."""
        if self.set["binning"] == 1:
            return False
        mode = self.set["full_resolution"]
        return (mode == "scores" and stage == "score") or (mode == "refine" and stage != "search")

    def pattern_shape(self):
        """engine.zig:1011-1017 — the level's size floor(size / factor)."""
        rows, cols, h, w = self.info()
        b = self.factor()
        return int(math.floor(h / b)), int(math.floor(w / b))

    def mask_of(self, h, w):
        """engine.zig:1444-1448"""
        if not self.set["mask"]:
            return (0.0, 0.0, 0.0)
        r = self.set["mask_radius"] * 0.5 * min(h, w)
        return (0.5 * (h - 1), 0.5 * (w - 1), r * r)

    def frame(self):
        """engine.zig:1567-1578"""
        h, w = self.pattern_shape()
        Rm = self.geo.rotation()
        fr = N.Frame()
        fr.h, fr.w = h, w
        for k in range(3):
            fr.c0[k], fr.c1[k], fr.c2[k] = Rm[k, 0], Rm[k, 1], Rm[k, 2]
        fr.mask[0], fr.mask[1], fr.mask[2] = self.mask_of(h, w)
        return fr

    def positions(self, cells, geo=None):
        """engine.zig:1601-1613 — the detector position for each cell, in pixels (float32)."""
        return self.positions64(cells, geo).astype(np.float32)

    def positions64(self, cells, geo=None):
        """The detector position for each cell (FP64; geometry.zig:80-83): the plane of source
        points' where the geometry has one, else the reference cell's less the beam's travel."""
        rows, cols, h, w = self.info()
        b = self.factor()
        g = self.geo if geo is None else geo
        cells = np.asarray(cells, np.int64)
        if g.plane_kind:
            from .plane import at

            pc = at(g.plane, cells // cols, cells % cols)  # [n][3]
            Rm = g.rotation()
            v = np.stack([0.5 - pc[:, 1] * (h / b), 0.5 - pc[:, 0] * (w / b), pc[:, 2] * (h / b)], 1)
            return v @ Rm.T
        t = g.translation(h / b, w / b)
        off = g.scan_offsets(cells // cols, cells % cols, 0.5 * (rows - 1), 0.5 * (cols - 1),
                             self.set["scan_x_sign"], self.set["scan_y_sign"], b)
        return t[None, :] - off

    def lattice(self, want):
        """engine.zig:1325-1341 — about `want` cells on a lattice over the map."""
        rows, cols = self.info()[:2]
        gy, gx = rows, cols
        if rows * cols > want:
            ratio = rows / cols
            gy = int(min(max(round(math.sqrt(want * ratio)), 1), rows))
            gx = int(min(max(want // gy, 1), cols))
        r = (2 * np.arange(gy) + 1) * rows // (2 * gy)
        c = (2 * np.arange(gx) + 1) * cols // (2 * gx)
        return (r[:, None] * cols + c[None, :]).reshape(-1).astype(np.int64)

    def region_cells(self):
        """engine.zig:2312-2330"""
        rows, cols = self.info()[:2]
        s = self.set
        x0, y0, w, h = 0, 0, cols, rows
        if s["roi_w"] and s["roi_h"]:
            x0 = min(s["roi_x"], cols - 1)
            y0 = min(s["roi_y"], rows - 1)
            w = min(s["roi_w"], cols - x0)
            h = min(s["roi_h"], rows - y0)
        return ((y0 + np.arange(h))[:, None] * cols + x0 + np.arange(w)[None, :]).reshape(-1).astype(np.int64)

    def static_background(self):
        """engine.zig:1344-1424 — the average of `static_patterns` lattice patterns; "file": the
        background the scan file stores (none where it stores none); "none"."""
        kind = self.set["static_background"]
        if kind == "file":
            src = (getattr(self, "scan_source", None) or {}).get("background")
            if src is None:
                if not getattr(self, "told_no_background", False):
                    self.log('static background: this scan stores none, so none is subtracted '
                             '(static_background: "average" takes the patterns\' own)')
                    self.told_no_background = True
                return None
            key = ("file", id(src), self.factor())
            if self.avg is None or self.avg[0] != key:
                avg = reduce_image(np.asarray(src, np.float64), self.factor()).astype(np.float32)
                self.avg = (key, torch.as_tensor(avg, device=self.dev))
            return self.avg[1]
        if kind != "average":
            return None
        key = ("average", self.set["static_patterns"], self.factor())
        if self.avg is None or self.avg[0] != key:
            cells = self.lattice(self.set["static_patterns"])
            rows, cols, h, w = self.info()
            n = len(cells)
            if self.pixel in (0, 1):
                # integer pixels: the sum is an exact integer in any order, so the device sums the
                # lattice's patterns (one copy of them, gathered on the host threads)
                raw = self.buf("static_raw", n * h * w, self.raw_dtype())[: n * h * w].view(n, h, w)
                self.upload_raw(cells, raw, torch.cuda.current_stream())
                x = raw.view(n, h * w)
                x = (x.view(torch.int16).to(torch.int32) & 0xFFFF) if self.pixel == 1 else x.to(torch.int32)
                acc = x.sum(0, dtype=torch.int64).view(h, w).cpu().numpy().astype(np.float64)
            else:
                flat = self.patterns.reshape(rows * cols, h, w)
                acc = np.zeros((h, w))
                for i in range(0, n, 1024):
                    acc += flat[cells[i:i + 1024]].sum(0, dtype=np.float64)
            avg = reduce_image(acc / n, self.factor()).astype(np.float32)
            self.avg = (key, torch.as_tensor(avg, device=self.dev))
            self.log(f"static background: the average of {len(cells)} patterns over the map")
        return self.avg[1]

    # ── phases ──

    def add_phase(self, path):
        return self.add_master(M.load_npz(path))

    def add_master(self, m):
        self.phases.append(Phase(m))
        self.chance_key = None
        self.log(f"phase {len(self.phases) - 1}: {m.name} ({m.side} px), orientations reduced by {len(m.rotations())} rotations")
        return len(self.phases) - 1

    def clear_phases(self):
        self.phases = []
        self.bands = {}
        self.dicts = {}
        self.chance_key = None

    def default_px(self):
        """engine.zig:948-956 — the detector's pixel size (µm) when none is set by hand: the scan
        file's, else the detector's width (settings.detector_width_mm) over the pattern's stored
        pixels across; 0 with no scan."""
        if self.patterns is None:
            return 0.0
        px = ((getattr(self, "scan_source", None) or {}).get("px_um")) or 0.0
        if px > 0:
            return float(px)
        return 1000.0 * float(self.set["detector_width_mm"]) / max(self.info()[3], 1)

    def pixel_angle(self):
        """engine.zig:1028-1035 — angular width of one reduced pixel, radians (0 before any scan is
        set, unless pixel_angle_deg gives it: the master is then baked unsmoothed)."""
        if self.patterns is None and not self.set["pixel_angle_deg"] > 0:
            return 0.0
        stored = (math.radians(self.set["pixel_angle_deg"]) if self.set["pixel_angle_deg"] > 0
                  else 1.0 / max(self.geo.pc[2] * self.info()[2], 1e-9))
        return stored * self.factor()

    def bake_key(self, p):
        """engine.zig:1674-1697 — what a phase's master must be filtered for: the smoothing (its
        pixel's width quantized in steps of 5 %), and the patterns' own band pass and CLAHE at the
        sizes they have on the sphere (CLAHE's tiles as wide as the patterns' are)."""
        s = self.set
        angle = self.pixel_angle()
        m = p.master
        px = angle * m.side / math.sqrt(2 * math.pi)
        if not px > 0:
            return (None, s["master_smooth"], False, 0.0, 0.0, False, 0, 0, 0.0)
        q = int(math.floor(math.log(px) / math.log(1.05) + 0.5))
        f = self.factor()
        fine, coarse = (s["bp_fine"] / f, s["bp_coarse"] / f) if s["bandpass"] else (0.0, 0.0)
        tiles = bins = 0
        clip = 0.0
        if s["clahe"]:
            tile = self.pattern_shape()[0] / s["clahe_grid"] * px
            tiles = int(min(max(math.floor(m.side / tile + 0.5), 1), 64))
            bins, clip = s["clahe_bins"], s["clahe_clip"]
        return (q, s["master_smooth"], bool(s["bandpass"]), fine, coarse, bool(s["clahe"]), tiles, bins, clip)

    def prepare_masters(self):
        """engine.zig:1699-1788 — each phase's master filtered as the patterns are (smoothed on the
        sphere by master_smooth pattern pixels; CLAHE on the sheets then the mean over the point
        group; the band pass as a difference of two smoothings on the sphere), the two sheets
        normalized together, and its gradient and pair tables."""
        if not self.phases:
            raise EngineError("NoPhases")
        for p in self.phases:
            m = p.master
            key = self.bake_key(p)
            if p.baked is not None and p.baked[0] == key:
                continue
            if key in p.bakes:  # a detector size or level met before: its master as baked then (the
                p.baked = p.bakes[key]  # chance calibration's key names each phase's bake)
                continue
            sheets = self.bake(p, key)
            grad = torch.empty(sheets.numel() * 4, dtype=torch.float32, device=self.dev)
            N.call("zeb_master_gradient", ptr(sheets), ptr(grad), m.side, stream_ptr())
            vpair = torch.empty(sheets.numel() * 2, dtype=torch.float32, device=self.dev)
            gpair = torch.empty(sheets.numel() * 8, dtype=torch.float32, device=self.dev)
            N.call("zeb_master_pairs", ptr(sheets), ptr(grad), m.side, ptr(vpair), ptr(gpair), stream_ptr())
            # the BF16 form's refinement table: each texel's 2 × 2 neighbourhood in FP16, one record
            quads = torch.empty(sheets.numel() * 32, dtype=torch.uint8, device=self.dev)
            N.call("zeb_master_quads", ptr(grad), m.side, ptr(quads), stream_ptr())
            p.quads[key] = quads
            p.baked = (key, sheets, grad, vpair, gpair)
            if len(p.bakes) >= 8:
                p.quads.pop(p.bakes.pop(next(iter(p.bakes)))[0], None)
            p.bakes[key] = p.baked
            self.chance_key = None

    def bake(self, p, key):
        """engine.zig:1738-1788 — the master's sheets filtered for `key` (bake_key), on the device."""
        m = p.master
        side = m.side
        q, smooth0, bandpass, fine0, coarse0, clahe, tiles, bins, clip = key
        sheets = torch.as_tensor(m.raw, device=self.dev)
        if q is None:
            return sheets
        pxq = 1.05 ** q
        smooth = smooth0 * pxq
        if not (smooth > 0.05 or bandpass or clahe):
            return sheets
        fine = fine0 * pxq
        if clahe:
            sheets = master_blur(sheets, side, smooth).contiguous()
            scratch = torch.empty(N.load().zeb_clahe_scratch_bytes(2, tiles, bins) // 4 + 1, dtype=torch.float32,
                                  device=self.dev)
            N.call("zeb_clahe", ptr(sheets), 2, side, side, tiles, bins, float(clip), ptr(scratch), stream_ptr())
            if len(m.ops) > 1:
                # CLAHE on the sheets as images does not respect the crystal's symmetry: the mean over
                # the master's own point group
                ops = torch.as_tensor(np.asarray(m.ops, np.float32).reshape(-1), device=self.dev)
                out = torch.empty_like(sheets)
                N.call("zeb_master_symmetrize", ptr(sheets), ptr(out), side, ptr(ops), len(m.ops), stream_ptr())
                sheets = out
        else:
            # what the pixel averages and the band pass's fine Gaussian compose into one
            fine = math.sqrt(smooth * smooth + fine * fine)
            if not bandpass:
                sheets = master_blur(sheets, side, smooth)
        if bandpass:
            low = master_blur(sheets.clone(), side, coarse0 * pxq)
            sheets = master_blur(sheets, side, fine) - low
        host = sheets.double()
        mean = host.mean()
        sd = torch.sqrt(((host - mean) ** 2).mean())
        return ((host - mean) / torch.clamp(sd, min=1e-30)).float().contiguous()

    def band(self, L):
        """engine.zig:1793-1836 — the tables of bandwidth L and every phase's, built on first use."""
        self.prepare_masters()
        b = self.bands.get(L)
        if b is None:
            b = {"tables": BandTables(L, self.dev), "phases": {}}
            self.bands[L] = b
        prec = self.set["precision"]
        cache = b.setdefault("cache", {})
        for i, p in enumerate(self.phases):
            key = (id(p.baked[1]), prec)
            pb = b["phases"].get(i)
            if pb is None or pb[0] != key:
                hit = cache.get((i, key))
                if hit is not None:
                    b["phases"][i] = (key, hit)
                    continue
                ph = PhaseBand(b["tables"], p.baked[1], p.master.side, L, prec)
                if len(cache) >= 16:
                    cache.pop(next(iter(cache)))
                cache[(i, key)] = ph
                b["phases"][i] = (key, ph)
                r = ph.rules
                self.log(f"phase {i}: bandwidth {L}, rotation order {r.n_fold} about z{', mirror' if r.mirror else ''}"
                         f"{', inversion' if r.inversion else ''}")
        return b

    def denominators(self, b, fr):
        """engine.zig:1839-1849, spherical.zig:448-464 — each phase's reciprocal denominator
        volume for the map-centre geometry (cached per geometry)."""
        rows, cols, h, w = self.info()
        bn = self.factor()
        t = self.geo.translation(h / bn, w / bn).astype(np.float32)
        key = (tuple(fr.c0), tuple(fr.c1), tuple(fr.c2), fr.h, fr.w, tuple(fr.mask), tuple(t))
        bt = b["tables"]
        for i, (k, ph) in b["phases"].items():
            if ph.rden_key == key:
                continue
            items = torch.as_tensor(np.array([[t[0], t[1], t[2], 0.0]], np.float32), device=self.dev)
            alm = torch.empty(bt.n_pairs * 2, dtype=torch.float32, device=self.dev)
            stats = torch.empty(4, dtype=torch.float32, device=self.dev)
            scratch = self.buf("sphere_scratch", N.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), 1) // 4 + 1)
            N.call("zeb_sphere_coefficients", None, ptr(items), 1, ctypes.byref(fr), ctypes.byref(bt.st), FLAG_WINDOW,
                   ptr(alm), ptr(stats), ptr(scratch), stream_ptr())
            cells = ph.volume_cells()
            vols = []
            for Y in (ph.Y_f, ph.Y_f2):
                U = self.buf("spec_window", N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), 1) // 4 + 1)
                self.spectrum(alm, 1, ph, Y, U, tensor_cores=False)
                vol = torch.empty(cells, dtype=torch.float32, device=self.dev)
                N.call("zeb_correlate_volume", ptr(U), 1, ctypes.byref(ph.dims), ptr(bt.tw), ptr(vol), stream_ptr())
                vols.append(vol)
            rden = torch.empty(cells, dtype=torch.float32, device=self.dev)
            N.call("zeb_rden_build", ptr(vols[0]), ptr(vols[1]), ptr(stats), 1, cells, ptr(rden), stream_ptr())
            ph.rden = rden
            ph.rden_key = key

    def spectrum(self, alm, n, ph, Y, U, tensor_cores=True):
        """spherical.zig:369-382 — U of n items: on the tensor cores (BF16 form) when the phase
        has its packed table, else in plain FP32."""
        if tensor_cores and ph.A is not None and Y is ph.Y_f:
            B = self.buf("tc_b", N.load().zeb_tc_patterns_bytes(ctypes.byref(ph.dims), ph.split, n), torch.uint8)
            N.call("zeb_spectrum_bf16", ptr(alm), n, ctypes.byref(ph.dims), ph.split, ptr(ph.A), ptr(B), ptr(U),
                   ptr(self.tc_status()), stream_ptr())
        else:
            N.call("zeb_spectrum_f32", ptr(alm), n, ctypes.byref(ph.dims), ptr(Y), ptr(U), stream_ptr())

    def tc_status(self):
        """One int on the device that a timed-out wait in the tensor-core spectrum sets."""
        t = self._buf.get("tc_status")
        if t is None:
            t = torch.zeros(1, dtype=torch.int32, device=self.dev)
            self._buf["tc_status"] = t
        return t

    def check_device(self):
        """After a readback: raise if a tensor-core spectrum gave up on a wait (its U incomplete)."""
        t = self._buf.get("tc_status")
        if t is not None:
            v = int(t.item())
            if v:
                t.zero_()
                raise EngineError(f"DeviceTimeout: tensor-core spectrum wait gave up (status {v})")

    # ── device passes ──

    def prep_options(self):
        h, w = self.pattern_shape()
        s = self.set
        dyn = {"none": 0, "subtract": 1, "divide": 2}[s["dynamic_background"]]
        sigma = s["dynamic_sigma"] * w if dyn else 0.0
        return dyn, sigma

    # ── averaging with neighbours (NLPAR) ──

    NLPAR_BYTES = 256 << 20  # one copy of a window's patterns on the device at most (engine.zig:1196)

    def nlpar_window(self, wanted):
        """engine.zig:1201-1258 — the cells averaging `wanted` needs: the wanted ones, then ring
        after ring of the map's cells around them (8-neighbourhoods) out to radius · passes + 1;
        counts[d] cells lie within d rings; nbr[k][slot] the list index of the cell at each offset
        up to radius · passes each way (rows first), 0xffffffff outside the map or the list."""
        rows, cols = self.info()[:2]
        R, P = int(self.set["nlpar_radius"]), int(self.set["nlpar_iterations"])
        wanted = np.asarray(wanted, np.int64)
        index = np.full(rows * cols, -1, np.int64)
        first = np.unique(wanted, return_index=True)[1]
        lst = [wanted[np.sort(first)]]
        index[lst[0]] = np.arange(len(lst[0]))
        counts = [len(lst[0])]
        grid = np.zeros((rows, cols), bool)
        grid.reshape(-1)[lst[0]] = True
        total = counts[0]
        for _ in range(R * P + 1):
            d = grid.copy()
            d[1:] |= grid[:-1]
            d[:-1] |= grid[1:]
            e = d.copy()
            e[:, 1:] |= d[:, :-1]
            e[:, :-1] |= d[:, 1:]
            new = np.flatnonzero((e & ~grid).reshape(-1))
            index[new] = total + np.arange(len(new))
            total += len(new)
            lst.append(new)
            counts.append(total)
            grid = e
        cells = np.concatenate(lst)
        r = R * P
        off = np.arange(-r, r + 1)
        y = (cells // cols)[:, None, None] + off[None, :, None]
        x = (cells % cols)[:, None, None] + off[None, None, :]
        inside = (y >= 0) & (y < rows) & (x >= 0) & (x < cols)
        at = np.where(inside, index[np.clip(y, 0, rows - 1) * cols + np.clip(x, 0, cols - 1)], -1)
        nbr = np.where(at >= 0, at, 0xFFFFFFFF).astype(np.uint32).reshape(len(cells), -1)
        return cells, counts, nbr

    def nlpar_average(self, cells, account=False):
        """engine.zig:1504-1553 — the cells' stored patterns averaged with their neighbours on the
        device (loaded at the reduced size, not yet filtered): [n·h·w] float32. In parts when a
        window's patterns would pass NLPAR_BYTES. account: keep what the averaging did to the
        first cell (its noise, the share of it left, its own share, its shares), for nlpar_view."""
        s = self.set
        rows, cols, sh, sw = self.info()
        h, w = self.pattern_shape()
        px = h * w
        cells = np.asarray(cells, np.int64)
        n = len(cells)
        R, P = int(s["nlpar_radius"]), int(s["nlpar_iterations"])
        F = (2 * R * P + 1) ** 2
        out = self.buf("nl_out", max(n, 1) * px)
        most = max(1, self.NLPAR_BYTES // (px * 4))
        t0, guess = 0, n
        mask = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
        while t0 < n:
            m = min(n - t0, guess)
            lst, counts, nbr = self.nlpar_window(cells[t0:t0 + m])
            while m > 1 and len(lst) > most:
                m = (m + 1) // 2
                lst, counts, nbr = self.nlpar_window(cells[t0:t0 + m])
            guess = 2 * m
            nw = len(lst)
            raw = self.buf("nl_raw", nw * sh * sw, self.raw_dtype())[: nw * sh * sw].view(nw, sh, sw)
            self.upload_raw(lst, raw, torch.cuda.current_stream())
            loaded = self.buf("nl_loaded", nw * px)
            sb = N.load().zeb_prep_scratch_bytes(nw, h, w, 0.0)
            N.call("zeb_prep_reduced", ptr(raw), self.pixel, nw, sh, sw, self.factor(), None, 0, 0.0, mask, 0,
                   ptr(loaded), ptr(self.buf("prep_scratch", sb // 4 + 1) if sb else None), stream_ptr())
            nbr_d = self.to_device("nl_nbr", nbr)
            cnt = (ctypes.c_int * len(counts))(*counts)
            scratch = self.buf("nl_scratch", N.load().zeb_nlpar_scratch_bytes(nw, px, R, P) // 4 + 1)
            sig = shares = None
            report = self._nl_report and t0 == 0
            if (account or report) and t0 == 0:
                sig = torch.empty(counts[R * P], dtype=torch.float32, device=self.dev)
                shares = torch.empty(counts[0] * F, dtype=torch.float32, device=self.dev)
            N.call("zeb_nlpar", ptr(loaded), px, ptr(nbr_d), cnt, R, P, float(s["nlpar_lambda"]), ptr(out[t0 * px:]),
                   ptr(sig), ptr(shares), ptr(scratch), stream_ptr())
            if sig is not None:
                sg, sh_ = sig.cpu().numpy(), shares.cpu().numpy()
                if account:
                    self._nl_view = self._nlpar_view(sg, sh_[:F], nbr[0], R * P)
                if report:
                    self._nl_report = False
                    self._log_nlpar(sg, sh_, nbr, counts[0], F)
            t0 += m
        return out[: n * px]

    def _log_nlpar(self, sig, shares, nbr, n, F):
        """engine.zig:1285-1321 — what the averaging did to a batch's n cells, logged: the stored
        patterns' noise (a pixel's standard deviation), the share of it an average keeps and the
        share of an average that is the pattern itself, each a mean over the cells."""
        s = self.set
        noise = kept = own = counted = 0.0
        for c in range(n):
            sh_ = shares[c * F:(c + 1) * F].astype(np.float64)
            nb = nbr[c]
            inside = nb != 0xFFFFFFFF
            before = float(sig[c])
            after = float((sh_[inside] ** 2 * sig[nb[inside].astype(np.int64)]).sum())
            own += sh_[F // 2]
            if not before > 0:
                continue
            noise += math.sqrt(before)
            kept += math.sqrt(after / before)
            counted += 1
        P, R = int(s["nlpar_iterations"]), int(s["nlpar_radius"])
        self.log(f"neighbour averaging: {P} pass{'' if P == 1 else 'es'} over {2 * R + 1} × {2 * R + 1} cells "
                 f"(λ {s['nlpar_lambda']:.2f}); noise about {noise / max(counted, 1):.2f} a pixel, "
                 f"{100 * kept / max(counted, 1):.0f} % of it left; an average is {100 * own / max(n, 1):.0f} % the "
                 f"pattern itself")

    @staticmethod
    def _nlpar_view(sig, share, nbr0, reach):
        """engine.zig:1285-1306 for one average: the stored pattern's noise (a pixel's standard
        deviation), the share of it the average keeps, the average's own share, and its shares of
        the stored patterns around it (NaN outside the map)."""
        side = 2 * reach + 1
        inside = nbr0 != 0xFFFFFFFF
        before = float(sig[0])
        after = float((share[inside].astype(np.float64) ** 2 * sig[nbr0[inside].astype(np.int64)]).sum())
        grid = np.where(inside, share, np.nan).reshape(side, side).astype(np.float32)
        return {"noise": float(np.sqrt(before)) if before > 0 else 0.0,
                "left": float(np.sqrt(after / before)) if before > 0 else 0.0,
                "own": float(share[len(share) // 2]), "shares": grid}

    def pattern(self, cell, stage, full=False):
        """exports.zig ze_pattern — one cell's pattern (float32 [h, w]) at the reduced size, or
        (full) the stored one: stage 0 as stored, 1 as indexed (averaged when nlpar is on, then
        filtered), 2 averaged with its neighbours and not filtered, 3 the static background."""
        rows, cols, sh, sw = self.info()
        h, w = self.pattern_shape()
        if full and (h, w) != (sh, sw) and stage != 0:
            with self.at_full():  # the filters (and the background) at the stored size's level
                return self.pattern(cell, stage, False)
        self._nl_view = None
        if stage == 3:
            bg = self.static_background()
            if bg is None:
                raise EngineError("NoStaticBackground")
            return bg.reshape(h, w).cpu().numpy()
        cells = np.array([int(cell)], np.int64)
        if not 0 <= cells[0] < rows * cols:
            raise EngineError("CellOutOfRange")
        if stage == 1:
            if self.set["nlpar"]:
                avg = self.nlpar_average(cells, account=True)
                view = self._nl_view
                out = self.filter_chain(avg, 2, 1, h, w, 1.0)
                self._nl_view = view
            else:
                out = self.upload(cells)
            return out[: h * w].reshape(h, w).cpu().numpy()
        if stage == 2 and self.set["nlpar"]:
            return self.nlpar_average(cells, account=True)[: h * w].reshape(h, w).cpu().numpy()
        raw = self.buf("raw_up", sh * sw, self.raw_dtype())[: sh * sw].view(1, sh, sw)
        self.upload_raw(cells, raw, torch.cuda.current_stream())
        oh, ow = (sh, sw) if full else (h, w)
        out = torch.empty(oh * ow, dtype=torch.float32, device=self.dev)
        mask = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
        N.call("zeb_prep_reduced", ptr(raw), self.pixel, 1, sh, sw, 1.0 if full else float(self.set["binning"]), None, 0,
               0.0, mask, 0, ptr(out), None, stream_ptr())
        return out.reshape(oh, ow).cpu().numpy()

    def preprocess(self, raw, n, cells=None, out=None):
        """engine.zig:1452-1563, prep.zig:143-204 — n stored patterns on the device (raw, the scan's
        pixel type) through the filter chain into the float32 pattern buffer (or `out`): with nlpar,
        first averaged with their neighbours (the cells' windows read from the scan); static
        background, dynamic background, CLAHE, band pass, then the mask and the normalization."""
        rows, cols, sh, sw = self.info()
        h, w = self.pattern_shape()  # reduced by binning as the patterns are unpacked
        s = self.set
        if s["nlpar"]:
            if cells is None:
                raise EngineError("nlpar: the cells of the patterns are needed to average them with their neighbours")
            raw = self.nlpar_average(cells)
            return self.filter_chain(raw, 2, n, h, w, 1.0, out=out)
        return self.filter_chain(raw, self.pixel, n, sh, sw, self.factor(), out=out)

    def filter_chain(self, raw, pixel, n, sh, sw, factor, out_name="pats", out=None):
        """prep.zig:143-204 — n patterns (pixel type, stored size sh × sw reduced by factor) through
        static background, dynamic background, CLAHE, band pass, mask and normalization, into the
        buffer `out_name` (or `out`, n·h·w float32 on the device)."""
        h, w = self.pattern_shape()
        s = self.set
        out = self.buf(out_name, n * h * w) if out is None else out
        static = self.static_background()
        dyn, sigma = self.prep_options()
        mask = (ctypes.c_float * 3)(*self.mask_of(h, w))
        bandpass = s["bandpass"] and s["bp_coarse"] > 0
        extra = s["clahe"] or bandpass

        def run(src, pixel, sh_, sw_, factor, bg, dyn_, sigma_, normalize, dst):
            sb = N.load().zeb_prep_scratch_bytes(n, h, w, sigma_)
            scratch = self.buf("prep_scratch", sb // 4 + 1) if sb else None
            N.call("zeb_prep_reduced", ptr(src), pixel, n, sh_, sw_, factor, ptr(bg), dyn_, sigma_, mask, normalize,
                   ptr(dst), ptr(scratch), stream_ptr())

        if not extra:
            run(raw, pixel, sh, sw, factor, static, dyn, sigma, 1, out)
            return out
        cur = self.buf("prep_cur", n * h * w)
        run(raw, pixel, sh, sw, factor, static, dyn, sigma, 0, cur)
        if s["clahe"]:
            cs = self.buf("clahe_scratch", N.load().zeb_clahe_scratch_bytes(n, s["clahe_grid"], s["clahe_bins"]) // 4 + 1)
            N.call("zeb_clahe", ptr(cur), n, h, w, s["clahe_grid"], s["clahe_bins"], float(s["clahe_clip"]), ptr(cs),
                   stream_ptr())
        if bandpass:
            f = self.factor()
            fine, coarse = s["bp_fine"] / f, s["bp_coarse"] / f
            low = self.buf("prep_low", n * h * w)
            run(cur, 2, h, w, 1.0, None, 3, coarse, 0, low)
            if fine > 0.05:
                high = self.buf("prep_high", n * h * w)
                run(cur, 2, h, w, 1.0, None, 3, fine, 0, high)
            else:
                high = cur
            N.call("zeb_combine", ptr(high), ptr(low), ptr(cur), n * h * w, 0, stream_ptr())
        run(cur, 2, h, w, 1.0, None, 0, 0.0, 1, out)
        return out

    RESIDENT_FRAC = 0.25  # of the device's memory: the most the kept filtered scan may take

    def _prep_key(self):
        """What the filter chain's output depends on: the scan, every setting, the level."""
        return (self.patterns.shape, self.set.to_json(), self._full, self.pattern_shape(), self.factor())

    def _resident_buffer(self):
        """The kept filtered scan's buffer for the current scan and settings (made, or re-keyed with
        no row valid, when they changed), or None where the scan does not fit RESIDENT_FRAC of the
        device's memory."""
        rows, cols = self.info()[:2]
        h, w = self.pattern_shape()
        total = rows * cols * h * w
        key = self._prep_key()
        r = self._resident
        if r is None or r["key"] != key:
            if total * 4 > self.RESIDENT_FRAC * torch.cuda.get_device_properties(self.dev).total_memory:
                self._resident = None
                return None
            old = r["pats"] if r is not None and r["pats"].numel() >= total else None
            self._resident = None
            r = {"key": key, "pats": old if old is not None else torch.empty(total, dtype=torch.float32, device=self.dev),
                 "valid": np.zeros(rows * cols, bool)}
            self._resident = r
        return r

    def resident_rows(self, cells):
        """Where a whole pass over a run of consecutive cells filters its patterns in place: those
        cells' rows of the kept filtered scan (a flat view), or None (scattered cells, or a scan too
        large to keep), for which keep_prepared copies the filtered batch instead."""
        c = np.asarray(cells, np.int64)
        n = len(c)
        if n == 0 or c[-1] - c[0] != n - 1 or (n > 1 and not (np.diff(c) == 1).all()):
            return None
        r = self._resident_buffer()
        if r is None:
            return None
        rows, cols = self.info()[:2]
        h, w = self.pattern_shape()
        view = r["pats"][: rows * cols * h * w].view(rows * cols, h * w)
        return view[int(c[0]):int(c[0]) + n].reshape(-1)

    def filter_pass(self, raw, n, cells):
        """preprocess for a device pass; a whole pass keeps its filtered patterns (in place for a
        run of consecutive cells, else copied by keep_prepared)."""
        direct = self.resident_rows(cells) if self._whole_pass else None
        pats = self.preprocess(raw, n, cells, out=direct)
        if direct is not None:
            self._resident["valid"][np.asarray(cells, np.int64)] = True
        elif self._whole_pass:
            self.keep_prepared(pats, cells)
        return pats

    def keep_prepared(self, pats, cells):
        """A whole pass's filtered patterns kept on the device, the scan's rows [cell][h·w] in FP32,
        where the scan fits RESIDENT_FRAC of the device's memory: what refine_patterns then starts
        from without uploading and filtering the patterns again (prepared)."""
        r = self._resident_buffer()
        if r is None:
            return
        rows, cols = self.info()[:2]
        h, w = self.pattern_shape()
        total = rows * cols * h * w
        n = len(cells)
        view = r["pats"][:total].view(rows * cols, h * w)
        src = pats[: n * h * w].view(n, h * w)
        c = np.asarray(cells, np.int64)
        if n and c[-1] - c[0] == n - 1 and (n == 1 or (np.diff(c) == 1).all()):
            view[int(c[0]):int(c[0]) + n].copy_(src)
        else:
            view.index_copy_(0, torch.as_tensor(c, device=self.dev), src)
        r["valid"][c] = True

    def prepared(self, cells):
        """The cells' patterns as the filter chain leaves them: the rows a whole pass kept on the
        device (keep_prepared) where they hold every cell under the current settings, a view for a
        run of consecutive cells; else uploaded and filtered (upload)."""
        r = self._resident
        c = np.asarray(cells, np.int64)
        n = len(c)
        if r is not None and n and r["key"] == self._prep_key() and r["valid"][c].all():
            rows, cols = self.info()[:2]
            h, w = self.pattern_shape()
            view = r["pats"][: rows * cols * h * w].view(rows * cols, h * w)
            if c[-1] - c[0] == n - 1 and (n == 1 or (np.diff(c) == 1).all()):
                return view[int(c[0]):int(c[0]) + n].reshape(-1)
            out = self.buf("pats_kept", n * h * w)[: n * h * w].view(n, h * w)
            torch.index_select(view, 0, torch.as_tensor(c, device=self.dev), out=out)
            return out.reshape(-1)
        return self.upload(cells)

    def upload(self, cells):
        """The cells' stored patterns to the device (from the pinned scan), preprocessed."""
        rows, cols, h, w = self.info()
        n = len(cells)
        raw = self.buf("raw_up", max(n, 1) * h * w, self.raw_dtype())[: n * h * w].view(n, h, w)
        self.upload_raw(cells, raw, torch.cuda.current_stream())
        return self.preprocess(raw, n, cells)

    def prepare(self, bandwidth=None, method="spherical", grid=None):
        """Everything a batch needs besides its patterns: tables, chance calibration, denominators
        (spherical), or each phase's dictionary (its simulated entries or components)."""
        if method != "spherical":
            self.prepare_masters()
            for pi in range(len(self.phases)):
                self.dictionary(pi, int(grid or self.set["dict_grid"]), method)
            self.calibrate_at_score_level()
            self.prepare_masters()
            return None
        L = int(bandwidth or self.set["bandwidth"])
        b = self.band(L)
        self.calibrate_at_score_level()
        self.prepare_masters()  # (the search level's bake)
        self.denominators(b, self.frame())
        return b

    def calibrate_at_score_level(self):
        """What chance gives, measured where the scores are taken (engine.zig:2250)."""
        if self.stage_full("score"):
            with self.at_full():
                self.calibrate()
        else:
            self.calibrate()

    def dictionary(self, pi, grid, method):
        """engine.zig:1851-1955 — phase pi's dictionary of this grid, simulated at the map's
        reference position (method "dictionary") or learned as components ("pca"); kept until the
        master, the geometry, the grid or the settings change."""
        p = self.phases[pi]
        d = self.dicts.get((pi, grid))
        if d is None:
            q = DI.cubochoric_grid(grid, p.master.rotations())
            d = DI.Dictionary(q, self.dev)
            self.dicts[(pi, grid)] = d
            self.log(f"dictionary: {d.n} orientations for the rotations {p.master.setting.rotation} (grid {grid})")
        rows, cols, h, w = self.info()
        bn = self.factor()
        t = self.geo.translation(h / bn, w / bn).astype(np.float32)
        fr = self.frame()
        s = self.set
        key = (method, id(p.baked[1]), tuple(fr.c0), tuple(fr.c1), tuple(fr.c2), fr.h, fr.w, tuple(fr.mask),
               tuple(t), s["pca_components"] if method == "pca" else 0, s["pca_epochs"] if method == "pca" else 0)
        if d.key != key:
            _, sheets, grad, vpair, gpair = p.baked
            d.key, d.panel = None, None
            if method == "pca":
                d.prepare_pca(fr, vpair, p.master.side, t, s["pca_components"], s["pca_epochs"], self.log)
            else:
                d.prepare_sims(fr, vpair, p.master.side, t)
            d.key = key
        return d

    def to_device(self, name, arr):
        """A small host array on the device without stalling the host: copied into one of a ring of
        page-locked buffers and from there asynchronously on the current stream (a copy from
        pageable memory would wait for all the work queued before it)."""
        arr = np.ascontiguousarray(arr)
        ring = self._stage.setdefault(name, [])
        k = self._stage_next.get(name, 0)
        self._stage_next[name] = (k + 1) % 4
        while len(ring) <= k:
            ring.append([None, None])
        slot = ring[k]
        nbytes = arr.nbytes
        if slot[0] is None or slot[0].numel() < nbytes:
            slot[0] = torch.empty(max(nbytes, 1 << 16), dtype=torch.uint8, pin_memory=True)
            slot[1] = None
        if slot[1] is not None:
            slot[1].synchronize()  # the copy that last read this buffer (four uses ago) is done
        host = slot[0][:nbytes].view(torch.from_numpy(arr).dtype).view(arr.shape)
        host.numpy()[...] = arr
        dev = torch.empty(arr.shape, dtype=host.dtype, device=self.dev)
        dev.copy_(host, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream())
        slot[1] = ev
        return dev

    def items_of(self, cells):
        """The cells' items (detector position in pixels, index in the batch) on the device, and
        their positions' bounding box in _batch_t."""
        cells = np.asarray(cells, np.int64)
        n = len(cells)
        fast = self._items_separable(cells) if n and not self.geo.plane_kind else None
        if fast is not None:
            items, self._batch_t = fast
            return self.to_device("items", items)
        t = self.positions(cells)
        if len(t):
            tt = np.ascontiguousarray(t.T)  # (a reduction along the long axis of a contiguous array)
            self._batch_t = (tt.min(1), tt.max(1))
        else:
            self._batch_t = None
        return self.to_device("items", np.concatenate([t, np.arange(len(cells), dtype=np.float32)[:, None]], 1))

    def _items_separable(self, cells):
        """items_of without a plane of source points, for a run of consecutive cells: the beam's
        travel is a row's plus a column's (geometry.zig:184-192), so each row's and each column's
        position is computed once, by positions64's arithmetic, and gathered (the same float32
        values); the box from the rows and columns the run reaches. None for scattered cells."""
        n = len(cells)
        if cells[-1] - cells[0] != n - 1 or (n > 1 and not (np.diff(cells) == 1).all()):
            return None
        rows, cols, h, w = self.info()
        b = self.factor()
        g = self.geo
        t = g.translation(h / b, w / b)
        ref_r, ref_c = 0.5 * (rows - 1), 0.5 * (cols - 1)
        sx, sy = self.set["scan_x_sign"], self.set["scan_y_sign"]
        prow = (t[0] - g.scan_offsets(np.arange(rows), np.zeros(rows), ref_r, ref_c, sx, sy, b)[:, 0]).astype(np.float32)
        pcol = (t[1] - g.scan_offsets(np.zeros(cols), np.arange(cols), ref_r, ref_c, sx, sy, b)[:, 1]).astype(np.float32)
        pz = np.float32(t[2] - 0.0)
        r, c = np.divmod(cells, cols)
        items = np.empty((n, 4), np.float32)
        items[:, 0] = prow[r]
        items[:, 1] = pcol[c]
        items[:, 2] = pz
        items[:, 3] = np.arange(n, dtype=np.float32)
        r0, r1, c0, c1 = int(r[0]), int(r[-1]), int(c[0]), int(c[-1])
        rr = prow[r0:r1 + 1]
        if r1 == r0:
            cc = pcol[c0:c1 + 1]
        elif r1 == r0 + 1 and c1 + 1 < c0:
            cc = np.concatenate([pcol[c0:], pcol[:c1 + 1]])
        else:
            cc = pcol
        box = (np.array([rr.min(), cc.min(), pz], np.float32), np.array([rr.max(), cc.max(), pz], np.float32))
        return items, box

    def spans(self, bt, fr):
        """The sphere's ring spans for the detector positions of the last items_of batch: the
        corners of their bounding box, two samples of margin (cached per geometry and box)."""
        if self._batch_t is None:
            return None
        lo, hi = self._batch_t
        key = (bt.L, tuple(fr.c0), tuple(fr.c1), tuple(fr.c2), fr.h, fr.w, tuple(fr.mask),
               tuple(np.round(lo, 3)), tuple(np.round(hi, 3)))
        hit = self._spans.get(key)
        if hit is not None:
            return hit
        if len(self._spans) > 64:
            self._spans = {}
        corners = np.array([[x, y, z, 0.0] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])],
                           np.float32)
        ts = self.to_device("corners", corners)
        sp = torch.empty(bt.n_theta * 2, dtype=torch.int32, device=self.dev)
        N.call("zeb_sphere_spans", ctypes.byref(fr), ctypes.byref(bt.st), ptr(ts), len(corners), 2, ptr(sp),
               stream_ptr())
        self._spans[key] = sp
        return sp

    def run_device(self, raw, cells, bandwidth=None, timer=None, method="spherical", grid=None, pre=None):
        """One pass of the device path over n = len(cells) stored patterns already on the device:
        records [phase][cell][8] as a device tensor (engine.zig:2005-2122, no readback). pre: the
        cells' items already on the device with their bounding box (items_of's two results), as
        index_pipelined copies them ahead of the pass's patterns."""
        self.counts["submits"] += 1
        if method != "spherical":
            return self.run_device_dictionary(raw, cells, method, int(grid or self.set["dict_grid"]), timer)
        n = len(cells)
        n_ph = len(self.phases)
        s = self.set
        b = self.prepare(bandwidth)
        fr = self.frame()
        mark = timer.mark if timer is not None else (lambda name: None)
        mark("prep")
        pats = self.filter_pass(raw, n, cells)
        if pre is not None:
            items, self._batch_t = pre
        else:
            items = self.items_of(cells)
        self.batch_stamp = self.batch_stamp % (1 << 24) + 1
        bt = b["tables"]
        recs = self.buf("recs", n_ph * n * 8)
        alm = self.buf("alm", n * bt.n_pairs * 2)
        stats = self.buf("stats", n * 4)
        sphere_scratch = self.buf("sphere_scratch", N.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), n) // 4 + 1)
        mark("sphere")
        spans = self.spans(bt, fr)
        N.call("zeb_sphere_coefficients_spans", ptr(pats), ptr(items), n, ctypes.byref(fr), ctypes.byref(bt.st),
               ptr(spans), FLAG_CENTER | FLAG_NORM, ptr(alm), ptr(stats), ptr(sphere_scratch), stream_ptr())
        opts = N.RefineOpts(s["refine_iters"] if s["refine"] else 0, math.radians(s["refine_step"]), 1.0, 0.02, 1e4,
                            s["nmi_bins"], float(self.batch_stamp))
        self._seeds = []
        for pi, p in enumerate(self.phases):
            ph = b["phases"][pi][1]
            peaks = self.buf(f"peaks{pi}" if self.stage_full("refine") else "peaks", n * 8)
            self._seeds.append(peaks)
            tile = self.tile_items(ph, n)
            for t0 in range(0, n, tile):
                nt = min(tile, n - t0)
                a0 = alm[t0 * bt.n_pairs * 2:]
                cand = self.buf("cand", N.load().zeb_peaks_scratch_bytes(ctypes.byref(ph.dims), nt) // 4 + 1)
                if ph.u_scale is not None:
                    # the BF16 form: the spectrum in FP16, the transform along a on the tensor cores
                    U16 = self.buf("spec16", N.load().zeb_spectrum_h_bytes(ctypes.byref(ph.dims), nt), torch.uint8)
                    B = self.buf("tc_b", N.load().zeb_tc_patterns_bytes(ctypes.byref(ph.dims), ph.split, nt), torch.uint8)
                    mark("spectrum")
                    N.call("zeb_spectrum_bf16_h", ptr(a0), nt, ctypes.byref(ph.dims), ph.split, ptr(ph.A), ptr(B),
                           ptr(U16), ph.u_scale, ptr(self.tc_status()), stream_ptr())
                    mark("peaks")
                    N.call("zeb_correlate_peaks_h", ptr(U16), nt, ctypes.byref(ph.dims), ph.u_scale, ptr(ph.rden),
                           ptr(peaks[t0 * 8:]), ptr(cand), ptr(self.tc_status()), stream_ptr())
                    continue
                U = self.buf("spec", N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), nt) // 4 + 1)
                mark("spectrum")
                self.spectrum(a0, nt, ph, ph.Y_f, U)
                mark("peaks")
                N.call("zeb_correlate_peaks", ptr(U), nt, ctypes.byref(ph.dims), ptr(bt.tw), ptr(ph.rden), 1 << 30,
                       ptr(peaks[t0 * 8:]), ptr(cand), stream_ptr())
            mark("refine")
            if not self.stage_full("refine"):
                self.refine(pats, items, peaks, n, fr, p, opts, recs[pi * n * 8:])
        self.finish_levels(raw, cells, pats, items, fr, recs, opts)
        mark("end")
        return recs[: n_ph * n * 8].view(n_ph, n, 8)

    def finish_levels(self, raw, cells, pats, items, fr, recs, opts):
        """engine.zig:2101-2119 — with settings.full_resolution "refine", each phase's refinement
        from its search seeds (self._seeds), with "scores", the refined records scored again (no
        step), at the stored size: the patterns filtered at that size, the detector positions and
        frame in its pixels, each phase's master baked for it. The records are written into recs."""
        lr, lc = self.stage_full("refine"), self.stage_full("score")
        if not (lr or lc):
            return
        n = len(cells)
        rows, cols, sh, sw = self.info()
        with self.at_full():
            self.prepare_masters()
            fp = self.filter_chain(raw, self.pixel, n, sh, sw, 1.0, out_name="pats_full") if not self.set["nlpar"] \
                else self.preprocess(raw, n, cells)
            t = self.positions(cells)
            fi = self.to_device("items_full", np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1))
            ff = self.frame()
            for pi, p in enumerate(self.phases):
                out = recs[pi * n * 8:]
                if lr:
                    self.refine(fp, fi, self._seeds[pi], n, ff, p, opts, out)
                else:  # the refined orientations scored again at the stored size (no step)
                    seeds = self.buf("rescore_seeds", n * 8)
                    seeds[: n * 8].copy_(out[: n * 8])
                    sc = N.RefineOpts(0, opts.max_step, opts.scale0, opts.scale_min, opts.scale_max, opts.nmi_bins,
                                      opts.stamp)
                    self.refine(fp, fi, seeds, n, ff, p, sc, out)
        self.prepare_masters()  # (back to the search level's bake)

    def run_device_dictionary(self, raw, cells, method, grid, timer=None):
        """run_device with a dictionary search (engine.zig:2094-2112): each pattern's best entry
        (by its pixels, or by its coefficients on the components) seeds the refinement."""
        n = len(cells)
        n_ph = len(self.phases)
        s = self.set
        self.prepare(None, method, grid)
        fr = self.frame()
        mark = timer.mark if timer is not None else (lambda name: None)
        mark("prep")
        pats = self.filter_pass(raw, n, cells)
        items = self.items_of(cells)
        self.batch_stamp = self.batch_stamp % (1 << 24) + 1
        recs = self.buf("recs", n_ph * n * 8)
        opts = N.RefineOpts(s["refine_iters"] if s["refine"] else 0, math.radians(s["refine_step"]), 1.0, 0.02, 1e4,
                            s["nmi_bins"], float(self.batch_stamp))
        x = pats[: n * fr.h * fr.w].view(n, fr.h * fr.w)
        tc = s["precision"] != "f32"
        self._seeds = []
        for pi, p in enumerate(self.phases):
            d = self.dictionary(pi, grid, method)
            mark("match")
            xs = d.project(x, tc, self.tc_status()) if method == "pca" else x  # their coefficients (pca.zig:159-162)
            peaks = d.seeds(xs.contiguous(), tc, self.tc_status(),
                            self.buf(f"peaks{pi}" if self.stage_full("refine") else "peaks", n * 8))
            self._seeds.append(peaks)
            mark("refine")
            if not self.stage_full("refine"):
                self.refine(pats, items, peaks, n, fr, p, opts, recs[pi * n * 8:])
        self.finish_levels(raw, cells, pats, items, fr, recs, opts)
        mark("end")
        return recs[: n_ph * n * 8].view(n_ph, n, 8)

    def mask_list(self, fr):
        """The frame's masked pixels in raster order on the device (zeb_mask_list), cached per
        frame; None when the list is beyond the list kernel (zeb_refine then takes the frame)."""
        key = (fr.h, fr.w, tuple(fr.mask))
        hit = getattr(self, "_mask_list", None)
        if hit is not None and hit[0] == key:
            return hit[1]
        npix = N.load().zeb_mask_pixels(ctypes.byref(fr))
        lst = None
        if 1 <= npix <= 25600:
            lst = torch.empty(npix, dtype=torch.int32, device=self.dev)
            N.call("zeb_mask_list", ctypes.byref(fr), ptr(lst), stream_ptr())
        self._mask_list = (key, lst)
        return lst

    def refine(self, pats, items, peaks, n, fr, p, opts, out):
        """detector.zig:178-202 — every item refined from its seed (peaks, stride 8) and scored;
        in the BF16 form from the FP16 neighbourhood records (zeb_refine_list_h)."""
        key, sheets, grad, vpair, gpair = p.baked
        lst = self.mask_list(fr)
        quads = p.quads.get(key) if self.set["precision"] == "bf16" else None
        if lst is not None and quads is not None:
            N.call("zeb_refine_list_h", ptr(pats), ptr(items), ptr(peaks), 8, n, ctypes.byref(fr), ptr(lst),
                   lst.numel(), ptr(vpair), ptr(quads), p.master.side, ctypes.byref(opts), ptr(out), stream_ptr())
        elif lst is not None:
            N.call("zeb_refine_list", ptr(pats), ptr(items), ptr(peaks), 8, n, ctypes.byref(fr), ptr(lst), lst.numel(),
                   ptr(vpair), ptr(gpair), p.master.side, ctypes.byref(opts), ptr(out), stream_ptr())
        else:
            N.call("zeb_refine", ptr(pats), ptr(items), ptr(peaks), 8, n, ctypes.byref(fr), ptr(vpair), ptr(gpair),
                   p.master.side, ctypes.byref(opts), ptr(out), stream_ptr())

    def pinned(self):
        """The stored patterns in page-locked host memory ([cell][h][w], the scan's pixel type),
        copied once per set_patterns: every upload is then a plain DMA from it."""
        if self._pinned is None:
            rows, cols, h, w = self.info()
            src = torch.from_numpy(self.patterns.reshape(rows * cols, h, w))
            nbytes = src.numel() * src.element_size()
            # one page-locked buffer kept across scans, grown when a scan needs more (allocating
            # page-locked memory per scan costs more than many small scans' indexing)
            if self._pin_buf is None or self._pin_buf.numel() < nbytes:
                self._pin_buf = None
                self._pin_buf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            torch.cuda.synchronize(self.dev)  # no copy from the buffer is still pending
            self._pinned = self._pin_buf[:nbytes].view(src.dtype).view(src.shape)
            self._pinned.copy_(src)
        return self._pinned

    STAGE_BYTES = 64 << 20
    PIN_MAX_BYTES = 16 << 30
    # more runs of consecutive cells than this are gathered into a staging slot on the host (one
    # copy) rather than copied run by run (one copy each)
    PINNED_RUNS = 32

    def raw_dtype(self):
        """The stored pixel type as a torch dtype."""
        return torch.from_numpy(np.zeros(1, self.patterns.dtype)).dtype

    def whole_pinned(self):
        """Whether uploads come from a page-locked copy of the whole scan: when it is made already,
        when the buffer kept from earlier scans holds it (no page-locking to pay), or from the
        scan's second index run on (a scan indexed once streams through the staging slots:
        page-locking gigabytes for one run costs more than the run). A scan above PIN_MAX_BYTES
        always streams: locking tens of gigabytes takes longer than a pass and holds that much of
        the host's memory twice."""
        if self._pinned is not None:
            return True
        nbytes = self.patterns.size * self.patterns.itemsize
        if nbytes > self.PIN_MAX_BYTES:
            return False
        return (self._pin_buf is not None and self._pin_buf.numel() >= nbytes) or self._index_calls >= 2

    def _slot(self):
        if not self._ring:
            self._ring = [[torch.empty(self.STAGE_BYTES, dtype=torch.uint8, pin_memory=True), None] for _ in range(2)]
        slot = self._ring[self._ring_i]
        self._ring_i ^= 1
        if slot[1] is not None:
            slot[1].synchronize()  # the copy that last read this slot has finished
        return slot

    FILL_PART = 4 << 20

    def _fill(self, host, src):
        """host[:] = src (a staging slot from the stored scan) in parts of FILL_PART bytes on a
        pool of host threads: numpy copies without the interpreter lock, and one thread's copy
        bandwidth, not the link's, bounds a streamed scan."""
        nb = src.nbytes
        parts = min(self._fill_threads(), max(1, nb // self.FILL_PART))
        if parts <= 1:
            np.copyto(host, src)
            return
        step = -(-len(src) // parts)
        futs = [self._pool.submit(np.copyto, host[i:i + step], src[i:i + step]) for i in range(0, len(src), step)]
        for f in futs:
            f.result()

    def _gather(self, host, flat, part):
        """host[:] = flat[part] (scattered cells into a staging slot) on the same pool of host
        threads; the cells are checked against the scan first, so that none is read out of it."""
        if len(part) and (part.min() < 0 or part.max() >= len(flat)):
            raise EngineError(f"cells outside the scan of {len(flat)} patterns")
        parts = min(self._fill_threads(), max(1, host.nbytes // self.FILL_PART))
        step = -(-len(part) // parts)
        futs = [self._pool.submit(np.take, flat, part[i:i + step], 0, host[i:i + step], "clip")
                for i in range(0, len(part), step)]
        for f in futs:
            f.result()

    def _fill_threads(self):
        if getattr(self, "_pool", None) is None:
            import concurrent.futures as cf
            import os

            self._pool_n = max(1, min(16, (os.cpu_count() or 2) - 2))
            self._pool = cf.ThreadPoolExecutor(self._pool_n, thread_name_prefix="zeb-fill")
        return self._pool_n

    def upload_raw(self, cells, dst, stream):
        """Enqueue on `stream` the copies of the given cells' stored patterns into dst[0:n]: one
        per run of consecutive cells from the page-locked copy of the scan, where it is held and
        the cells make few runs; otherwise through two page-locked slots of 64 MB in turn, each
        filled on the host (a run copied, scattered cells gathered) while the other's copy runs."""
        cells = np.asarray(cells, np.int64)
        if len(cells) == 0:
            return
        cut = np.flatnonzero(np.diff(cells) != 1) + 1
        if self.whole_pinned() and len(cut) < self.PINNED_RUNS:
            starts = np.concatenate([[0], cut])
            ends = np.concatenate([cut, [len(cells)]])
            src = self.pinned()
            with torch.cuda.stream(stream):
                for a0, a1 in zip(starts, ends):
                    c0 = int(cells[a0])
                    dst[a0:a1].copy_(src[c0:c0 + (a1 - a0)], non_blocking=True)
            return
        rows, cols, h, w = self.info()
        flat = self.patterns.reshape(rows * cols, h, w)
        per = h * w * self.patterns.itemsize
        most = max(1, self.STAGE_BYTES // per)
        if per > self.STAGE_BYTES:
            raise EngineError("PatternTooLarge: one pattern exceeds the staging slot")
        td = self.raw_dtype()
        with torch.cuda.stream(stream):
            for o in range(0, len(cells), most):
                part = cells[o:o + most]
                k = len(part)
                slot = self._slot()
                host = slot[0].numpy()[: k * per].view(self.patterns.dtype).reshape(k, h, w)
                if k == 1 or bool((np.diff(part) == 1).all()):
                    self._fill(host, flat[int(part[0]):int(part[0]) + k])
                else:
                    self._gather(host, flat, part)
                dst[o:o + k].copy_(slot[0][: k * per].view(td).view(k, h, w), non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
                slot[1] = ev

    def refine_patterns(self, cells, quaternions, phase, trust, rounds, gradient):
        """planefit.zig:570-622 (settle, k = 6) for the given cells against one phase."""
        from . import adjoint

        if not self.phases:
            raise EngineError("NoPhases")
        if not 0 <= phase < len(self.phases):
            raise EngineError(f"phase {phase} of {len(self.phases)}")
        self.prepare_masters()
        rows, cols, h, w = self.info()
        n = len(cells)
        if quaternions is None:
            q0 = self.res["quat"][cells].astype(np.float64)
        else:
            q0 = np.asarray(quaternions, np.float64).reshape(n, 4)
        pats = self.prepared(cells)
        items = self.items_of(cells)
        fr = self.frame()
        _, sheets, grad, vpair, gpair = self.phases[phase].baked
        lst = self.mask_list(fr)
        if lst is not None and lst.numel() > 51200:
            lst = None
        plan = adjoint.Plan(pats, items, fr, vpair, gpair, self.phases[phase].master.side, lst)
        s = self.set
        trust_px = (s["plane_trust"] if trust is None else float(trust)) * h
        most = int(s["plane_iters"] if rounds is None else rounds)
        q, shift, ncc, it = adjoint.refine6(plan, torch.as_tensor(q0, device=self.dev), trust_px, most, gradient)
        J = adjoint.pc_jacobian(self.geo, h, w)
        # the pattern centres on the device: pc = pc0 + J⁻¹·shift for every pattern
        Ji = torch.as_tensor(np.linalg.inv(J).T, dtype=torch.float64, device=self.dev)
        pc = torch.as_tensor(self.geo.pc[None, :], dtype=torch.float64, device=self.dev) + shift @ Ji
        return {"quaternions": q.cpu().numpy(), "shift": shift.cpu().numpy(), "pc": pc.cpu().numpy(),
                "ncc": ncc.cpu().numpy(), "rounds": int(it)}

    def fz_of(self, recs):
        """Each phase's records reduced to its fundamental zone on the device, with their Bunge
        angles (the landing's conversion): ([phase][n][4], [phase][n][3]) device tensors."""
        n_ph, n = recs.shape[0], recs.shape[1]
        fz = self.buf("fz", max(n_ph * n * 4, 1))[: n_ph * n * 4].view(n_ph, n, 4)
        bg = self.buf("fz_bunge", max(n_ph * n * 3, 1))[: n_ph * n * 3].view(n_ph, n, 3)
        for pi, p in enumerate(self.phases):
            ops = getattr(p, "ops_dev", None)
            if ops is None:
                ops = torch.as_tensor(np.ascontiguousarray(p.master.rotations(), np.float64), device=self.dev)
                p.ops_dev = ops
            N.call("zeb_records_fz_bunge", ptr(recs[pi]), n, ptr(ops), ops.shape[0], ptr(fz[pi]), ptr(bg[pi]),
                   stream_ptr())
        return fz, bg

    def index_cells(self, cells, bandwidth=None, method="spherical", grid=None, whole_pass=True):
        """engine.zig:1990-2137 — index the given cells against every phase: records
        [phase][cell][8] = (q, NCC, NMI, last improving step, z). whole_pass: the call counts as
        one pass over the scan (whole_pinned); index_step counts only its sweep's first step."""
        cells = np.asarray(cells, np.int64)
        n = len(cells)
        n_ph = len(self.phases)
        if n_ph == 0:
            raise EngineError("NoPhases")
        if n == 0:
            return np.zeros((n_ph, 0, 8), np.float32)
        if whole_pass:
            self._index_calls += 1  # (a scan indexed a second time is pinned whole: whole_pinned)
        self.prepare(bandwidth, method, grid)
        rows, cols, h, w = self.info()
        raw = self.buf("raw_up", n * h * w, self.raw_dtype()).view(-1)[: n * h * w].view(n, h, w)
        self.upload_raw(cells, raw, torch.cuda.current_stream())
        recs = self.run_device(raw, cells, bandwidth, method=method, grid=grid)
        fzd, bgd = self.fz_of(recs)
        self._last_fz = (fzd.cpu().numpy(), bgd.cpu().numpy())
        out = recs.cpu().numpy()
        self.counts["reads"] += 2
        self.counts["waits"] += 2
        self.check_device()
        return self.finish(out)

    def device_batch(self):
        """Patterns per device pass of a pipelined run (16 384 unless tune() found better)."""
        return int(self.tuned.get("device_batch", 16384))

    def tune(self, progress=None):
        """Fit how the work is cut up to this GPU and this scan: a sample of the region (about
        32 768 patterns at L ≤ 64, fewer above) is indexed through the pipelined path and timed,
        with nothing landed, and each knob in turn climbs from its value — doubled while that is
        faster, else halved while that is (the reference's tune, engine.zig ze_tune_*):
        `device_batch` (patterns per device pass, 2 048 … 65 536) and `tile_mb` (the memory a
        pass's spectra may take, which sets the items per spectrum tile, 512 … 8 192). Neither
        the orientations found nor which matches are accepted depend on them. progress(trials)
        after each trial; False stops (the best so far stays). Returns (before, after, summary)."""
        import time

        s = self.set
        bw, dg, method = s.sweep(self.index_sweep if self.index_cells_list is not None else 0)
        region = self.region_cells()
        want = 65536 if bw <= 32 else 32768 if bw <= 64 else 8192 if bw <= 128 else 2048
        n = min(len(region), want)
        cells = region[((2 * np.arange(n) + 1) * len(region)) // (2 * n)] if n < len(region) else region
        before = {"device_batch": self.device_batch(), "tile_mb": int(s["tile_mb"])}
        knobs = {"device_batch": (2048, 65536), "tile_mb": (512, 8192)}
        trials = [0]
        stop = [False]

        def apply(k, v):
            if k == "device_batch":
                self.tuned["device_batch"] = v
            else:
                s.apply({"tile_mb": v})

        def timed(k, v):
            apply(k, v)
            torch.cuda.synchronize(self.dev)
            t0 = time.perf_counter()
            try:
                self.index_pipelined(cells, bw, lambda *x: None, method=method, grid=dg)
                torch.cuda.synchronize(self.dev)
                sec = time.perf_counter() - t0
            except (RuntimeError, N.NativeError):  # a value this GPU cannot run (memory) just loses
                sec = float("inf")
            trials[0] += 1
            if progress is not None and progress(trials[0]) is False:
                stop[0] = True
            return sec

        timed("device_batch", before["device_batch"])  # warm-up: tables, buffers
        for k, (lo, hi) in knobs.items():
            if stop[0]:
                break
            cur = before[k] if k == "device_batch" else int(s["tile_mb"])
            best = timed(k, cur)
            for direction in (2.0, 0.5):
                moved = False
                while not stop[0]:
                    v = int(cur * direction)
                    if not lo <= v <= hi:
                        break
                    t = timed(k, v)
                    if t < best:
                        best, cur, moved = t, v, True
                    else:
                        break
                if moved:
                    break
            apply(k, cur)
        after = {"device_batch": self.device_batch(), "tile_mb": int(s["tile_mb"])}
        summary = (f"tuned on {len(cells)} patterns in {trials[0]} trials: device_batch {after['device_batch']}, "
                   f"tile_mb {after['tile_mb']}")
        self.log(summary)
        return before, after, summary

    def index_pipelined(self, cells, bandwidth, on_batch, keep_going=lambda: True, method="spherical", grid=None):
        """engine.zig:1990-2137 over many cells at once: device passes of device_batch() cells,
        each pass's upload (a copy stream, from the pinned scan) overlapping the previous pass's
        kernels, its records read back asynchronously and handed to on_batch(cells, records, fz,
        bunge) on
        the host while the next pass runs.  keep_going() is asked before each new pass."""
        cells = np.asarray(cells, np.int64)
        n_ph = len(self.phases)
        if n_ph == 0:
            raise EngineError("NoPhases")
        if len(cells) == 0:
            return
        self.prepare(bandwidth, method, grid)
        rows, cols, h, w = self.info()
        B = min(self.device_batch(), len(cells))
        comp = torch.cuda.current_stream()
        if getattr(self, "_copy_stream", None) is None:
            self._copy_stream = torch.cuda.Stream(device=self.dev)
        cps = self._copy_stream
        raw = [self.buf(f"raw_pipe{k}", B * h * w, self.raw_dtype())[: B * h * w].view(B, h, w) for k in range(2)]
        # the copy stream starts after everything already queued on the compute stream: memory the
        # caching allocator hands out here may have been freed by work still pending there
        cps.wait_stream(comp)
        host = [torch.empty(n_ph * B * 8, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        hfz = [torch.empty(n_ph * B * 4, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        hbg = [torch.empty(n_ph * B * 3, dtype=torch.float32, pin_memory=True) for _ in range(2)]

        def hv(buf, m, width):
            """A pass of m cells' readback, [phase][m][width], at the start of a page-locked buffer:
            contiguous, so that the copy into it stays asynchronous (a strided destination would be
            staged through pageable memory, the host waiting for the pass)."""
            return buf[: n_ph * m * width].view(n_ph, m, width)
        # a small first pass (its upload is the one nothing hides), then passes of B
        first = min(len(cells), max(1, B // 4))
        parts = [cells[:first]] + [cells[i:i + B] for i in range(first, len(cells), B)]
        up_done = [None, None]
        comp_done = [None, None]
        back = [None, None]  # (event, cells, stamp)

        pre = [None, None]

        def issue_upload(i):
            k = i % 2
            if comp_done[k] is not None:
                cps.wait_event(comp_done[k])  # the pass that last read this buffer has finished
            if method == "spherical":
                # the cells' detector positions, copied on this stream ahead of their patterns: a
                # small copy on the compute stream would wait behind the next pass's upload
                with torch.cuda.stream(cps):
                    items = self.items_of(parts[i])
                items.record_stream(comp)
                pre[k] = (items, self._batch_t)
            self.upload_raw(parts[i], raw[k], cps)
            ev = torch.cuda.Event()
            ev.record(cps)
            up_done[k] = ev

        def drain(k):
            ev, cb, stamp = back[k]
            ev.synchronize()
            self.counts["reads"] += 2  # the records and their fundamental-zone orientations
            self.counts["waits"] += 1
            back[k] = None
            out = hv(host[k], len(cb), 8).numpy().copy()
            fz = hv(hfz[k], len(cb), 4).numpy().copy()
            bg = hv(hbg[k], len(cb), 3).numpy().copy()
            on_batch(cb, self.finish(out, stamp), fz, bg)

        issue_upload(0)
        for i in range(len(parts)):
            k = i % 2
            comp.wait_event(up_done[k])
            cb = parts[i]
            recs = self.run_device(raw[k][: len(cb)], cb, bandwidth, method=method, grid=grid, pre=pre[k])
            ev = torch.cuda.Event()
            ev.record(comp)
            comp_done[k] = ev
            if i + 1 < len(parts):
                # the next pass's upload, its host fill (a scan streamed through the staging
                # slots) done while this pass runs
                issue_upload(i + 1)
            if back[k] is not None:
                drain(k)
            fzd, bgd = self.fz_of(recs)
            hv(host[k], len(cb), 8).copy_(recs, non_blocking=True)
            hv(hfz[k], len(cb), 4).copy_(fzd, non_blocking=True)
            hv(hbg[k], len(cb), 3).copy_(bgd, non_blocking=True)
            evb = torch.cuda.Event()
            evb.record(comp)
            back[k] = (evb, cb, self.batch_stamp)
            if back[1 - k] is not None:
                drain(1 - k)
            if not keep_going():
                break
        for k in (0, 1):
            if back[k] is not None:
                drain(k)
        torch.cuda.current_stream().wait_stream(cps)
        self.check_device()

    def finish(self, out, stamp=None):
        """engine.zig:2127-2137 — the batch stamp checked, and each NMI on the scan's chance scale."""
        stamp = self.batch_stamp if stamp is None else stamp
        if self.pending_skip > 0:
            # a readback that did not come from this batch (what a device that silently skipped the
            # batch would hand back): the stamp check below rejects it
            self.pending_skip -= 1
            out = out.copy()
            out[..., 7] = float(stamp - 1)
        if not (out[..., 7] == float(stamp)).all():
            raise EngineError("DeviceSkippedBatch")
        for pi in range(out.shape[0]):
            out[pi, :, 7] = (out[pi, :, 5] - self.chance_med[pi]) / self.chance_spread[pi]
        return out

    def tile_items(self, ph, n):
        """Items whose spectra one pass holds: tile_mb of them, at least 512 (spherical.zig:311-315),
        spread evenly over the passes a batch needs (no short last tile)."""
        if ph.u_scale is not None:  # the FP16 spectrum: half the bytes per item
            per = N.load().zeb_spectrum_h_bytes(ctypes.byref(ph.dims), 128) // 128
        else:
            per = N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), 1)
        most = int(max(1, min(n, max(512, (self.set["tile_mb"] << 20) // per))))
        tiles = -(-n // most)
        return -(-n // tiles)

    def calibrate(self):
        """engine.zig:2202-2292 — chance NMI per phase: ~256 region cells × 8 random orientations;
        median and 1.4826 × median absolute deviation."""
        n_ph = len(self.phases)
        s = self.set
        key = (s["static_background"], s["static_patterns"], s["dynamic_background"], s["dynamic_sigma"], s["mask"],
               s["mask_radius"], s["nmi_bins"], self.factor(), s["master_smooth"], s["pixel_angle_deg"], self.geo.key(),
               tuple(id(p.baked[1]) if p.baked else None for p in self.phases), s["roi_x"], s["roi_y"], s["roi_w"],
               s["roi_h"], id(self.patterns))
        if key == self.chance_key and len(self.chance_med) == n_ph:
            return
        self.prepare_masters()
        region = self.region_cells()
        n = min(len(region), 256)
        cells = region[((2 * np.arange(n) + 1) * len(region)) // (2 * n)]
        draws = 8
        pats = self.upload(cells)
        t = self.positions(cells)
        items = torch.as_tensor(np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1), device=self.dev)
        fr = self.frame()
        self.chance_med, self.chance_spread = [], []
        for pi, p in enumerate(self.phases):
            out = torch.empty(draws * n, dtype=torch.float32, device=self.dev)
            N.call("zeb_chance", ptr(pats), ptr(items), n, draws, ctypes.byref(fr), ptr(p.baked[3]), p.master.side,
                   s["nmi_bins"], ptr(out), stream_ptr())
            c = np.sort(out.cpu().numpy())
            med = c[len(c) // 2]
            dev = np.sort(np.abs(c - med))
            spread = max(1.4826 * dev[len(c) // 2], 1e-6)
            self.chance_med.append(float(med))
            self.chance_spread.append(float(spread))
            self.log(f"chance, phase {pi}: NMI {med:.4f} ± {spread:.4f} over {n} patterns at random orientations; "
                     f"z {s['accept_z']:.0f} is NMI {med + s['accept_z'] * spread:.4f}")
        self.chance_key = key

    def choose_phase(self, recs):
        """engine.zig:2295-2307 — per cell, the phase with the largest NMI (or NCC)."""
        col = 5 if self.set["phase_by"] == "nmi" else 4
        return np.argmax(recs[:, :, col], axis=0)

    # ── indexing in sweeps ──

    def index_begin(self):
        if not self.phases:
            raise EngineError("NoPhases")
        if "euler" not in self.res or self.res["euler"].shape[0] != self.res["quat"].shape[0]:
            self.res["euler"] = R.to_bunge(self.res["quat"].astype(np.float64)).astype(np.float32)
        cells = self.region_cells()
        self.index_cells_list = cells
        self.index_done = 0
        self.index_region = len(cells)
        self.index_sweep = 0
        self.index_accepted = 0
        self.cancel = False
        self.res["phase"][cells] = -1
        self.res["sweep"][cells] = -1
        self.res["z"][cells] = 0
        self._nl_report = bool(self.set["nlpar"])  # the run's first batch says what the averaging did

    def land(self, cells, recs, fz=None, bunge=None):
        """engine.zig:2392-2419 — each cell keeps the better match; accepted ones their sweep.
        fz: the records' orientations already in each phase's fundamental zone ([phase][cell][4],
        zeb_records_fz), bunge their Bunge angles ([phase][cell][3], zeb_records_fz_bunge); computed
        here on the host when absent."""
        s = self.set
        res = self.res
        cells = np.asarray(cells, np.int64)
        settle = math.radians(s["accept_step_deg"])
        best = self.choose_phase(recs)
        r = recs[best, np.arange(len(cells))]
        good = r[:, 5] >= s["accept_nmi"] if s["accept_nmi"] > 0 else r[:, 7] >= s["accept_z"]
        replace = (res["phase"][cells] < 0) | (good & (r[:, 6] <= settle)) | (r[:, 7] > res["z"][cells])
        if fz is not None:
            q = fz[best, np.arange(len(cells))]
        else:
            q = np.empty((len(cells), 4))
            for p in np.unique(best):
                sel = best == p
                q[sel] = R.to_fz(r[sel, :4].astype(np.float64), self.phases[int(p)].master.rotations())
        n = len(cells)
        if n and replace.all() and cells[-1] - cells[0] == n - 1 and (n == 1 or (np.diff(cells) == 1).all()):
            # every cell of a run of consecutive cells takes its record (a first sweep's pass): the
            # same writes as slices
            sel = slice(int(cells[0]), int(cells[0]) + n)
            res["quat"][sel] = q
            if bunge is not None and fz is not None:
                res["euler"][sel] = bunge[best, np.arange(n)]
            else:
                res["euler"][sel] = R.to_bunge(q.astype(np.float64)).astype(np.float32)
            res["ncc"][sel] = r[:, 4]
            res["nmi"][sel] = r[:, 5]
            res["z"][sel] = r[:, 7]
            res["phase"][sel] = best
            res["settled"][sel] = r[:, 6] <= settle
        else:
            sel = cells
            idx = cells[replace]
            res["quat"][idx] = q[replace]
            if bunge is not None and fz is not None:
                res["euler"][idx] = bunge[best, np.arange(n)][replace]
            else:
                res["euler"][idx] = R.to_bunge(q[replace].astype(np.float64)).astype(np.float32)
            res["ncc"][idx] = r[replace, 4]
            res["nmi"][idx] = r[replace, 5]
            res["z"][idx] = r[replace, 7]
            res["phase"][idx] = best[replace]
            res["settled"][idx] = r[replace, 6] <= settle
        kept = res["nmi"][sel] >= s["accept_nmi"] if s["accept_nmi"] > 0 else res["z"][sel] >= s["accept_z"]
        newly = (res["sweep"][sel] < 0) & kept & res["settled"][sel]
        res["sweep"][cells[newly]] = self.index_sweep
        self.index_accepted += int(newly.sum())
        self.index_done += len(cells)
        self.events.append({"kind": "progress", "stage": "index", "done": int(self.index_done),
                            "total": int(len(self.index_cells_list)), "sweep": self.index_sweep, "sweeps": s["sweeps"]})

    def index_step(self):
        """engine.zig:2426-2465 — about 4096 cells of the sweep in progress; returns cells left."""
        s = self.set
        cells_all = self.index_cells_list
        left = len(cells_all) - self.index_done
        if left == 0 or self.cancel:
            return 0
        batch = max(s["batch"], 1)
        n = min(left, batch * min(max(4096 // batch, 2), 16))
        cells = cells_all[self.index_done:self.index_done + n]
        bw, dg, method = s.sweep(self.index_sweep)
        # a scan stepped through once is one pass: only the first step of the first sweep counts
        first = self.index_done == 0 and self.index_sweep == 0
        self._whole_pass = True
        try:
            recs = self.index_cells(cells, bw, method, dg, whole_pass=first)
        finally:
            self._whole_pass = False
        self.land(cells, recs, *self._last_fz)
        self.next_sweep(bw)
        return len(self.index_cells_list) - self.index_done

    STEP_RUN_CELLS = 1 << 18

    def index_step_run(self, most=None):
        """index_step over up to `most` cells (STEP_RUN_CELLS by default) of the sweep in progress
        as one pipelined run (index_pipelined: the cells, records and landing of index_step, with
        uploads, kernels, readbacks and landing overlapped; none in flight when it returns);
        returns the cells left. What the C ABI's ze_index_step runs."""
        s = self.set
        left = len(self.index_cells_list) - self.index_done
        if left == 0 or self.cancel:
            return 0
        most = self.STEP_RUN_CELLS if most is None else max(1, int(most))
        bw, dg, method = s.sweep(self.index_sweep)
        part = self.index_cells_list[self.index_done:self.index_done + most]
        if self.index_done == 0 and self.index_sweep == 0:
            self._index_calls += 1  # (a scan indexed a second time is pinned whole: whole_pinned)
        self._whole_pass = True
        try:
            self.index_pipelined(part, bw, lambda cb, recs, fz, bg: self.land(cb, recs, fz, bg),
                                 keep_going=lambda: not self.cancel, method=method, grid=dg)
        finally:
            self._whole_pass = False
        self.next_sweep(bw)
        return len(self.index_cells_list) - self.index_done

    def next_sweep(self, bw):
        """engine.zig:2452-2463 — at the end of a sweep, the cells not yet accepted go on to the next."""
        s = self.set
        cells_all = self.index_cells_list
        if self.index_done == len(cells_all) and self.index_sweep + 1 < s["sweeps"]:
            keep = cells_all[self.res["sweep"][cells_all] < 0]
            _, dg, method = s.sweep(self.index_sweep)
            what = {"spherical": f"spherical, bandwidth {bw}", "dictionary": f"dictionary, grid {dg}",
                    "pca": f"dictionary components, grid {dg}"}[method]
            self.log(f"sweep {self.index_sweep + 1} of {s['sweeps']} ({what}): "
                     f"{len(cells_all) - len(keep)} of {len(cells_all)} patterns accepted, {len(keep)} left")
            if len(keep):
                self.index_cells_list = keep
                self.index_done = 0
                self.index_sweep += 1

    def index_run(self, progress=None):
        """Every sweep to the end (or until cancelled, or until progress(status) returns False),
        each through index_pipelined: the same cells, records and landing as repeated
        index_step calls, with uploads, kernels, readbacks and landing overlapped."""
        s = self.set
        self._index_calls += 1
        self._whole_pass = True
        try:
            self._index_sweeps(progress)
        finally:
            self._whole_pass = False

    def _index_sweeps(self, progress):
        s = self.set
        while len(self.index_cells_list) - self.index_done > 0 and not self.cancel:
            bw, dg, method = s.sweep(self.index_sweep)
            stop = [False]

            def on_batch(cb, recs, fz, bg):
                self.land(cb, recs, fz, bg)  # a pass already in flight when the stop came still lands
                if progress is not None and not stop[0] and progress(self.status()) is False:
                    stop[0] = True

            self.index_pipelined(self.index_cells_list[self.index_done:], bw, on_batch,
                                 keep_going=lambda: not (stop[0] or self.cancel), method=method, grid=dg)
            if stop[0]:
                return
            self.next_sweep(bw)

    def status(self):
        s = self.set
        bw, dg, method = s.sweep(self.index_sweep)
        return {"sweep": self.index_sweep, "sweeps": s["sweeps"], "bandwidth": bw, "dict_grid": dg,
                "done": int(self.index_done), "total": int(len(self.index_cells_list) if self.index_cells_list is not None else 0),
                "region": int(self.index_region), "accepted": int(self.index_accepted), "method": method}

    # ── simulation ──

    def simulate_device(self, phase, cells, quats, shifts=None):
        """The simulated patterns as a device tensor [n, h, w] (see simulate); `shifts` [n, 3]
        (pixels, sample frame) moves each pattern's source from its cell's position, as a
        pattern-centre offset does."""
        self.prepare_masters()
        cells = np.asarray(cells, np.int64)
        q = np.asarray(quats, np.float32).reshape(-1, 4)
        n = len(cells)
        h, w = self.pattern_shape()
        t = self.positions(cells)
        if shifts is not None:
            t = (t + np.asarray(shifts, np.float32).reshape(n, 3)).astype(np.float32)
        pd = torch.as_tensor(np.concatenate([t, np.zeros((n, 1), np.float32), q], 1), device=self.dev)
        out = torch.empty(n * h * w, dtype=torch.float32, device=self.dev)
        p = self.phases[phase]
        fr = self.frame()
        N.call("zeb_project", ptr(p.baked[1]), p.master.side, ptr(pd), n, ctypes.byref(fr), ptr(out), stream_ptr())
        return out.view(n, h, w)

    def simulate(self, phase, cells, quats):
        """engine.zig:2753-2769 — simulated patterns of a phase at the given orientations, each as
        cell cells[k] would record it (from the master as smoothed for the patterns)."""
        self.prepare_masters()
        cells = np.asarray(cells, np.int64)
        q = np.asarray(quats, np.float32).reshape(-1, 4)
        n = len(cells)
        h, w = self.pattern_shape()
        t = self.positions(cells)
        poses = np.concatenate([t, np.zeros((n, 1), np.float32), q], 1)
        pd = torch.as_tensor(poses, device=self.dev)
        out = torch.empty(n * h * w, dtype=torch.float32, device=self.dev)
        p = self.phases[phase]
        fr = self.frame()
        N.call("zeb_project", ptr(p.baked[1]), p.master.side, ptr(pd), n, ctypes.byref(fr), ptr(out), stream_ptr())
        return out.view(n, h, w).cpu().numpy()
