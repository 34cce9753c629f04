"""zebsdsolve_b200: the spherical cross-correlation indexing path of zebsdsolve, on one B200.

A drop-in for the reference's Python API on this path (zebsdsolve 0.2.8, python/zebsdsolve):

    import zebsdsolve_b200 as ze

    result = ze.index(patterns, ["Ni.npz"], pc=(0.5, 0.3, 0.6), bandwidth=64)
    result.quaternions, result.ncc, result.phase       # per map cell

`Solver` is the engine itself for driving the steps one at a time (configure, set_patterns,
set_geometry, add_phase, index / index_begin / index_step, results, ...).  Conventions as the
reference's: quaternions (w, x, y, z) map sample directions to crystal directions, Bunge angles
in radians, map cells row-major, the pattern centre in the Bruker convention.

Every computation on the path runs in the CUDA library libzebsdsolve_b200.so (hand-written
sm_100a kernels behind the C ABI of include/zebsdsolve_b200.h); there is no CPU fallback. The
reference's own C ABI, its ze_* calls, is libzebsdsolve.so (include/zebsdsolve.h, ze_abi.py),
which carries each call onto this package's Solver.
"""

import math

import numpy as np

__version__ = "0.2.8"

LAUE = {1: "-1", 2: "2/m", 3: "mmm", 4: "4/m", 5: "4/mmm", 6: "-3", 7: "-3m", 8: "6/m", 9: "6/mmm", 10: "m-3", 11: "m-3m"}
METHODS = ("spherical", "dictionary", "pca")


class Error(RuntimeError):
    """An engine call failed; the message says which and why (the reference's ze.Error)."""


def _engine():
    from .engine import Engine

    try:
        return Engine()
    except Exception as e:  # noqa: BLE001 - surfaced as the API's own error
        raise Error(f"engine: {e}") from e


class Solver:
    """One engine on one GPU device (python/zebsdsolve/__init__.py:65-951, the indexing path)."""

    def __init__(self):
        self._e = _engine()

    def close(self):
        self._e = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, what, fn, *a, **k):
        try:
            return fn(*a, **k)
        except Error:
            raise
        except Exception as e:  # noqa: BLE001
            raise Error(f"{what}: {e}") from e

    @property
    def adapter(self):
        import torch

        return torch.cuda.get_device_name(self._e.dev)

    def events(self):
        out, self._e.events = self._e.events, []
        return out

    def cancel(self):
        self._e.cancel = True

    # ── settings and geometry ──

    def configure(self, **settings):
        if settings:
            self._call("configure", self._e.set.apply, settings)
        return self

    @property
    def settings(self):
        return self._e.set.as_dict()

    @property
    def geometry(self):
        return self._e.geo.as_dict()

    def set_geometry(self, **fields):
        """Set any of the geometry's fields (pc, rot, sample_tilt_deg, detector_tilt_deg, px_um,
        step_x_um, step_y_um, plane_kind, plane). A pattern centre set by hand is one for the whole
        map again (the plane of source points goes unless one comes with it)."""
        self._call("set_geometry", self._e.geo.given, fields, self._e.geo_given)
        if not self._e.geo.px_um > 0:  # (no pixel size: the scan's own, or its detector's width's)
            self._e.geo.px_um = self._e.default_px()
        return self

    # ── scan ──

    def set_patterns(self, patterns):
        """Patterns from an array: (rows, cols, h, w) or (n, h, w), uint8, uint16 or float32."""
        self._call("set_patterns", self._e.set_patterns, patterns)
        return self

    @property
    def scan(self):
        rows, cols, h, w = self._call("scan", self._e.info)
        src = getattr(self._e, "scan_source", None) or {}
        return {"rows": rows, "cols": cols, "pattern_shape": (h, w),
                "dtype": ["uint8", "uint16", "float32"][self._e.pixel], "format": src.get("format", "array"),
                "voltage_kv": src.get("voltage_kv", float("nan")), "pc_note": src.get("pc_note", ""),
                "has_background": src.get("background") is not None, "has_pc": src.get("pc") is not None,
                "has_px": bool(src.get("px_um")),
                "pattern_kinds": src.get("pattern_kinds", [])}

    def open(self, *paths):
        """Open a scan file, and the side files it needs after it (__init__.py:216-240): EDAX .up1 /
        .up2 (with its scan's .ang for the map's shape, the steps and the pattern centre), Oxford
        .ebsp (uncompressed), NORDIF Pattern.dat (its Setting.txt picked up from beside it when not
        given), and HDF5: h5ebsd (kikuchipy, Bruker, EDAX), Oxford .h5oina, EMsoft's EMEBSD output.
        The geometry takes what the file says (steps, tilts, pattern centre, pixel size, Oxford's
        detector orientation); the region of interest goes back to the whole map. A file that
        stores processed and unprocessed patterns side by side (an Oxford acquisition can) is read
        as the setting `stored_patterns` says; `scan["pattern_kinds"]` names the kinds it stores.
        A static background the file stores is what `static_background: "file"` subtracts."""
        import os

        from . import scan as SC

        paths = [str(p) for p in paths]
        if len(paths) == 1 and paths[0].lower().endswith(".dat"):
            side = os.path.join(os.path.dirname(paths[0]), "Setting.txt")
            if os.path.isfile(side):
                paths.append(side)
        sc = self._call("open", SC.open_scan, paths,
                        unprocessed=self._e.set["stored_patterns"] == "unprocessed")
        info = sc.info
        self.set_patterns(np.asarray(sc.map()))
        self.configure(roi_x=0, roi_y=0, roi_w=0, roi_h=0)
        geo = {k: info[k] for k in ("step_x_um", "step_y_um", "sample_tilt_deg", "detector_tilt_deg")
               if np.isfinite(info[k])}
        if info["pc"] is not None:  # (engine.zig:933-946: a file's pattern centre comes unturned)
            geo["pc"] = tuple(info["pc"])
            geo["rot"] = (0.0, 0.0, 0.0)
        if info.get("detector_rot") is not None:
            geo["rot"] = tuple(info["detector_rot"])
        if np.isfinite(info.get("px_um", float("nan"))) and info["px_um"] > 0:
            geo["px_um"] = float(info["px_um"])
        if geo:
            self.set_geometry(**geo)
        px = info.get("px_um", float("nan"))
        self._e.scan_source = {"px_um": float(px) if np.isfinite(px) and px > 0 else None,
                               "format": sc.format, "voltage_kv": info["voltage_kv"], "pc_note": info["pc_note"],
                               "paths": paths, "pc": info["pc"], "background": info.get("background"),
                               "pattern_kinds": info.get("pattern_kinds", []),
                               "overview": info.get("overview", (0, None)), "stored": info.get("stored")}
        self._e.avg = None
        return self

    def stored_overview(self):
        """The scan file's stored acquisition quality map, or None; never computes pattern statistics
        (__init__.py:365-375): {"kind": 1 band contrast, 2 image quality, 3 Radon quality, 4 pattern
        quality; "label"; "values": float32 (rows, cols), NaN where the file's value is not finite}.
        HDF5 files store it beside the patterns under one of the makers' names (scan.zig:294-332); an
        EDAX .up takes the image quality column of its .ang."""
        from . import scan as SC

        src = getattr(self._e, "scan_source", None)
        kind, read = (src or {}).get("overview") or (0, None)
        if not kind:
            return None
        values = self._call("stored_overview", read)
        info = self.scan
        return {"kind": kind, "label": SC.OVERVIEW_LABELS[kind], "values": values.reshape(info["rows"], info["cols"])}

    def stored_orientations(self):
        """The orientations the scan file stores from its maker's indexing, as it stores them
        (__init__.py:814-824, scan.zig:220-291): {"euler": (rows, cols, 3) Bunge angles in radians,
        "phase": (rows, cols) labels, −1 where not indexed}, or None when it stores none (Oxford's
        Euler, Bruker's phi1/PHI/phi2 in degrees, EDAX's phi1/Phi/phi2, an .up's .ang records)."""
        src = getattr(self._e, "scan_source", None)
        read = (src or {}).get("stored")
        got = self._call("stored_orientations", read) if read is not None else None
        if got is None:
            return None
        info = self.scan
        return {"euler": got["euler"].reshape(info["rows"], info["cols"], 3),
                "phase": got["phase"].reshape(info["rows"], info["cols"])}

    def export(self, path):
        """Write the results by the path's extension (__init__.py:879-905): an EDAX .ang or an HKL
        .ctf, the orientations in the engine's own frame. (The reference's .h5oina export copies an
        Oxford acquisition's HDF5 file: not part of this engine.)"""
        ext = str(path).rsplit(".", 1)[-1].lower()
        if ext not in ("ang", "ctf"):
            raise Error(f"export: .{ext} is not written by this engine (.ang, .ctf)")
        text = self.export_text(ext)
        with open(path, "w") as fh:
            fh.write(text)

    def export_text(self, kind):
        """The results as the text of an EDAX .ang (`kind` "ang") or an HKL .ctf ("ctf")."""
        from . import output

        e = self._e
        rows, cols, h, w = self._call("export", e.info)
        phases = [{"name": p.master.name, "laue": p.master.laue, "lattice": p.master.lattice,
                   "space_group": p.master.space_group} for p in e.phases]
        src = getattr(e, "scan_source", None) or {}
        return self._call("export", output.export_text, kind, e.res, phases, e.geo, rows, cols, h, w,
                          src.get("voltage_kv", float("nan")), getattr(e, "convention", None))

    @property
    def frame(self):
        """The reference frame convention the exports write orientations in (__init__.py:858-867):
        `axes` (the convention's sample X, Y, Z as the engine's axes, 1 x on the surface toward the
        detector, 2 y the tilt axis, 3 z out of the surface, negative reversed), `active`,
        `crystal` (x_a_z_cstar, the masters' own; x_astar_z_c; y_b_z_cstar; y_bstar_z_c) and
        `text`, a line naming it. The engine's own until identified (`identify_frame`) or set; a
        new scan resets it."""
        from .convention import Frame

        return (getattr(self._e, "convention", None) or Frame()).as_dict()

    @frame.setter
    def frame(self, value):
        from .convention import Frame

        self._e.convention = None if value is None else self._call("set_frame", Frame.from_dict, dict(value))

    def identify_frame(self, euler=None, phase=None):
        """The reference frame convention a maker's orientations are in, found against the results
        (__init__.py:826-856, engine.zig:784-812, convention.zig:254-404): from `euler` (Bunge
        angles, radians, (rows, cols, 3) or (n, 3), one per map cell) and `phase` (a label per cell,
        negative where not indexed), or with neither the scan file's own. Every convention of the
        sample's axes, the rotation's sense and the crystal's axes on the lattice is tried, cell by
        cell under each phase's own symmetry.

        Returns a dict: `frame` (as `frame` has it), `cells` compared, `within` (the fraction within
        2°), `median_deg`, `runner_up_deg` (the best other convention's median), `matched` (the
        reference's label for each phase), `installed` (the exports take the convention when it was
        told clearly: median under 5°, and the best other's at least twice that and 5° more), and
        the misorientation left, which no convention removes and nothing applies:
        `misorientation` (rotation vector, radians, about the engine's x, y, z, at the map's
        middle), `misorientation_rows` and `misorientation_cols` (its change from the first row to
        the last and from the first column to the last) and `misorientation_cells`."""
        from . import convention as C

        e = self._e
        if not e.phases:
            raise Error("identify_frame: NoPhases")
        if euler is None:
            got = self.stored_orientations()
            if got is None:
                raise Error("identify_frame: NoStoredOrientations")
            euler, phase = got["euler"], got["phase"]
        euler = np.asarray(euler, np.float64).reshape(-1, 3)
        phase = np.asarray(phase, np.int32).reshape(-1)
        if len(phase) != len(euler):
            raise Error("identify_frame: euler and phase differ in length")
        rows, cols, h, w = self._call("identify_frame", e.info)
        views = [(p.master.rotations(), p.master.lattice) for p in e.phases[:C.MAX_PHASES]]
        frame, out = self._call("identify_frame", C.identify, e.res["quat"], e.res["phase"], cols, euler, phase,
                                views)
        holds = out["median_deg"] < 5 and out["runner_up_deg"] >= 2 * out["median_deg"] + 5
        if holds:
            e.convention = frame
        m = np.array(out["misorientation"])
        th = float(np.linalg.norm(m))
        u = m / th if th > 0 else np.zeros(3)
        e.log((
            f"frame of the stored orientations: {frame.describe()}; {out['cells']} cells, median "
            f"{out['median_deg']:.2f}°, {100 * out['within']:.0f} % within 2°, {out['runner_up_deg']:.1f}° under the "
            f"next convention{'; the exports take it' if holds else '; not told clearly, the exports keep theirs'}; "
            f"misorientation left {math.degrees(th):.2f}° about ({u[0]:.3f}, {u[1]:.3f}, {u[2]:.3f}) (x, y, z: toward "
            f"the detector, the tilt axis, out of the surface), changing "
            f"{math.degrees(np.linalg.norm(out['misorientation_rows'])):.2f}° from the first row to the last and "
            f"{math.degrees(np.linalg.norm(out['misorientation_cols'])):.2f}° from the first column to the last"))
        return {"frame": frame.as_dict(), **out, "installed": holds}

    def shape(self, full=False):
        """(h, w) of a pattern as the search sees it (reduced by `binning`), or (full) as stored."""
        if full:
            return tuple(self._call("scan", self._e.info)[2:])
        return self._call("pattern_shape", self._e.pattern_shape)

    def pattern_stats(self, cells=None):
        """(mean, standard deviation) of the stored patterns of the given map cells (all of them by
        default, shaped (rows, cols)), over every stored pixel in FP64 (engine.zig:2696-2728): maps
        of either show the microstructure before indexing."""
        rows, cols, h, w = self._call("scan", self._e.info)
        whole = cells is None
        c = np.arange(rows * cols) if whole else np.asarray(cells, np.int64).reshape(-1)
        if len(c) and (c.min() < 0 or c.max() >= rows * cols):
            raise Error("pattern_stats: OutOfRange")
        flat = self._e.patterns.reshape(rows * cols, h * w)
        mean = np.empty(len(c), np.float32)
        std = np.empty(len(c), np.float32)
        for i in range(0, len(c), 4096):
            x = flat[c[i:i + 4096]].astype(np.float64)
            m = x.mean(1)
            mean[i:i + 4096] = m
            std[i:i + 4096] = np.sqrt(np.maximum((x * x).mean(1) - m * m, 0.0))
        return (mean.reshape(rows, cols), std.reshape(rows, cols)) if whole else (mean, std)

    @property
    def pattern_shape(self):
        return self.shape()

    def lattice(self, n):
        return self._call("lattice", self._e.lattice, n).astype(np.uint64)

    @property
    def pixel_angle(self):
        return float(np.degrees(self._e.pixel_angle() / self._e.set["binning"]))

    # ── phases ──

    def add_phase(self, path):
        return self._call("add_phase", self._e.add_phase, str(path))

    def clear_phases(self):
        self._e.clear_phases()

    @property
    def phases(self):
        out = []
        for p in self._e.phases:
            m = p.master
            from .rotations import LAUE_NAMES

            out.append({"name": m.name, "side": m.side, "point_group": m.point_group, "space_group": m.space_group,
                        "laue": LAUE_NAMES[m.laue], "voltage_kv": m.voltage_kv, "rotations": len(m.rotations())})
        return out

    def master(self, phase=0):
        """A phase's master as the search compares patterns with it: (2, side, side)."""
        self._call("master", self._e.prepare_masters)
        p = self._e.phases[phase]
        return p.baked[1].cpu().numpy().reshape(2, p.master.side, p.master.side)

    # ── simulation ──

    def synthesize(self, **settings):
        """A toy scan from the phases loaded, in place of any scan open, and its answer
        (__init__.py:233-258, engine.zig:2778-2896): a dict with quaternions (rows, cols, 4), phase
        (rows, cols; −1 a blank cell), grain (rows, cols) and geometry (the one it was simulated
        under, its true one).

        Keywords are settings. The microstructure, from `toy_seed`: `toy_rows` × `toy_cols` cells,
        each in the grain of the nearest of `toy_grains` points scattered over the map, each grain
        with a uniformly random orientation and phase; `toy_spread_deg` turns every cell a little
        within its grain; `toy_blank` is the share of cells holding no crystal. The detector:
        patterns of `toy_height` × `toy_width`, the simulation (darkest pixel 0, mean 1 over the
        crystals) weighted `toy_contrast` on a background of mean 1 (flat, or a Gaussian hump of
        `toy_background_sigma` × the width). The counting: a Poisson draw per pixel at a mean of
        `toy_counts` electrons (0: none), from `toy_noise_seed` (0: from `toy_seed`). The draws
        are numpy's (PCG64), so a seed gives the reference's distributions, not its numbers."""
        from . import rotations as R

        if settings:
            self.configure(**settings)
        e = self._e
        if not e.phases:
            raise Error("synthesize: NoPhases")
        st = e.set
        rows, cols, h, w = st["toy_rows"], st["toy_cols"], st["toy_height"], st["toy_width"]
        n, px = rows * cols, h * w
        geometry = self.geometry
        # an empty scan of the shape first: a cell's place in it is part of its geometry
        self.set_patterns(np.zeros((rows, cols, h, w), np.float32))
        rng = np.random.default_rng(int(st["toy_seed"]))
        k = min(int(st["toy_grains"]), n)
        gx, gy = rng.random(k) * cols, rng.random(k) * rows
        gq = R.qstd(rng.normal(size=(k, 4)))  # four normal numbers, normalized: uniform over the rotations
        gp = rng.integers(0, len(e.phases), k)
        grain = np.empty(n, np.int64)
        x = np.arange(cols) + 0.5
        for r in range(rows):  # the nearest point, a row at a time (the first of equals)
            d = (gx[None, :] - x[:, None]) ** 2 + (gy[None, :] - (r + 0.5)) ** 2
            grain[r * cols:(r + 1) * cols] = np.argmin(d, 1)
        q = gq[grain]
        spread = math.radians(st["toy_spread_deg"]) / math.sqrt(3.0)
        if spread > 0:
            q = R.qstd(R.qmul(R.exp_map(spread * rng.normal(size=(n, 3))), q))
        phase = gp[grain].astype(np.int32)
        if st["toy_blank"] > 0:
            phase[rng.random(n) < st["toy_blank"]] = -1
        data = np.zeros((n, px), np.float32)
        chunk = max(1, (4 << 20) // px)
        made = 0
        with e.at_full():  # simulated at the stored size (engine.zig:2828)
            for p in range(len(e.phases)):
                cells = np.flatnonzero(phase == p)
                for i in range(0, len(cells), chunk):
                    c = cells[i:i + chunk]
                    sims = self._call("synthesize", e.simulate, p, c, q[c].astype(np.float32))
                    data[c] = np.asarray(sims).reshape(len(c), px)
                    made += len(c)
                    e.events.append({"kind": "progress", "stage": "synthesize", "done": made, "total": n})
        # the detector: the simulation (its darkest pixel 0, its mean 1) on a background (mean 1)
        crystal = phase >= 0
        mean = float(data[crystal].mean(dtype=np.float64)) if crystal.any() else 0.0
        low = float(data[crystal].min()) if crystal.any() else 0.0
        gain = 1.0 / (mean - low) if crystal.any() and mean > low else 0.0
        back = np.ones(px)
        if st["toy_background_sigma"] > 0:
            sg = st["toy_background_sigma"] * w
            yy, xx = np.mgrid[0:h, 0:w]
            back = np.exp(-((xx + 0.5 - 0.5 * w) ** 2 + (yy + 0.5 - 0.5 * h) ** 2) / (2 * sg * sg)).reshape(-1)
            back *= px / back.sum()
        blank = (~crystal) | (gain == 0)
        signal = np.where(blank[:, None], 1.0, (data - low) * gain)
        intensity = (1 - st["toy_contrast"]) * back[None, :] + st["toy_contrast"] * signal
        if st["toy_counts"] > 0:
            noise = np.random.default_rng(int(st["toy_noise_seed"]) or (int(st["toy_seed"]) ^ 0x9E3779B97F4A7C15))
            data = noise.poisson(st["toy_counts"] * intensity).astype(np.float32)
        else:
            data = intensity.astype(np.float32)
        self.set_patterns(data.reshape(rows, cols, h, w))
        e.log(f"toy scan: {rows} × {cols} patterns of {h} × {w}, {k} grains of {len(e.phases)} phase(s), "
              f"{int((~crystal).sum())} blank cells, contrast {st['toy_contrast']:.2f}, {st['toy_counts']:.4f} "
              f"electrons a pixel, seed {st['toy_seed']}")
        return {"quaternions": q.astype(np.float32).reshape(rows, cols, 4), "phase": phase.reshape(rows, cols),
                "grain": grain.astype(np.int32).reshape(rows, cols), "geometry": geometry}

    def simulate(self, quaternions, cells=None, phase=0):
        q = np.asarray(quaternions, np.float32).reshape(-1, 4)
        cells = np.arange(len(q)) if cells is None else np.asarray(cells).reshape(-1)
        return self._call("simulate", self._e.simulate, phase, cells, q)

    # ── six unknowns per pattern (source and orientation) ──

    def refine_patterns(self, cells, quaternions=None, phase=0, trust=None, rounds=None, gradient="reference"):
        """Each given pattern refined by itself over its orientation and its source's place (its
        pattern centre): the per-pattern Levenberg–Marquardt of the reference's plane fit
        (planefit.zig:570-622 with six unknowns; Winkelmann et al., kikuchipy's
        refine_orientation_projection_center). quaternions: the starting orientations (default:
        the cells' current results). trust: how far a source may move, in pattern heights
        (default plane_trust); rounds: at most this many (default plane_iters). gradient:
        "reference" (the master's gradient table, as the reference) or "adjoint" (the exact
        derivative of the projection, through the torch.autograd.Function of `adjoint.py`).
        Returns a dict: quaternions (n, 4), shift (n, 3, pixels in the sample's axes), pc (n, 3),
        ncc (n), rounds."""
        c = np.asarray(cells, np.int64).reshape(-1)
        if gradient not in ("reference", "adjoint"):
            raise Error(f"refine_patterns: gradient {gradient!r}")
        return self._call("refine_patterns", self._e.refine_patterns, c, quaternions, phase, trust, rounds, gradient)

    # ── indexing ──

    def index_cells(self, cells, method=None, bandwidth=None, dict_grid=None):
        c = np.asarray(cells, np.int64).reshape(-1)
        st = self._e.set
        method = method if method is not None else st["method"]
        if method not in ("spherical", "dictionary", "pca"):
            raise Error(f"index_cells: unknown method {method!r}")
        r = self._call("index_cells", self._e.index_cells, c, bandwidth, method, dict_grid)
        return {"quaternions": r[..., :4].copy(), "ncc": r[..., 4].copy(), "nmi": r[..., 5].copy(),
                "step": r[..., 6].copy(), "z": r[..., 7].copy()}

    def tune(self, progress=None):
        """Fit how the work is cut up to this GPU and this scan (a sample of the region indexed and
        timed, nothing stored touched): the knobs that matter here are the patterns per device pass
        and the memory a pass's spectra may take; the reference's workgroup sizes (`batch`,
        `refine_pixels`, `wg_refine`, `wg_fft`) have no counterpart on this engine. Returns the
        knobs before and after and a summary; progress(trials) after each timed trial, False stops."""
        before, after, summary = self._call("tune", self._e.tune, progress)
        return {"before": before, "after": after, "summary": summary}

    # ── the pattern-centre vote ──

    def fit_pc(self):
        """Fit the pattern centre by the voting search (settings fit_grid, fit_bandwidth, pc_*;
        __init__.py:426-434): the geometry takes the result. Returns pc, start, score (the fit
        patterns' mean best correlation at the fitted centre), start_score, n_patterns,
        n_candidates, levels, at_border."""
        from . import pcfit

        r = self._call("fit_pc", pcfit.run, self._e)
        return {"pc": list(r["pc"]), "start": list(r["start"]), "score": r["score"], "start_score": r["start_score"],
                "n_patterns": r["n_patterns"], "n_candidates": r["n_candidates"], "levels": r["levels"],
                "at_border": bool(r["at_border"])}

    def pc_scores(self):
        """The last search grid's votes: (scores[nz, ny, nx], pcx values, pcy values, pcz values)."""
        h = self._e.pc_history
        if not h:
            e = np.zeros(0)
            return np.zeros((0, 0, 0), np.float32), e, e.copy(), e.copy()
        x, y, z = h[-1]["axes"]
        return h[-1]["scores"].reshape(len(z), len(y), len(x)).copy(), x.copy(), y.copy(), z.copy()

    def pc_levels(self):
        """Every grid the last pattern-centre search scored, in order (__init__.py:446-477): scores,
        x, y, z, winner (ix, iy, iz), walked, pattern_best (rows of ix, iy, iz), pattern_ncc,
        pattern_scores[n, nz, ny, nx]; density (None when the mean decided), peak, ballots, inliers."""
        out = []
        for lv in self._e.pc_history:
            x, y, z = lv["axes"]
            nx, ny, nz = len(x), len(y), len(z)

            def split(c):
                c = np.asarray(c, np.int64)
                return np.stack([c % nx, (c // nx) % ny, c // (nx * ny)], -1)

            out.append({"scores": lv["scores"].reshape(nz, ny, nx).copy(), "x": x.copy(), "y": y.copy(), "z": z.copy(),
                        "pattern_scores": lv["pat_scores"].reshape(-1, nz, ny, nx).copy(),
                        "density": None if lv["density"] is None else lv["density"].reshape(nz, ny, nx).copy(),
                        "peak": tuple(float(v) for v in lv["peak"]), "ballots": int(lv["ballots"]),
                        "inliers": int(lv["inliers"]), "winner": tuple(int(v) for v in split(lv["best"])),
                        "walked": bool(lv["walked"]), "pattern_best": split(lv["pat_best"]),
                        "pattern_ncc": lv["pat_ncc"].copy()})
        return out

    # ── the plane of source points ──

    def fit_plane(self):
        """Fit the plane of source points (planefit.zig; __init__.py:487-523): every plane_stride-th
        cell each way (at most plane_patterns_max) fitted by itself, its orientation and the place
        of its own source, from the geometry as it stands; then the transformation of the scan's
        indices through those points (plane_kind affine or projective; plane_method "points"), or
        fitted to all the patterns at once ("joint"). The geometry takes the plane. Returns the
        reference's dict: plane (4 × 3), kind, frame, model, method, pc, pc_se, start_pc, rot,
        n_patterns, n_used, rmsd, ncc, start_ncc, iterations, said (rot, rot_se, sample_tilt_deg,
        sample_tilt_se_deg, step, step_se, skew, skew_se, blocks)."""
        from . import planefit

        return self._plane_result(self._call("fit_plane", planefit.fit_plane, self._e))

    def fit_geometry(self):
        """The automatic fit from the geometry as it was given (set_geometry): the vote for the
        pattern centre, then the fit patterns' own source points from there and the simplest model
        of how they move over the scan the map supports (one centre with the scan's steps, a tilt
        line, or the plane); `models` gives each one's cross-validated error (cv, cv_se)."""
        from . import planefit

        return self._plane_result(self._call("fit_geometry", planefit.auto, self._e))

    def _plane_result(self, r):
        import math

        models = ("centre", "line", "affine", "projective")
        g = self.geometry
        se = r["se"]
        sd = r["said"]
        return {"plane": r["plane"].copy(), "kind": ("none", "affine", "projective")[r["kind"]],
                "frame": "follow" if r["frame"] else "nominal", "model": r["model"], "method": r["method"],
                "models": {m: {"cv": r["cv"][i], "cv_se": r["cv_se"][i]} for i, m in enumerate(models)
                           if r["compared"] and r["cv"][i] > 0},
                "pc": list(r["pc"]), "pc_se": list(se[6:9]), "start_pc": r["start_pc"], "rot": r["rot"],
                "n_patterns": r["n_patterns"], "n_used": r["n_used"], "rmsd": list(r["rmsd"]), "ncc": r["ncc"],
                "start_ncc": r["start_ncc"], "iterations": r["iterations"],
                "said": {"rot": list(sd["rot"]), "rot_se": list(se[0:3]),
                         "sample_tilt_deg": g["sample_tilt_deg"] - math.degrees(sd["rot"][1]),
                         "sample_tilt_se_deg": math.degrees(se[1]), "step": list(sd["step"]), "step_se": list(se[3:5]),
                         "skew": sd["skew"], "skew_se": float(se[5]), "blocks": r["blocks"]}}

    def plane_points(self):
        """The source points the last plane fit measured, one a fit pattern: cells, pc (n × 3: where
        each pattern's own fit put its source), fit (n × 3: where the plane has it), ncc, used."""
        p = self._e.plane_points
        if p is None:
            z = np.zeros((0, 3))
            return {"cells": np.zeros(0, np.uint64), "pc": z, "fit": z.copy(), "ncc": np.zeros(0),
                    "used": np.zeros(0, bool)}
        return {k: v.copy() for k, v in p.items()}

    # ── one pattern ──

    def pattern(self, cell, processed=True, full=False):
        """One pattern as float32 (h, w), at the reduced size (the `binning` setting) or (`full`) the
        stored one (__init__.py:306-319). `processed`: True, as it is indexed (averaged with its
        neighbours when `nlpar` is on, then filtered); False, as it is stored; "averaged", averaged
        with its neighbours and not filtered; "background", the static background subtracted from
        every pattern (an error when `static_background` subtracts none)."""
        stage = {"averaged": 2, "background": 3}.get(processed) if isinstance(processed, str) else int(bool(processed))
        if stage is None:
            raise Error(f"pattern: processed={processed!r}")
        return self._call("pattern", self._e.pattern, int(cell), stage, bool(full))

    def nlpar_view(self):
        """What averaging with its neighbours did to the pattern `pattern` last returned
        (__init__.py:321-334): noise (its standard deviation a pixel, as stored), left (the share of
        it the average keeps), own (the average's share of the pattern itself) and shares (side ×
        side of the stored patterns around it, NaN outside the map); None when it was not averaged."""
        v = self._e._nl_view
        return None if v is None else dict(v, shares=v["shares"].copy())

    def fit_patterns(self):
        """The last fit's patterns: (cells, phases, quaternions in the fundamental zone, scores)."""
        f = self._e.fit
        if f is None:
            return np.zeros(0, np.uint64), np.zeros(0, np.int32), np.zeros((0, 4), np.float32), np.zeros(0, np.float32)
        return f["cells"].astype(np.uint64), f["phase"].copy(), f["quats"].copy(), f["ncc"].copy()

    def chance(self, phase=0):
        self._call("chance", self._e.calibrate)
        return float(self._e.chance_med[phase]), float(self._e.chance_spread[phase])

    def index_begin(self):
        self._call("index", self._e.index_begin)

    def index_step(self):
        return self._call("index", self._e.index_step)

    @property
    def index_status(self):
        return self._e.status()

    @property
    def sweep_plan(self):
        return [tuple(self._e.set.sweep(i)) for i in range(self._e.set["sweeps"])]

    def index(self, progress=None):
        """Index the region through every sweep (the loop of index_step, pipelined on the device);
        progress(status) is called after each device pass and stops the run by returning False
        (the one pass already in flight then still lands)."""
        self.index_begin()
        self._call("index", self._e.index_run, progress)
        return self.results()

    def results(self):
        rows, cols, h, w = self._e.info()
        r = self._e.res
        return {"quaternions": r["quat"].reshape(rows, cols, 4).copy(),
                "euler": r["euler"].reshape(rows, cols, 3).copy(),
                "ncc": r["ncc"].reshape(rows, cols).copy(), "nmi": r["nmi"].reshape(rows, cols).copy(),
                "phase": r["phase"].reshape(rows, cols).copy(), "z": r["z"].reshape(rows, cols).copy(),
                "sweep": r["sweep"].reshape(rows, cols).copy()}

    def map(self, kind="ipf_z"):
        """A result map as RGBA uint8 (rows, cols, 4) (__init__.py:790-795, output.zig:15-84): "ncc",
        "nmi" and "z" as gray between the indexed cells' extremes, "phase" and "sweep" in the
        reference's palette (dark gray: no sweep accepted the cell); cells not indexed transparent
        black. The IPF maps ("ipf_x", "ipf_y", "ipf_z") are not built: they raise."""
        from . import output as O

        rows, cols, h, w = self._call("map", self._e.info)
        if kind not in O.MAPS:
            raise Error(f"map: UnknownKind {kind!r}")
        return self._call("map", O.result_map, O.MAPS[kind], self._e.res).reshape(rows, cols, 4)

    def cell_under(self, cell, bandwidth=None, full=False, **fields):
        """Index one map cell and simulate it under another geometry than the one in use, which
        stays as it is (__init__.py:198-212): the fields given change it as for `set_geometry`
        (e.g. cell_under(c, pc=file_pc) to set two pattern centres side by side). The spherical
        correlation at `bandwidth` (default fit_bandwidth), then the refinement. Returns the best
        phase's {phase, quaternion, ncc, nmi, simulation} (the simulation at the stored size with
        `full`)."""
        bw = int(bandwidth or self._e.set["fit_bandwidth"])
        p, recs, sim = self._cell_under(cell, bw, full, fields)
        r = recs[p, 0]
        return {"phase": p, "quaternion": r[:4].copy(), "ncc": float(r[4]), "nmi": float(r[5]), "simulation": sim}

    def _cell_under(self, cell, bw, full, fields):
        """cell_under's work: (the best phase, every phase's record [phases][1][8], its simulation)."""
        e = self._e
        keep = e.geo
        tmp = keep.copy()
        self._call("cell_under", tmp.given, fields, type(keep)())
        if not tmp.px_um > 0:
            tmp.px_um = e.default_px()
        try:
            e.geo = tmp
            recs = self._call("cell_under", e.index_cells, np.array([int(cell)], np.int64), bw, "spherical", None,
                              False)
            p = int(e.choose_phase(recs)[0])
            r = recs[p, 0]
            binning = e.set["binning"]
            if full and binning != 1:
                e.set.apply({"binning": 1.0})
            try:
                sim = self._call("cell_under", e.simulate, p, np.array([int(cell)]), r[None, :4])[0]
            finally:
                if full and binning != 1:
                    e.set.apply({"binning": binning})
        finally:
            e.geo = keep
        return p, recs, sim

    # ── the device's own accounts ──

    def gpu_counts(self):
        """GPU traffic since the last call (__init__.py:938-942): kernel launches (dispatches),
        device passes (submits), readbacks to the host (reads) and host waits on the device (waits)."""
        from . import _native as N

        c = self._e.counts
        now = {"dispatches": N.launches["count"], "submits": c["submits"], "reads": c["reads"], "waits": c["waits"]}
        last, self._counts_seen = getattr(self, "_counts_seen", None) or dict.fromkeys(now, 0), now
        return {k: int(now[k] - last[k]) for k in now}

    def profile(self, on=True):
        """Time every kernel entry point on the GPU from now on (CUDA events on the stream it runs
        on; __init__.py:944-946); profile_report() gives the totals. Returns True (timing is
        always available here)."""
        from . import _native as N

        if on and not N.profiling["on"]:
            N.profiling["pairs"], N.profiling["totals"] = [], {}
        N.profiling["on"] = bool(on)
        return True

    def profile_report(self):
        """The profile's totals per entry point since profile(True): calls, device milliseconds,
        microseconds a call and share of the whole, largest first (__init__.py:948-951)."""
        from . import _native as N

        N.profile_flush(wait=True)
        rows = sorted(N.profiling["totals"].items(), key=lambda kv: -kv[1][1])
        total = sum(v[1] for _, v in rows) or 1.0
        lines = [f"{'entry point':<34} {'calls':>7} {'ms':>10} {'us/call':>10} {'share':>7}"]
        for name, (n, ms) in rows:
            lines.append(f"{name:<34} {n:>7d} {ms:>10.3f} {1000 * ms / max(n, 1):>10.1f} {100 * ms / total:>6.1f}%")
        lines.append(f"{'total':<34} {sum(v[0] for _, v in rows):>7d} {total if rows else 0.0:>10.3f}")
        return "\n".join(lines) + "\n"

    def reduce(self, quaternions, phase=0):
        from .rotations import to_bunge, to_fz

        q = to_fz(np.asarray(quaternions, np.float64).reshape(-1, 4), self._e.phases[phase].master.rotations())
        return q.astype(np.float32), to_bunge(q)

    def disorientation(self, a, b, phase=0):
        from .rotations import disorientation

        qa = np.asarray(a, np.float32).reshape(-1, 4).astype(np.float64)
        qb = np.asarray(b, np.float32).reshape(-1, 4).astype(np.float64)
        return disorientation(qa, qb, self._e.phases[phase].master.rotations())


from .api import Result, fit_pattern_center, fit_plane, index, load_patterns  # noqa: E402,F401
