"""Pattern-centre fit by voting (the reference's src/pcfit.zig, run 319-574).

A few patterns on a fit_grid × fit_grid lattice over the region are correlated on the sphere
under every candidate pattern centre of a grid around the current one. A wrong centre distorts
a pattern on the sphere so that no rotation of the master fits it, so each pattern's best
normalized correlation is a surface over the candidates that is high near the truth. The
surfaces decide by `pc_vote`: "mean" takes the highest mean; "ballots" (the default) lets each
pattern vote for its pc_top_k best candidates (gated at pc_gate × its own best), spreads the
ballots by a Gaussian of pc_kde_sigma on the detector, takes the densest place, moves it once to
the weighted centre of the ballots within pc_inlier_radius and finds the mode of those alone.
The search repeats pc_levels times, narrowing by pc_shrink, and a grid whose choice lies on its
border is first moved onto it at the same width (up to four times per level).

Device side: every candidate has its own window on the sphere and therefore its own denominator
volume; one tile holds whole candidates (their windows' volumes built together, FP32), and the
tile's items — each fit pattern at each candidate's position less its beam offset — go through
the same sphere, spectrum (tensor cores in the BF16 forms) and peak kernels as indexing, item b
of the tile normalized by volume b / n_patterns (zeb_correlate_peaks' rden_div). With several
phases each item is also scored on the detector (NCC, NMI at its peak, no refinement) so that the
phases compete as in indexing. One readback per grid; the vote itself is host arithmetic.
"""
import ctypes
import math

import numpy as np
import torch

from . import _native as N
from . import rotations as R
from .device import ptr, stream_ptr

MAX_WALK = 4  # times one level's grid may be moved onto a winner at its border (pcfit.zig:43)
FLAG_CENTER, FLAG_NORM, FLAG_WINDOW = 1, 2, 4


class PcError(RuntimeError):
    """NoPcSupport, NoPcCandidates, SearchTooLarge, NoPhases: the reference's error names."""


# ── the fit patterns ──

def _rect(region, cols):
    c_first, c_last = int(region[0]), int(region[-1])
    x0, y0 = c_first % cols, c_first // cols
    return x0, y0, c_last % cols - x0 + 1, c_last // cols - y0 + 1


def fit_cells(region, cols, grid):
    """pcfit.zig:63-87 — grid × grid cells, each at the centre of its share of the region's
    rectangle (the whole region when it is smaller than the lattice)."""
    x0, y0, w, h = _rect(region, cols)
    gy, gx = min(grid, h), min(grid, w)
    rows = y0 + (2 * np.arange(gy) + 1) * h // (2 * gy)
    cs = x0 + (2 * np.arange(gx) + 1) * w // (2 * gx)
    return (rows[:, None] * cols + cs[None, :]).reshape(-1).astype(np.int64)


def fit_cells_every(region, cols, stride):
    """pcfit.zig:91-113 — every stride-th cell of the region along rows and columns, centred."""
    x0, y0, w, h = _rect(region, cols)
    st = max(int(stride), 1)
    gy, gx = (h + st - 1) // st, (w + st - 1) // st
    oy, ox = (h - 1 - (gy - 1) * st) // 2, (w - 1 - (gx - 1) * st) // 2
    rows = y0 + oy + np.arange(gy) * st
    cs = x0 + ox + np.arange(gx) * st
    return (rows[:, None] * cols + cs[None, :]).reshape(-1).astype(np.int64)


# ── the vote's arithmetic ──

def axis(centre, span, steps):
    """pcfit.zig:115-121 — steps values over centre ± span (the centre alone for one step)."""
    if steps == 1:
        return np.array([centre], np.float64)
    k = np.arange(steps, dtype=np.float64)
    return centre - span + 2 * span * k / (steps - 1)


def valid_depth(z, zmin):
    """pcfit.zig:125-127 — in front of the detector and no nearer than pc_z_min."""
    return bool(math.isfinite(z) and z > 0 and z >= zmin)


def vertex(lo, mid, hi):
    """pcfit.zig:130-134 — offset (steps) of the parabola's maximum through three values."""
    den = lo - 2 * mid + hi
    if den >= -1e-15:
        return 0.0
    return min(max(0.5 * (lo - hi) / den, -0.5), 0.5)


def max_of(m, lo, hi):
    """pcfit.zig:177-188 — the first candidate of [lo, hi) with the largest finite value above 0."""
    v = np.asarray(m[lo:hi], np.float64)
    ok = np.isfinite(v) & (v > 0)
    if not ok.any():
        raise PcError("NoPcSupport")
    v = np.where(ok, v, -np.inf)
    return lo + int(np.argmax(v))


def peak_at(m, lo, hi, n, best):
    """pcfit.zig:192-206 — the maximum at `best`, each coordinate moved by the parabola through
    its two neighbours where both are scored."""
    at = (best % n[0], (best // n[0]) % n[1], best // (n[0] * n[1]))
    strides = (1, n[0], n[0] * n[1])
    out = [float(a) for a in at]
    for a in range(3):
        if n[a] < 3 or at[a] == 0 or at[a] == n[a] - 1:
            continue
        i0, i1 = best - strides[a], best + strides[a]
        if i0 >= lo and i1 < hi:
            out[a] += vertex(float(m[i0]), float(m[best]), float(m[i1]))
    return out


def _sigma(s, step):
    """The spread of a ballot in candidate steps along each axis: pc_kde_sigma on the detector,
    never narrower than the candidates can show (pcfit.zig:248-250)."""
    return [max(s["pc_kde_sigma"] / step[a], 0.75) if step[a] > 0 else 1.0 for a in range(3)]


def splat(ballots, n, sigma):
    """pcfit.zig:210-236 — the ballots' density over the grid (float32, ballot by ballot), by the
    library's host function zeb_pc_splat."""
    out = np.zeros(n[0] * n[1] * n[2], np.float32)
    at = np.ascontiguousarray([b[0] for b in ballots], np.int32).reshape(-1, 3)
    w = np.ascontiguousarray([b[1] for b in ballots], np.float64)
    nn = np.ascontiguousarray(n, np.int32)
    sg = np.ascontiguousarray(sigma, np.float64)
    N.call("zeb_pc_splat", at.ctypes.data, w.ctypes.data, len(ballots), nn.ctypes.data, sg.ctypes.data,
           out.ctypes.data)
    return out


def _ballots(s, pat_scores, n_pat, n):
    """Each pattern's best candidates from the top down, while at least pc_gate × its best and
    above 0, at most pc_top_k of them (pcfit.zig:258-296); with pc_nms only local maxima."""
    n_c = n[0] * n[1] * n[2]
    k = min(int(s["pc_top_k"]), n_c)
    half = int(s["pc_nms"]) // 2 if s["pc_nms"] > 1 else 0
    out = []
    for b in range(n_pat):
        sc = pat_scores[b * n_c:(b + 1) * n_c]
        top = float(sc.max())
        order = np.argsort(-sc, kind="stable")
        v = sc[order].astype(np.float64)
        ok = (v >= s["pc_gate"] * top) & (v > 0)
        stop = int(np.argmin(ok)) if not ok.all() else n_c
        cast = 0
        for c in order[:stop]:
            if cast == k:
                break
            c = int(c)
            at = (c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1]))
            if half > 0:
                vol = sc.reshape(n[2], n[1], n[0])
                nb = vol[max(at[2] - half, 0):at[2] + half + 1, max(at[1] - half, 0):at[1] + half + 1,
                         max(at[0] - half, 0):at[0] + half + 1]
                if (nb > sc[c]).any():
                    continue
            out.append((at, float(sc[c])))
            cast += 1
    return out


def consensus(s, pat_scores, n_pat, n, step, lo, hi):
    """pcfit.zig:244-318 — the grid's choice by ballots: (peak in candidate steps, winner,
    the first density, (ballots cast, inliers))."""
    sigma = _sigma(s, step)
    ballots = _ballots(s, pat_scores, n_pat, n)
    if not ballots:
        raise PcError("NoPcSupport")
    density = splat(ballots, n, sigma)
    best = max_of(density, lo, hi)
    mode = peak_at(density, lo, hi, n, best)
    r2 = s["pc_inlier_radius"] * s["pc_inlier_radius"]
    at = np.array([b[0] for b in ballots], np.float64)  # [B][3]
    w = np.array([b[1] for b in ballots], np.float64)
    st = np.asarray(step, np.float64)

    def near(p):
        d = (at - np.asarray(p, np.float64)[None, :]) * st[None, :]
        return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2] <= r2

    # once to the weighted centre of the ballots around the mode (sums in ballot order) …
    sel = near(mode)
    if sel.any():
        acc = [float(np.cumsum(w[sel] * at[sel, a])[-1]) for a in range(3)] + [float(np.cumsum(w[sel])[-1])]
    else:
        acc = [0.0] * 4
    pk = [acc[a] / acc[3] for a in range(3)] if acc[3] > 0 else mode
    keep = near(pk)  # … then the mode of those alone
    kept = [bw for bw, k in zip(ballots, keep) if k]
    if not kept:
        raise PcError("NoPcSupport")
    inl = splat(kept, n, sigma)
    winner = max_of(inl, lo, hi)
    return peak_at(inl, lo, hi, n, winner), winner, density, (len(ballots), len(kept))


def search(s, pc0, n_pat, score):
    """pcfit.zig:319-574 without the device: score(candidates [k][3]) gives the fit patterns'
    scores under those candidates ([n_pat][k] float32, each pattern's phase chosen). Returns
    (result fields, the grids as scored, the index of the winner in the last grid)."""
    steps = (int(s["pc_steps"]), int(s["pc_steps"]), int(s["pc_steps_z"]))
    span = [s["pc_span"], s["pc_span"], s["pc_span_z"]]
    n_c = steps[0] * steps[1] * steps[2]
    if n_c * n_pat > 4 << 20:
        raise PcError("SearchTooLarge")
    xy = steps[0] * steps[1]
    pc = [float(v) for v in pc0]
    res = {"start": list(pc), "n_patterns": int(n_pat), "n_candidates": 0, "levels": int(s["pc_levels"]),
           "start_score": 0.0, "score": 0.0, "at_border": False}
    history = []
    level, walked, best_c = 0, 0, 0
    while level < s["pc_levels"]:
        axes = [axis(pc[a], span[a], steps[a]) for a in range(3)]
        if not (np.isfinite(axes[0]).all() and np.isfinite(axes[1]).all()):
            raise PcError("NoPcCandidates")
        ok = [valid_depth(float(z), s["pc_z_min"]) for z in axes[2]]
        if not any(ok):
            raise PcError("NoPcCandidates")
        z0 = ok.index(True)
        z1 = z0 + 1
        while z1 < len(ok) and ok[z1]:
            z1 += 1
        lo, hi = z0 * xy, z1 * xy
        c = np.arange(lo, hi)
        cands = np.stack([axes[0][c % steps[0]], axes[1][(c // steps[0]) % steps[1]], axes[2][c // xy]], 1)
        got = np.asarray(score(cands), np.float32).reshape(n_pat, hi - lo)
        pat = np.zeros((n_pat, n_c), np.float32)
        pat[:, lo:hi] = np.where(np.isfinite(got), got, np.float32(0))
        acc = np.zeros(hi - lo, np.float64)
        for b in range(n_pat):  # pattern by pattern, as the reference sums
            acc += pat[b, lo:hi]
        scores = np.zeros(n_c, np.float32)
        scores[lo:hi] = (acc / n_pat).astype(np.float32)
        best_c = max_of(scores, lo, hi)
        res["n_candidates"] += hi - lo
        pb = lo + np.argmax(pat[:, lo:hi], axis=1)
        lvl = {"axes": axes, "scores": scores, "pat_scores": pat.reshape(-1), "pat_best": pb.astype(np.uint32),
               "pat_ncc": pat[np.arange(n_pat), pb].astype(np.float32), "density": None, "peak": [0.0] * 3,
               "ballots": 0, "inliers": 0, "walked": 0, "scored": (lo, hi)}
        history.append(lvl)
        voted = None
        if s["pc_vote"] == "ballots":
            step = [float(axes[a][1] - axes[a][0]) if steps[a] > 1 else 0.0 for a in range(3)]
            voted, best_c, lvl["density"], (lvl["ballots"], lvl["inliers"]) = consensus(
                s, lvl["pat_scores"], n_pat, steps, step, lo, hi)
        lvl["best"] = int(best_c)
        bi = (best_c % steps[0], (best_c // steps[0]) % steps[1], best_c // xy)
        if voted is not None:
            peak = list(voted)
        elif level + 1 == s["pc_levels"]:
            peak = peak_at(scores, lo, hi, steps, best_c)
        else:
            peak = [float(v) for v in bi]
        lvl["peak"] = peak
        if level == 0 and walked == 0:
            mid = (steps[0] // 2) + steps[0] * ((steps[1] // 2) + steps[1] * (steps[2] // 2))
            res["start_score"] = float(scores[mid])
        for a in range(3):
            st = float(axes[a][1] - axes[a][0]) if steps[a] > 1 else 0.0
            pc[a] = float(axes[a][bi[a]]) + (peak[a] - bi[a]) * st
        if not (math.isfinite(pc[0]) and math.isfinite(pc[1]) and valid_depth(pc[2], s["pc_z_min"])):
            raise PcError("NoPcCandidates")
        res["score"] = float(scores[best_c])
        res["at_border"] = any(steps[a] > 1 and bi[a] in (0, steps[a] - 1) for a in range(3))
        if res["at_border"] and walked < MAX_WALK:
            lvl["walked"] = 1
            walked += 1
            continue
        walked = 0
        level += 1
        if level < s["pc_levels"]:
            span = [v * s["pc_shrink"] for v in span]
    res["pc"] = pc
    return res, history, int(best_c)


# ── the device side ──

class Scorer:
    """Scores the fit patterns under candidate pattern centres on the device (pcfit.zig:397-488):
    per candidate tile, the windows' denominator volumes, then every (candidate, pattern) item's
    coefficients, spectrum and peak; with several phases also its NCC and NMI at the peak."""

    def __init__(self, e, cells, timer=None):
        self.e = e
        self.mark = timer.mark if timer is not None else (lambda name: None)
        s = e.set
        self.cells = np.asarray(cells, np.int64)
        self.n_pat = len(self.cells)
        self.b = e.band(int(s["fit_bandwidth"]))
        self.fr = e.frame()
        rows, cols, h, w = e.info()
        bn = s["binning"]
        self.size = (h / bn, w / bn)
        # each pattern's beam offset (pixels), the same under every candidate (engine.zig:1588-1598)
        self.offs = e.geo.scan_offsets(self.cells // cols, self.cells % cols, 0.5 * (rows - 1), 0.5 * (cols - 1),
                                       s["scan_x_sign"], s["scan_y_sign"], bn)
        hb, wb = e.pattern_shape()
        self.pats = e.upload(self.cells)[: self.n_pat * hb * wb].clone()  # (the engine's buffer is shared)
        self.n_ph = len(e.phases)
        per = max(N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), 1) for _, ph in self.b["phases"].values())
        tile = int(min(4096, max(512, (int(s["tile_mb"]) << 20) // per)))  # spherical.zig:311-315
        self.tile = tile
        self.cand_per_tile = max(1, tile // self.n_pat)
        self.last = None  # the last grid's peaks and phase choice, for the fit patterns' poses

    def _window_rden(self, ph, ts):
        """Reciprocal denominators of k windows at positions ts ([k][3]): [k][cells]
        (spherical.zig:448-464, as Engine.denominators for many windows at once)."""
        e, bt, fr = self.e, self.b["tables"], self.fr
        k = len(ts)
        cells = ph.volume_cells()
        rden = torch.empty(k * cells, dtype=torch.float32, device=e.dev)
        for w0 in range(0, k, 512):
            nw = min(512, k - w0)
            items = e.to_device("pc_windows", np.concatenate([ts[w0:w0 + nw], np.zeros((nw, 1))], 1).astype(np.float32))
            alm = e.buf("pc_walm", nw * bt.n_pairs * 2)
            stats = e.buf("pc_wstats", nw * 4)
            scratch = e.buf("sphere_scratch", N.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), nw) // 4 + 1)
            self.mark("windows_sphere")
            N.call("zeb_sphere_coefficients", None, ptr(items), nw, ctypes.byref(fr), ctypes.byref(bt.st), FLAG_WINDOW,
                   ptr(alm), ptr(stats), ptr(scratch), stream_ptr())
            U = e.buf("spec", N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), nw) // 4 + 1)
            vols = []
            for name, Y in (("pc_vol_f", ph.Y_f), ("pc_vol_f2", ph.Y_f2)):
                self.mark("windows_spectrum")
                e.spectrum(alm, nw, ph, Y, U, tensor_cores=False)
                vol = e.buf(name, nw * cells)
                self.mark("windows_volume")
                N.call("zeb_correlate_volume", ptr(U), nw, ctypes.byref(ph.dims), ptr(self.b["tables"].tw), ptr(vol),
                       stream_ptr())
                vols.append(vol)
            self.mark("windows_rden")
            N.call("zeb_rden_build", ptr(vols[0]), ptr(vols[1]), ptr(stats), nw, cells, ptr(rden[w0 * cells:]),
                   stream_ptr())
        return rden

    def __call__(self, cands):
        """The fit patterns' scores under the candidates ([k][3] pattern centres): [n_pat][k]."""
        e, s, fr = self.e, self.e.set, self.fr
        bt = self.b["tables"]
        n_pat, k_all = self.n_pat, len(cands)
        c = np.asarray(cands, np.float64)
        rows, cols = self.size
        # each candidate's detector position (geometry.zig:74-76), all at once
        v = (0.5 - c[:, 1] * rows, 0.5 - c[:, 0] * cols, c[:, 2] * rows)
        Rm = e.geo.rotation()
        t_c = np.stack([Rm[i, 0] * v[0] + Rm[i, 1] * v[1] + Rm[i, 2] * v[2] for i in range(3)], 1)
        # one set of ring spans for the whole grid (every item's position inside its box), so that
        # how the grid is cut into tiles changes no bit of the coefficients
        t_all = (t_c[:, None, :] - self.offs[None, :, :]).reshape(-1, 3).astype(np.float32)
        e._batch_t = (t_all.min(0), t_all.max(0))
        spans = e.spans(bt, fr)
        peaks = torch.empty(self.n_ph * k_all * n_pat * 8, dtype=torch.float32, device=e.dev)
        recs = torch.empty(self.n_ph * k_all * n_pat * 8, dtype=torch.float32, device=e.dev) if self.n_ph > 1 else None
        opts = N.RefineOpts(0, math.radians(s["refine_step"]), 1.0, 0.02, 1e4, s["nmi_bins"], 1.0)
        for c0 in range(0, k_all, self.cand_per_tile):
            if e.cancel:
                raise PcError("Cancelled")
            k = min(self.cand_per_tile, k_all - c0)
            self.mark("windows")
            rdens = [self._window_rden(self.b["phases"][pi][1], t_c[c0:c0 + k]) for pi in range(self.n_ph)]
            # the tile's items: candidate-major, each pattern at the candidate's position less its offset
            t = t_all[c0 * n_pat:(c0 + k) * n_pat]
            idx = np.tile(np.arange(n_pat, dtype=np.float32), k)[:, None]
            n_items = k * n_pat
            whole = n_items <= self.tile  # whole candidates in one go, else one candidate in parts
            for f0 in range(0, n_items, n_items if whole else self.tile):
                ni = min(n_items - f0, n_items if whole else self.tile)
                items = e.to_device("pc_items", np.concatenate([t[f0:f0 + ni], idx[f0:f0 + ni]], 1))
                alm = e.buf("alm", ni * bt.n_pairs * 2)
                stats = e.buf("stats", ni * 4)
                scratch = e.buf("sphere_scratch", N.load().zeb_sphere_scratch_bytes(ctypes.byref(bt.st), ni) // 4 + 1)
                self.mark("sphere")
                N.call("zeb_sphere_coefficients_spans", ptr(self.pats), ptr(items), ni, ctypes.byref(fr),
                       ctypes.byref(bt.st), ptr(spans), FLAG_CENTER | FLAG_NORM, ptr(alm), ptr(stats), ptr(scratch),
                       stream_ptr())
                # whole candidates: item j reads the volume of its candidate, j / n_pat; a part of
                # one candidate: that candidate's volume alone
                div = n_pat if whole else 1 << 30
                for pi, p in enumerate(e.phases):
                    ph = self.b["phases"][pi][1]
                    U = e.buf("spec", N.load().zeb_spectrum_bytes(ctypes.byref(ph.dims), ni) // 4 + 1)
                    self.mark("spectrum")
                    e.spectrum(alm, ni, ph, ph.Y_f, U)
                    cand = e.buf("cand", N.load().zeb_peaks_scratch_bytes(ctypes.byref(ph.dims), ni) // 4 + 1)
                    self.mark("peaks")
                    at = (pi * k_all * n_pat + c0 * n_pat + f0) * 8
                    N.call("zeb_correlate_peaks", ptr(U), ni, ctypes.byref(ph.dims), ptr(bt.tw), ptr(rdens[pi]), div,
                           ptr(peaks[at:]), ptr(cand), stream_ptr())
                    if recs is not None:  # the phases compete on their NMI (or NCC) at their peaks
                        self.mark("records")
                        e.refine(self.pats, items, peaks[at:], ni, fr, p, opts, recs[at:])
        self.mark("readback")
        pk = peaks.cpu().numpy().reshape(self.n_ph, k_all, n_pat, 8)
        e.check_device()
        if recs is not None:
            rc = recs.cpu().numpy().reshape(self.n_ph, k_all, n_pat, 8)
            col = 5 if s["phase_by"] == "nmi" else 4
            v = rc[..., col]
            choice = np.argmax(np.where(np.isnan(v), -np.inf, v), axis=0)  # the first best; 0 when none
        else:
            choice = np.zeros((k_all, n_pat), np.int64)
        val = np.take_along_axis(pk[..., 4], choice[None], 0)[0]  # [k][n_pat]
        pk[..., 4] = np.where(np.isfinite(pk[..., 4]), pk[..., 4], np.float32(0))
        self.last = (pk, choice)
        self.mark("vote")  # (until the next grid's first mark: the host's share)
        return val.T

    def poses(self, j):
        """The fit patterns' orientations (fundamental zone), phases and scores at candidate j
        of the last grid scored (pcfit.zig:540-561)."""
        pk, choice = self.last
        ph = choice[j]
        r = pk[ph, j, np.arange(self.n_pat)]  # [pattern][8], each of its own phase
        q = np.empty((self.n_pat, 4), np.float32)
        for p in np.unique(ph):
            sel = ph == p
            q[sel] = R.to_fz(r[sel, :4].astype(np.float64), self.e.phases[int(p)].master.rotations())
        return q, ph.astype(np.int32), r[:, 4].astype(np.float32)


def run(e, timer=None):
    """The vote (pcfit.zig:319-574): the fitted pattern centre goes into the geometry and the
    record of the search into the engine; nothing changes when the search fails. timer.mark(stage)
    (CUDA events) at the stage boundaries when given."""
    if not e.phases:
        raise PcError("NoPhases")
    s = e.set
    rows, cols = e.info()[:2]
    cells = fit_cells(e.region_cells(), cols, int(s["fit_grid"]))
    mark = timer.mark if timer is not None else (lambda name: None)
    mark("setup")  # the band's tables, the fit patterns' upload
    sc = Scorer(e, cells, timer)
    res, history, best = search(s, e.geo.pc, len(cells), sc)
    mark("end")
    lo = history[-1]["scored"][0]
    q, ph, ncc = sc.poses(best - lo)
    # (the vote moves one pattern centre, the scan's steps saying how the beam went from it: a
    # plane fitted before goes)
    e.geo.pc = np.array(res["pc"], np.float64)
    e.geo.plane_kind = 0
    e.pc_history = history
    e.fit = {"cells": cells, "quats": q, "phase": ph, "ncc": ncc}
    e.log(f"pattern centre {res['pc'][0]:.5f} {res['pc'][1]:.5f} {res['pc'][2]:.5f}  mean NCC {res['score']:.4f} "
          f"(was {res['start_score']:.4f})")
    return res
