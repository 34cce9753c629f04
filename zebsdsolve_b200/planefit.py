"""The plane of source points: the geometry's fit after the pattern-centre vote (the reference's
src/planefit.zig; Winkelmann, Nolze, Cios, Tokarski and Bała, Materials 13 (2020) 2816; kikuchipy's
refine_orientation_projection_center then EBSDDetector.fit_pc).

Every plane_stride-th cell of the region each way (at most plane_patterns_max) is indexed at the
geometry as it stands; those whose match indexing would accept take part. Each is refined by
itself by Levenberg–Marquardt on its normalized cross-correlation with its simulation, over its
orientation and (method "points") the place of its own source: the device gives every pattern's 43
Gauss–Newton sums in one launch (zeb_sums6_list, the master bilinear, bicubic or by Keys' six-point
kernel as plane_interp says), the host forms each pattern's NCC, gradient and Gauss–Newton matrix
and takes all the patterns' damped steps at once, one readback a round. A transformation of the
scan's indices is then fitted through the measured source points (plane.py), or (method "joint")
the transformation's own numbers are fitted to all the patterns' scores at once. The geometry takes
the plane: every cell's source is then where it says.
"""
import ctypes
import math

import numpy as np
import torch

from . import _native as N
from . import plane as PL
from . import rotations as R
from .device import ptr, stream_ptr
from .pcfit import fit_cells_every

NS = 43
CHANCE_Z = 3.0  # planefit.zig:291-297: above chance by this many spreads when too few are accepted
CHANCE_SHARE = 10
INTERP = {"bilinear": 0, "bicubic": 1, "keys6": 2}
BL = 6  # blocks each way of the map for the model comparison and the standard errors


class PlaneError(RuntimeError):
    """NoPhases, TooFewFitPatterns, PatternTooLarge, Cancelled: the reference's error names."""


def pc_of(Rm, t, rows, cols):
    """geometry.zig:171-174 — pattern centres of detector positions t [n, 3]."""
    p = np.asarray(t, np.float64) @ Rm  # Rᵀ t, row by row
    return np.stack([(0.5 - p[..., 1]) / cols, (0.5 - p[..., 0]) / rows, p[..., 2] / rows], -1)


def local_of(s):
    """planefit.zig:176-200 for every pattern from its 43 sums [n, 43] (float32): (ok, NCC, g [n,6],
    H [n,6,6]) in FP64; ok false (and the rest zero) where the simulation has no variance."""
    s = np.asarray(s, np.float32)
    nn = np.maximum(s[:, 0], np.float32(1)).astype(np.float64)
    s = s.astype(np.float64)
    mean = s[:, 1] / nn
    var_n = s[:, 2] - nn * mean * mean
    ok = var_n > 1e-12
    inv = np.where(ok, 1.0 / np.sqrt(np.where(ok, var_n, 1.0)), 0.0)
    ncc = np.where(ok, s[:, 3] * inv, 0.0)
    sd = s[:, 4:10]
    au = (s[:, 10:16] - mean[:, None] * sd) * inv[:, None]
    g = np.where(ok[:, None], (s[:, 16:22] - ncc[:, None] * au) * inv[:, None], 0.0)
    P = np.zeros((len(s), 6, 6))
    iu = np.triu_indices(6)
    P[:, iu[0], iu[1]] = s[:, 22:43]
    P[:, iu[1], iu[0]] = s[:, 22:43]
    H = (P - sd[:, :, None] * sd[:, None, :] / nn[:, None, None] - au[:, :, None] * au[:, None, :]) \
        * (inv * inv)[:, None, None]
    H = np.where(ok[:, None, None], H, 0.0)
    return ok, ncc, g, H


def solve_batch(A, b):
    """planefit.zig:203-233 for many small systems at once: x [n, k] with A [n, k, k] x = b [n, k] by
    elimination with partial pivoting (the first largest pivot); ok false where a pivot is below
    1e-300 (x then zero)."""
    A = np.array(A, np.float64)
    b = np.array(b, np.float64)
    n, k = b.shape
    ok = np.ones(n, bool)
    idx = np.arange(n)
    for c in range(k):
        p = c + np.argmax(np.abs(A[:, c:, c]), axis=1)
        ok &= np.abs(A[idx, p, c]) >= 1e-300
        swap = p != c
        if swap.any():
            rows_c, rows_p = A[idx, c].copy(), A[idx, p].copy()
            A[idx[swap], c], A[idx[swap], p[swap]] = rows_p[swap], rows_c[swap]
            bc, bp = b[idx, c].copy(), b[idx, p].copy()
            b[idx[swap], c], b[idx[swap], p[swap]] = bp[swap], bc[swap]
        piv = np.where(ok, A[:, c, c], 1.0)
        for r in range(c + 1, k):
            f = A[:, r, c] / piv
            f = np.where(ok, f, 0.0)
            A[:, r, c:] -= f[:, None] * A[:, c, c:]
            b[:, r] -= f * b[:, c]
    x = np.zeros((n, k))
    for r in range(k - 1, -1, -1):
        acc = b[:, r].copy()
        for q in range(r + 1, k):
            acc -= A[:, r, q] * x[:, q]
        x[:, r] = acc / np.where(ok, A[:, r, r], 1.0)
    return np.where(ok[:, None], x, 0.0), ok


def damped(k, H, g, lam):
    """planefit.zig:236-248 — each pattern's system over its last k unknowns (3: the rotation; 6:
    with the source's shift), its diagonal × (1 + λ) + 1e-9 · trace + 1e-30."""
    o = 6 - k
    A = H[:, o:, o:].copy()
    tr = np.trace(A, axis1=1, axis2=2)
    d = np.arange(k)
    A[:, d, d] = A[:, d, d] * (1 + np.asarray(lam, np.float64).reshape(-1, 1)) + (1e-9 * tr)[:, None] + 1e-30
    return A, g[:, o:].copy()


def profiled(H, g):
    """planefit.zig:634-660 — each pattern's information on its source with its rotation profiled
    out: S = H_tt − H_tq H_qq⁻¹ H_qt, g̃ = g_t − H_tq H_qq⁻¹ g_q (symmetrized); ok false where the
    rotation is not told."""
    B, _ = damped(3, H, g, 0.0)
    S = np.empty((len(H), 3, 3))
    ok = np.ones(len(H), bool)
    for c in range(3):
        col, good = solve_batch(B, H[:, c, 3:6])
        ok &= good
        S[:, :, c] = H[:, 0:3, c] - np.einsum("nik,nk->ni", H[:, 0:3, 3:6], col)
    xg, good = solve_batch(B, g[:, 3:6])
    ok &= good
    gt = g[:, 0:3] - np.einsum("nik,nk->ni", H[:, 0:3, 3:6], xg)
    S = 0.5 * (S + np.transpose(S, (0, 2, 1)))
    return S, gt, ok


def _qstep(d, q):
    return R.qstd(R.qmul(R.exp_map(d), q))


class Fit:
    """planefit.zig:300-632 — the fit patterns, indexed at the geometry as it stands, each with its
    orientation and its source's shift away from where the geometry puts it."""

    def __init__(self, e, every, most):
        s = e.set
        e.cancel = False
        if not e.phases:
            raise PlaneError("NoPhases")
        self.e = e
        rows, cols, h, w = e.info()
        hb, wb = e.pattern_shape()
        self.sz = (h / s["binning"], w / s["binning"])
        region = e.region_cells()
        stride = int(every)
        cells = fit_cells_every(region, cols, stride)
        while len(cells) > 1 and most > 0 and len(cells) > most:
            stride += 1
            cells = fit_cells_every(region, cols, stride)
        if stride != every:
            e.log(f"fit patterns: a stride of {stride} cells each way, {len(cells)} patterns (asked every {every}; "
                  f"no more than {most})")
        self.cells = cells
        n = self.n = len(cells)
        self.geo0 = e.geo.copy()
        recs = e.index_cells(cells, bandwidth=s["fit_bandwidth"], method=s["method"], grid=s["dict_grid"])
        best = e.choose_phase(recs)
        self.phase = best.astype(np.int32)
        r = recs[best, np.arange(n)]
        still = np.float32(math.radians(s["accept_step_deg"]))
        good = r[:, 5] >= s["accept_nmi"] if s["accept_nmi"] > 0 else r[:, 7] >= s["accept_z"]
        self.use = good & ((not s["refine"]) | (r[:, 6] <= still))
        self.seed_ncc = r[:, 4].astype(np.float32)
        self.q = R.qstd(r[:, :4].astype(np.float64))
        self.shift = np.zeros((n, 3))
        self.base = e.positions64(cells)
        if self.use.sum() < 3:
            accepted = int(self.use.sum())
            self.use = r[:, 7] >= CHANCE_Z
            e.log(f"plane fit: {accepted} of the {n} fit patterns have a match that would be accepted here; fitting "
                  f"to the {int(self.use.sum())} above chance (z ≥ {CHANCE_Z:g})")
            if self.use.sum() < 3 or self.use.sum() * CHANCE_SHARE < n:
                raise PlaneError("TooFewFitPatterns")
        elif self.use.sum() < n:
            e.log(f"plane fit: {n - int(self.use.sum())} of the {n} fit patterns left out, their matches not accepted")
        self.n_used = int(self.use.sum())
        # the device side: the fit patterns filtered, the frame's pixel list, the engine's masters
        self.fr = e.frame()
        self.pats = e.upload(cells)[: n * hb * wb].clone()
        npix = N.load().zeb_mask_pixels(ctypes.byref(self.fr))
        if not 1 <= npix <= 51200:
            raise PlaneError(f"PatternTooLarge: {npix} masked pixels (the fit's kernel takes at most 51200)")
        self.list = torch.empty(npix, dtype=torch.int32, device=e.dev)
        N.call("zeb_mask_list", ctypes.byref(self.fr), ptr(self.list), stream_ptr())
        self.interp = INTERP[s["plane_interp"]]
        self.masters = None  # the fit's own resampled masters, or the engine's
        self.master_px = 0.0
        self.keep = None
        if s["plane_master_auto"]:
            # the master's pixel that suits these patterns: of a few widths, the one under which the
            # fit patterns correlate best, each with its orientations settled there
            seeds = self.q.copy()
            best_w, top, said = 0.0, -math.inf, []
            for width in (0.0, 0.5, 1.0, 1.5, 2.0):
                self.resample(width)
                self.q = seeds.copy()
                self.settle(3, 0.0, 60)
                said.append(f"{width:g}: {self.ncc:.4f}")
                if self.ncc > top:
                    top, best_w = self.ncc, width
            self.q = seeds.copy()
            self.resample(best_w)
            self.master_px = best_w
            e.log(f"plane fit: master pixel {best_w:g} detector pixels (0: as it is), the best of [{', '.join(said)}] "
                  "by the fit patterns' mean NCC")
        else:
            self.resample(s["plane_master_px"])
            self.master_px = s["plane_master_px"]
        self.ncc, self.keep = self.eval(self.q, self.shift)

    def resample(self, want):
        """planefit.zig:377-454 — the fit's own masters: each phase's filtered sheets resampled so
        that a master pixel is `want` detector pixels wide at the pattern centre (a tent-weighted
        average of the old pixels within one new pixel, along each way of the sheet); none (the
        engine's) for want ≤ 0 or where the sheet is already that coarse."""
        e = self.e
        self.masters = None
        if not want > 0:
            return
        pixel = e.pixel_angle()
        if not pixel > 0:
            return
        masters = []
        for p in e.phases:
            side = p.master.side
            across = math.sqrt(2.0 * math.pi) / (want * pixel)
            new = int(min(max(math.floor(across + 0.5) + 1, 16), side))
            if new >= side:
                masters.append(None)
                continue
            work = p.baked[1].reshape(2, side, side).cpu().numpy().astype(np.float32)
            ratio = (side - 1) / (new - 1)
            reach = int(math.ceil(ratio))
            span = 2 * reach + 1
            x = np.arange(new) * ratio
            first = np.maximum(np.floor(x) - reach + 1, 0).astype(np.int64)
            idx = first[:, None] + np.arange(span)[None, :]
            wts = np.maximum(1.0 - np.abs(idx - x[:, None]) / ratio, 0.0)
            wts = np.where(idx < side, wts, 0.0)
            wsum = wts.sum(1, keepdims=True)
            wts = (wts.astype(np.float32) / wsum).astype(np.float32)
            idx = np.minimum(idx, side - 1)
            out = np.empty((2, new, new), np.float32)
            for sh in range(2):
                src = work[sh]
                rows = np.zeros((side, new), np.float32)
                for k in range(span):  # along the columns, term by term in order
                    rows += wts[None, :, k] * src[:, idx[:, k]]
                acc = np.zeros((new, new), np.float32)
                for k in range(span):  # then along the rows
                    acc += wts[:, k, None] * rows[idx[:, k], :]
                out[sh] = acc
            sheets = torch.as_tensor(out.reshape(-1), device=e.dev)
            grad = torch.empty(sheets.numel() * 4, dtype=torch.float32, device=e.dev)
            N.call("zeb_master_gradient", ptr(sheets), ptr(grad), new, stream_ptr())
            vpair = torch.empty(sheets.numel() * 2, dtype=torch.float32, device=e.dev)
            gpair = torch.empty(sheets.numel() * 8, dtype=torch.float32, device=e.dev)
            N.call("zeb_master_pairs", ptr(sheets), ptr(grad), new, ptr(vpair), ptr(gpair), stream_ptr())
            masters.append((sheets, gpair, new))
        self.masters = masters

    def master_of(self, pi):
        own = self.masters[pi] if self.masters is not None else None
        if own is not None:
            return own
        p = self.e.phases[pi]
        return p.baked[1], p.baked[4], p.master.side

    def eval(self, q, shift):
        """planefit.zig:458-492 — the used patterns' mean NCC at orientations q and shifts, and every
        pattern's system (ok, NCC, g, H; zero for those left out)."""
        e, n = self.e, self.n
        t = (self.base + shift).astype(np.float32)
        items = e.to_device("plane_items", np.concatenate([t, np.arange(n, dtype=np.float32)[:, None]], 1))
        x = e.buf("plane_x", n * 6)[: n * 6]
        x.zero_()
        q0 = e.to_device("plane_q", np.asarray(q, np.float32))
        sums = torch.empty((len(e.phases), n, NS), dtype=torch.float32, device=e.dev)
        for pi in range(len(e.phases)):
            sheets, gpair, side = self.master_of(pi)
            N.call("zeb_sums6_list", ptr(self.pats), ptr(items), n, ctypes.byref(self.fr), ptr(self.list),
                   self.list.numel(), ptr(sheets), ptr(gpair), side, self.interp, ptr(x), ptr(q0), ptr(sums[pi]),
                   stream_ptr())
        sh = sums.cpu().numpy()
        own = sh[np.clip(self.phase, 0, len(e.phases) - 1), np.arange(n)]
        ok, ncc, g, H = local_of(own)
        live = self.use & (self.phase >= 0)
        ok = ok & live
        ncc = np.where(live, ncc, 0.0)
        g = np.where(live[:, None], g, 0.0)
        H = np.where(live[:, None, None], H, 0.0)
        return float(ncc[self.use].sum() / max(self.n_used, 1)), (ok, ncc, g, H)

    def settle(self, k, trust, most):
        """planefit.zig:570-622 — every used pattern to its own best by itself (k = 3: its
        orientation; k = 6: with its source's shift, clamped to ±trust pixels): each round all take a
        damped step together, kept where the pattern's own score rose (λ/3, at least 1e-4), else
        λ × 5 (at most 1e8); until a round gains the mean less than 1e-7 (a round whose every step
        overshot goes again) or after `most` rounds. Returns the rounds taken."""
        u = self.use
        count = max(self.n_used, 1)
        self.ncc, keep = self.eval(self.q, self.shift)
        lam = np.full(self.n, 1e-3)
        it = 0
        while it < most:
            if self.e.cancel:
                raise PlaneError("Cancelled")
            A, b = damped(k, keep[3], keep[2], lam)
            d, good = solve_batch(A, b)
            step = u & good
            q_t, s_t = self.q.copy(), self.shift.copy()
            if k == 6:
                s_t[step] = np.clip(self.shift[step] + d[step, :3], -trust, trust)
            q_t[step] = _qstep(d[step, k - 3:], self.q[step])
            _, now = self.eval(q_t, s_t)
            up = u & (now[1] > keep[1])
            gain = float((now[1] - keep[1])[up].sum())
            kept = int(up.sum())
            damp = int((u & ~up & (lam < 1e8)).sum())
            self.q[up], self.shift[up] = q_t[up], s_t[up]
            keep = tuple(np.where(up.reshape(-1, *([1] * (a.ndim - 1))), a2, a) for a, a2 in zip(keep, now))
            lam = np.where(up, np.maximum(lam / 3, 1e-4), np.where(u, np.minimum(lam * 5, 1e8), lam))
            if kept == 0 and damp > 0:  # (every step overshot: not converged, they go again)
                it += 1
                continue
            if gain / count < 1e-7:
                break
            it += 1
        self.keep = keep
        self.ncc = float(keep[1][u].sum() / count)
        return it


class Joint:
    """planefit.zig:635-700 — the joint fit's coordinates: a source's place y = (PCx · aspect, PCy,
    PCz) becomes the detector position t = R (½ − h y₁, ½ − h y₀, h y₂), ∂t/∂y = h M."""

    def __init__(self, fit, fr, Rm, h, cols):
        self.fit, self.fr, self.R, self.h, self.cols = fit, fr, Rm, h, cols
        self.M = np.array([[-Rm[k, 1], -Rm[k, 0], Rm[k, 2]] for k in range(3)])
        self.row = (fit.cells // cols).astype(np.float64)
        self.col = (fit.cells % cols).astype(np.float64)

    def sources(self, theta):
        """Each pattern's source where the model puts it, as a shift from where the fit began."""
        y, _ = PL.model_at(theta, self.fr, self.row, self.col)
        v = np.stack([0.5 - y[:, 1] * self.h, 0.5 - y[:, 0] * self.h, y[:, 2] * self.h], 1)
        return v @ self.R.T - self.fit.base

    def own_steps(self):
        """Each used pattern's pseudo-point step dy = W⁻¹ p and weight W = h² Mᵀ S M, p = h Mᵀ g̃
        (planefit.zig:676-691); told false where its pattern does not tell it."""
        f = self.fit
        ok, _, g, H = f.keep
        S, gt, good = profiled(H, g)
        W = np.einsum("ki,nkl,lj->nij", self.M, S, self.M) * (self.h * self.h)
        tr = np.trace(W, axis1=1, axis2=2)
        told = f.use & ok & good & (tr > 0)
        p = np.einsum("ki,nk->ni", self.M, gt) * self.h
        Wr = W + (1e-6 * tr)[:, None, None] * np.eye(3)
        dy, g2 = solve_batch(np.where(told[:, None, None], Wr, np.eye(3)), np.where(told[:, None], p, 0.0))
        told &= g2
        W = W + (1e-9 * tr)[:, None, None] * np.eye(3)
        return dy, W, told


def joint_fit(j, which, theta, most):
    """planefit.zig:712-820 — the model's numbers fitted to all the used patterns' mean NCC at once
    (Levenberg–Marquardt), each pattern's orientation profiled out of the step and taken along
    with it; the projective slopes held near zero as the points' fit holds them. Returns the
    rounds; leaves the orientations, the systems and the mean NCC in the fit."""
    f = j.fit
    F = list(PL.FREE[which])
    used = max(f.n_used, 1)
    f.shift = j.sources(theta)
    f.ncc, f.keep = f.eval(f.q, f.shift)
    lam = 1e-3
    it = 0
    while it < most:
        if f.e.cancel:
            raise PlaneError("Cancelled")
        ok, _, g, H = f.keep
        S, gt, good = profiled(H, g)
        live = f.use & ok & good
        _, J = PL.model_at(theta, j.fr, j.row, j.col)
        Jt = j.h * np.einsum("kl,nlm->nkm", j.M, J)  # [n][3][N]
        JF = Jt[live][:, :, F]
        A = np.zeros((PL.N, PL.N))
        v = np.zeros(PL.N)
        A[np.ix_(F, F)] = np.einsum("nkm,nkl,nlo->mo", JF, S[live], JF)
        v[F] = np.einsum("nkm,nk->m", JF, gt[live])
        prior = 0.0
        if which == "projective":
            dy, W, told = j.own_steps()
            chi2 = float(np.einsum("nk,nkl,nl->", dy[told], W[told], dy[told]))
            nt = int(told.sum())
            if nt * 3 > len(F):
                prior = PL.slope_weight(chi2, nt * 3 - len(F))
            for fi in F:
                if fi >= 9:
                    A[fi, fi] += prior
                    v[fi] -= prior * theta[fi]
        Am = A[np.ix_(F, F)].copy()
        tr = float(np.trace(Am)) / len(F)
        dg = np.arange(len(F))
        Am[dg, dg] = Am[dg, dg] * (1 + lam) + 1e-12 * tr + 1e-300
        d = PL.solve(len(F), Am, v[F])
        if d is None:
            break
        trial = np.array(theta, np.float64)
        trial[F] += d
        if which == "projective" and not PL.bounded(trial):
            lam *= 5  # (a step that would take the denominator near zero somewhere: a shorter one)
            if lam > 1e8:
                break
            it += 1
            continue
        s_t = j.sources(trial)
        A3, _ = damped(3, H, g, lam)
        dt = s_t - f.shift
        r = g[:, 3:6] - np.einsum("nik,nk->ni", H[:, 3:6, 0:3], dt)
        dq, gq = solve_batch(A3, r)
        mv = f.use & ok & gq
        q_t = f.q.copy()
        q_t[mv] = _qstep(dq[mv], f.q[mv])
        now, loc = f.eval(q_t, s_t)
        share = prior / (2 * used)
        after = now - share * (trial[9] ** 2 + trial[10] ** 2)
        before = f.ncc - share * (theta[9] ** 2 + theta[10] ** 2)
        if after > before:
            gain = after - before
            theta[:] = trial
            f.q, f.shift, f.keep, f.ncc = q_t, s_t, loc, now
            lam = max(lam / 3, 1e-6)
            if gain < 1e-8:
                it += 1
                break
        else:
            lam *= 5
            if lam > 1e8:
                break
        it += 1
    f.ncc, f.keep = f.eval(f.q, f.shift)
    return it


def pseudo_points(j, theta):
    """planefit.zig:823-840 — what each used pattern says of its own source, one Newton step from
    where the model puts it, with its information as the weight."""
    y, _ = PL.model_at(theta, j.fr, j.row, j.col)
    dy, W, told = j.own_steps()
    pts = PL.Points(j.row, j.col, y, None, np.zeros(len(y), bool))
    pts.y[told] = y[told] + dy[told]
    pts.w[told] = W[told]
    pts.used[:] = told
    return pts


def _drop_far(pts, resid_of, outlier, drop):
    """One round of the outlier rule: the used points further than `outlier` robust standard
    deviations (the median of a three-component Gaussian error's length is 1.538 σ); returns the
    indices dropped (none with fewer than 8 points)."""
    u = np.flatnonzero(pts.used)
    if len(u) < 8:
        return np.zeros(0, np.int64)
    r = resid_of(u)
    dist = np.sqrt(np.maximum(np.einsum("pk,pkl,pl->p", r, pts.w[u], r), 0.0))
    sigma = np.sort(dist)[len(u) // 2] / 1.538
    gone = u[dist > outlier * sigma]
    drop(gone)
    return gone


def joint_plane(j, which, outlier, most):
    """planefit.zig:844-890 — the joint fit of the model from the geometry as it stands, the
    patterns whose pull is far beyond the others' left out and the fit run again (up to 4 times)."""
    f = j.fit
    pc = pc_of(j.R, f.base, j.h, j.h * j.fr.aspect)
    pts = PL.Points(j.row, j.col, pc * np.array([j.fr.aspect, 1.0, 1.0]))
    theta = PL.fit_theta(which, pts, j.fr)
    if theta is None:
        raise PlaneError("TooFewFitPatterns")
    rounds = joint_fit(j, which, theta, most)
    pts = pseudo_points(j, theta)
    if not outlier > 0:
        return rounds, theta, pts
    for _ in range(4):
        def resid(u):
            y, _ = PL.model_at(theta, j.fr, pts.row[u], pts.col[u])
            return pts.y[u] - y

        def drop(gone):
            f.use[gone] = False
            f.n_used -= len(gone)

        if len(_drop_far(pts, resid, outlier, drop)) == 0:
            break
        rounds += joint_fit(j, which, theta, most)
        pts = pseudo_points(j, theta)
    return rounds, theta, pts


def points_plane(f, M, kind, fr, aspect, trust, cols):
    """planefit.zig:904-990 — each pattern's own source point (after settle over six unknowns),
    weighed by how sharply its pattern tells it (plane_weights "information") or alike, and the
    plane through them, the points far from it left out and the plane fitted again (up to 8
    times)."""
    s = f.e.set
    Rm = f.geo0.rotation()
    pc = pc_of(Rm, f.base + f.shift, f.sz[0], f.sz[1])
    at_edge = (np.abs(f.shift) >= trust * (1 - 1e-9)).any(1)
    pts = PL.Points(f.cells // cols, f.cells % cols, pc * np.array([aspect, 1.0, 1.0]), None, f.use & ~at_edge)
    if s["plane_weights"] == "information":
        ok, _, g, H = f.keep
        S, _, good = profiled(H, g)
        W = np.einsum("ki,nkl,lj->nij", M, S, M)
        tr = np.trace(W, axis1=1, axis2=2)
        W = 0.5 * (W + np.transpose(W, (0, 2, 1))) + (1e-9 * tr)[:, None, None] * np.eye(3)
        told = good & (tr > 0)
        weigh = f.use
        pts.used &= ~(weigh & ~told)
        pts.w[weigh & told] = W[weigh & told]
    P = PL.fit(kind, pts, fr)
    if P is None:
        raise PlaneError("TooFewFitPatterns")
    if s["plane_outlier"] > 0:
        for _ in range(8):
            def resid(u):
                return pts.y[u] - PL.at(P, pts.row[u], pts.col[u]) * np.array([aspect, 1.0, 1.0])

            def drop(gone):
                pts.used[gone] = False

            if len(_drop_far(pts, resid, s["plane_outlier"], drop)) == 0:
                break
            P = PL.fit(kind, pts, fr)
            if P is None:
                raise PlaneError("TooFewFitPatterns")
    return P, pts


def _blocks(cells, rows, cols):
    return (cells // cols * BL // rows) * BL + (cells % cols) * BL // cols


def choose(models, pts, cells, rows, cols, fr, aspect, res):
    """planefit.zig:111-168 — each model fitted without one block of the map and asked where that
    block's points stand (mean rᵀ W r); the simplest whose error is within the standard error of
    its difference from the best's (paired over the blocks) is the one the map supports."""
    was = pts.used.copy()
    at = _blocks(cells, rows, cols)
    err = []
    for gb in range(BL * BL):
        inb = was & (at == gb)
        if not inb.any():
            continue
        pts.used = was & (at != gb)
        row, ok = [0.0] * 4, True
        for m in models:
            P = PL.fit_model(m, pts, fr)
            if P is None:
                ok = False
                break
            row[PL.MODELS.index(m)] = float(PL.misfit(P, pts, aspect)[inb].sum() / inb.sum())
        if ok:
            err.append(row)
    pts.used = was
    res["compared"] = True
    if len(err) < 3:
        return models[-1]
    E = np.array(err)
    G = len(err)
    best = models[0]
    for m in models:
        i = PL.MODELS.index(m)
        res["cv"][i] = float(E[:, i].mean())
        if res["cv"][i] < res["cv"][PL.MODELS.index(best)]:
            best = m
    bi = PL.MODELS.index(best)
    for m in models:
        i = PL.MODELS.index(m)
        dlt = E[:, i] - E[:, bi]
        res["cv_se"][i] = float(math.sqrt(((dlt - dlt.mean()) ** 2).sum() / (G - 1) / G))
    for m in models:
        i = PL.MODELS.index(m)
        if res["cv"][i] - res["cv"][bi] <= res["cv_se"][i]:
            return m
    return best


def steps_kept(f, pts, fr, aspect, before, pc):
    """planefit.zig:985-997 — one centre: the scan's steps keep the source's path, and the pattern
    centre at the map's middle is the model's less where the steps put the fit patterns on
    average, each weighed as in the fit."""
    at = pc_of(before.rotation(), f.base, f.sz[0], f.sz[1])
    by = pts.copy()
    by.y = (at - before.pc[None, :]) * np.array([aspect, 1.0, 1.0])
    off = PL.fit_theta("centre", by, fr)
    if off is None:
        raise PlaneError("TooFewFitPatterns")
    return [pc[0] - off[2] / aspect, pc[1] - off[5], pc[2] - off[8]]


def _said(P, geo, e, rows, cols, aspect):
    s = e.set
    return PL.said(P, geo, rows, cols, aspect, float(e.info()[2]), s["scan_x_sign"], s["scan_y_sign"])


def fit_plane(e, compare=False):
    """planefit.zig:896-983 (fitPlane) and 1000-1143 (finishPlane): the plane (or with `compare`
    the simplest model the map supports), its standard errors by blocks, and the geometry taking
    it. The geometry stays as it was when anything fails."""
    s = e.set
    before = e.geo.copy()
    try:
        return _fit_plane(e, compare, before)
    except BaseException:
        e.geo = before
        raise


def _fit_plane(e, compare, before):
    s = e.set
    rows, cols, h_st, w_st = e.info()
    f = Fit(e, s["plane_stride"], s["plane_patterns_max"])
    sz = f.sz
    aspect = sz[1] / sz[0]
    res = {"start_pc": list(map(float, before.pc)), "start_ncc": f.ncc, "n_patterns": f.n_used, "compared": False,
           "cv": [0.0] * 4, "cv_se": [0.0] * 4, "method": s["plane_method"]}
    trust = s["plane_trust"] * sz[0]
    Rm = before.rotation()
    M = np.array([[-Rm[k, 1], -Rm[k, 0], Rm[k, 2]] for k in range(3)])
    kind = "projective" if s["plane_kind"] == "projective" else "affine"
    fr = PL.Frame(rows, cols, aspect)
    full = kind
    j = Joint(f, fr, Rm, sz[0], cols)
    if s["plane_method"] == "joint":
        f.settle(3, 0.0, s["plane_iters"])
        res["start_ncc"] = f.ncc
        res["iterations"], theta, pts = joint_plane(j, full, s["plane_outlier"], s["plane_iters"])
        P = PL.to_plane(full, theta, fr)
    else:
        res["iterations"] = f.settle(6, trust, s["plane_iters"])
        P, pts = points_plane(f, M, kind, fr, aspect, trust, cols)
    if P is None:
        raise PlaneError("TooFewFitPatterns")
    res["ncc"] = f.ncc
    model = choose(["centre", "line", full], pts, f.cells, rows, cols, fr, aspect, res) if compare else full
    res["model"] = model
    if model != full:
        if s["plane_method"] == "joint":
            theta = PL.fit_theta(model, pts, fr)
            if theta is None:
                raise PlaneError("TooFewFitPatterns")
            res["iterations"] += joint_fit(j, model, theta, s["plane_iters"])
            res["ncc"] = f.ncc
            P = PL.to_plane(model, theta, fr)
        else:
            P = PL.fit_model(model, pts, fr)
        if P is None:
            raise PlaneError("TooFewFitPatterns")
    said = _said(P, before, e, rows, cols, aspect)
    if model == "centre":
        said["pc"] = steps_kept(f, pts, fr, aspect, before, said["pc"])
    return _finish(e, f, res, before, P, model, kind, pts, fr, aspect, said)


def _finish(e, f, res, before, P, model, kind, pts, fr, aspect, said):
    """planefit.zig:1000-1143 — each number's standard error by blocks, the geometry taking the
    model, the points kept, and the fit patterns' orientations in the sample frame now in use."""
    s = e.set
    rows, cols = e.info()[:2]
    # the standard errors: the plane fitted again without one block of the map at a time
    was = pts.used.copy()
    at = _blocks(f.cells, rows, cols)
    vals = []
    for gb in range(BL * BL):
        if not (was & (at == gb)).any():
            continue
        pts.used = was & (at != gb)
        Pg = PL.fit_model(model, pts, fr)
        if Pg is None:
            continue
        w = _said(Pg, before, e, rows, cols, aspect)
        vals.append(list(w["rot"]) + list(w["step"]) + [w["skew"]] + list(w["pc"]))
    pts.used = was
    se = np.zeros(9)
    if len(vals) >= 2:
        V = np.array(vals)
        G = len(vals)
        se = np.sqrt(((V - V.mean(0)) ** 2).sum(0) * (G - 1) / G)
    res["blocks"] = len(vals)
    res["kind"] = 0 if model == "centre" else (2 if model == "projective" else 1)
    res["frame"] = s["plane_frame"] == "follow" and model != "centre"
    res["plane"] = np.asarray(P, np.float64).reshape(4, 3)
    res["pc"], res["said"] = list(said["pc"]), said
    res["se"] = se
    g = before.copy()
    g.pc = np.array(said["pc"], np.float64)
    if model != "centre":
        g.plane_kind = res["kind"]
        g.plane = np.asarray(P, np.float64).copy()
        if s["plane_frame"] == "follow":
            g.rot = np.array(said["rot"], np.float64)
    e.geo = g
    res["rot"] = list(map(float, g.rot))
    # the points, for the view
    R_before = before.rotation()
    if model == "centre":
        fitpc = pc_of(R_before, f.base, f.sz[0], f.sz[1]) - before.pc[None, :] + np.array(said["pc"])[None, :]
    else:
        fitpc = PL.at(P, pts.row, pts.col)
    own = pts.y / np.array([aspect, 1.0, 1.0])
    ncc = np.where(f.use, f.keep[1], f.seed_ncc)
    e.plane_points = {"cells": f.cells.astype(np.uint64), "pc": own, "fit": fitpc, "ncc": ncc.astype(np.float64),
                      "used": pts.used.copy()}
    u = pts.used
    res["n_used"] = int(u.sum())
    res["rmsd"] = list(np.sqrt(((own[u] - fitpc[u]) ** 2).sum(0) / max(u.sum(), 1)))
    # the fit patterns' orientations in the sample frame as the geometry now has it: a rotation of
    # the detector from E to E' turns that frame, q' = q h(E) h(E')⁻¹, h = Exp(R0 log E)
    R0 = before.nominal()
    frame_rot = R.qmul(R.exp_map(R0 @ before.rot), R.qconj(R.exp_map(R0 @ g.rot)))
    quats = np.empty((f.n, 4), np.float32)
    turned = R.qmul(f.q, frame_rot[None, :])
    for p in np.unique(f.phase):
        sel = f.phase == p
        quats[sel] = R.to_fz(turned[sel], e.phases[int(p)].master.rotations())
    e.fit = {"cells": f.cells, "quats": quats, "phase": f.phase.copy(),
             "ncc": np.where(f.use, f.keep[1], f.seed_ncc).astype(np.float32)}
    deg = 180.0 / math.pi
    if res["compared"]:
        e.log("the source over the scan, each model asked where a block of the map stands from the others (mean "
              f"misfit a point): one centre {res['cv'][0]:.3f}, a tilt line {res['cv'][1]:.3f}, the {kind} plane "
              f"{res['cv'][PL.MODELS.index(kind)]:.3f}; the map supports {model}")
    e.log(f"plane of source points ({model}): {res['n_used']} of {res['n_patterns']} fit patterns used; about it they "
          f"scatter by {res['rmsd'][0]:.5f} {res['rmsd'][1]:.5f} {res['rmsd'][2]:.5f} (PCx, PCy, PCz); mean NCC "
          f"{res['ncc']:.4f} with each pattern at its own best (was {res['start_ncc']:.4f})")
    e.log(f"plane: source at the map's middle {said['pc'][0]:.5f} {said['pc'][1]:.5f} {said['pc'][2]:.5f}; tilt "
          f"{said['rot'][1] * deg:.2f}° ± {se[1] * deg:.2f}°")
    return res


def auto(e):
    """planefit.zig:1149-1157 — the automatic fit from the geometry as it was given: the vote for
    the pattern centre, then the plane of source points with the simplest model the map supports."""
    from . import pcfit

    before = e.geo.copy()
    try:
        e.geo = e.geo_given.copy()
        pcfit.run(e)
        if e.cancel:
            raise PlaneError("Cancelled")
        return _fit_plane(e, True, e.geo.copy())
    except BaseException:
        e.geo = before
        raise
