"""Pattern-centre vote: oracle restatement of zebsdsolve `src/pcfit.zig` (test infrastructure —
what zebsdsolve_b200.pcfit is tested against, never part of the product path).

Scalar Python loops over the vote's host arithmetic, in the reference's order, so that the
product's vectorized version can be held to the same numbers:

* fit_cells (pcfit.zig:63-87), fit_cells_every (91-113): the fit patterns' lattices;
* axis (115-121), valid_depth (125-127), vertex (130-134);
* max_of (177-188), peak_at (192-206), splat (210-236), consensus (244-318);
* search (run, 319-574): the levels, border walks and narrowing over a score function that
  returns every fit pattern's score under each candidate;
* candidate_score: one pattern's score under one candidate in FP64 — the candidate's window
  denominators (spherical.zig:448-464) and the largest normalized correlation (pcfit.zig:430-450).
"""
import math

import numpy as np

from . import spherical as osp

MAX_WALK = 4  # pcfit.zig:43


class NoPcSupport(Exception):
    pass


class NoPcCandidates(Exception):
    pass


class SearchTooLarge(Exception):
    pass


def fit_cells(region, cols, grid):
    """pcfit.zig:63-87 — grid × grid cells at the centres of their shares of the region's rectangle."""
    c_first, c_last = int(region[0]), int(region[-1])
    x0, y0 = c_first % cols, c_first // cols
    w = c_last % cols - x0 + 1
    h = c_last // cols - y0 + 1
    gy, gx = min(grid, h), min(grid, w)
    out = []
    for r in range(gy):
        for c in range(gx):
            row = y0 + (2 * r + 1) * h // (2 * gy)
            col = x0 + (2 * c + 1) * w // (2 * gx)
            out.append(row * cols + col)
    return np.array(out, np.int64)


def fit_cells_every(region, cols, stride):
    """pcfit.zig:91-113 — every stride-th cell along rows and columns, the lattice centred."""
    c_first, c_last = int(region[0]), int(region[-1])
    x0, y0 = c_first % cols, c_first // cols
    w = c_last % cols - x0 + 1
    h = c_last // cols - y0 + 1
    st = max(stride, 1)
    gy, gx = (h + st - 1) // st, (w + st - 1) // st
    oy = (h - 1 - (gy - 1) * st) // 2
    ox = (w - 1 - (gx - 1) * st) // 2
    return np.array([(y0 + oy + r * st) * cols + x0 + ox + c * st for r in range(gy) for c in range(gx)], np.int64)


def axis(centre, span, steps):
    """pcfit.zig:115-121"""
    return [centre if steps == 1 else centre - span + 2 * span * k / (steps - 1) for k in range(steps)]


def valid_depth(z, zmin):
    """pcfit.zig:125-127"""
    return math.isfinite(z) and z > 0 and z >= zmin


def vertex(lo, mid, hi):
    """pcfit.zig:130-134"""
    den = lo - 2 * mid + hi
    if den >= -1e-15:
        return 0.0
    return min(max(0.5 * (lo - hi) / den, -0.5), 0.5)


def max_of(m, lo, hi):
    """pcfit.zig:177-188"""
    best, top = None, 0.0
    for i in range(lo, hi):
        v = float(m[i])
        if math.isfinite(v) and v > top:
            best, top = i, v
    if best is None:
        raise NoPcSupport
    return best


def peak_at(m, lo, hi, n, best):
    """pcfit.zig:192-206"""
    at = (best % n[0], (best // n[0]) % n[1], best // (n[0] * n[1]))
    strides = (1, n[0], n[0] * n[1])
    out = [float(a) for a in at]
    for a in range(3):
        if n[a] < 3 or at[a] == 0 or at[a] == n[a] - 1:
            continue
        lo_i, hi_i = best - strides[a], best + strides[a]
        if lo_i >= lo and hi_i < hi:
            out[a] += vertex(float(m[lo_i]), float(m[best]), float(m[hi_i]))
    return out


def splat(ballots, n, sigma):
    """pcfit.zig:210-236 — float32 accumulation, ballot by ballot."""
    out = np.zeros(n[0] * n[1] * n[2], np.float32)
    r = [int(min(math.ceil(3 * sigma[a]), n[a] - 1)) for a in range(3)]
    inv = [1.0 / (2 * sigma[a] * sigma[a]) for a in range(3)]
    for at, w in ballots:
        c = [int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5)) for v in at]
        for z in range(max(c[2] - r[2], 0), min(c[2] + r[2], n[2] - 1) + 1):
            for y in range(max(c[1] - r[1], 0), min(c[1] + r[1], n[1] - 1) + 1):
                for x in range(max(c[0] - r[0], 0), min(c[0] + r[0], n[0] - 1) + 1):
                    d = (float(x - c[0]), float(y - c[1]), float(z - c[2]))
                    e = d[0] * d[0] * inv[0] + d[1] * d[1] * inv[1] + d[2] * d[2] * inv[2]
                    i = x + n[0] * (y + n[1] * z)
                    out[i] = np.float32(out[i] + np.float32(w * math.exp(-e)))
    return out


def consensus(s, pat_scores, n_pat, n, step, lo, hi):
    """pcfit.zig:244-318 — returns (peak in candidate steps, winner, first density, (ballots, inliers))."""
    n_c = n[0] * n[1] * n[2]
    k = min(s["pc_top_k"], n_c)
    sigma = [max(s["pc_kde_sigma"] / step[a], 0.75) if step[a] > 0 else 1.0 for a in range(3)]
    half = s["pc_nms"] // 2 if s["pc_nms"] > 1 else 0
    ballots = []
    for b in range(n_pat):
        sc = [float(v) for v in pat_scores[b * n_c:(b + 1) * n_c]]
        top = max(sc)
        order = sorted(range(n_c), key=lambda i: -sc[i])  # stable: ties keep the lower index first
        cast = 0
        for c in order:
            if cast == k or not (sc[c] >= s["pc_gate"] * top) or not (sc[c] > 0):
                break
            at = (c % n[0], (c // n[0]) % n[1], c // (n[0] * n[1]))
            if half > 0:
                is_max = True
                for z in range(max(at[2] - half, 0), min(at[2] + half, n[2] - 1) + 1):
                    for y in range(max(at[1] - half, 0), min(at[1] + half, n[1] - 1) + 1):
                        for x in range(max(at[0] - half, 0), min(at[0] + half, n[0] - 1) + 1):
                            if sc[x + n[0] * (y + n[1] * z)] > sc[c]:
                                is_max = False
                if not is_max:
                    continue
            ballots.append(((float(at[0]), float(at[1]), float(at[2])), sc[c]))
            cast += 1
    if not ballots:
        raise NoPcSupport
    density = splat(ballots, n, sigma)
    best = max_of(density, lo, hi)
    mode = peak_at(density, lo, hi, n, best)
    r2 = s["pc_inlier_radius"] * s["pc_inlier_radius"]

    def near(b, p):
        d = [(b[0][a] - p[a]) * step[a] for a in range(3)]
        return d[0] * d[0] + d[1] * d[1] + d[2] * d[2] <= r2

    acc = [0.0, 0.0, 0.0, 0.0]
    for b in ballots:
        if near(b, mode):
            for a in range(3):
                acc[a] += b[1] * b[0][a]
            acc[3] += b[1]
    pk = [acc[a] / acc[3] for a in range(3)] if acc[3] > 0 else mode
    kept = [b for b in ballots if near(b, pk)]
    if not kept:
        raise NoPcSupport
    inl = splat(kept, n, sigma)
    winner = max_of(inl, lo, hi)
    return peak_at(inl, lo, hi, n, winner), winner, density, (len(ballots), len(kept))


def search(s, pc0, n_pat, score):
    """pcfit.zig:319-574 over score(candidates [k][3], pc units) → the fit patterns' scores under
    each candidate ([n_pat][k], float32, the phase of each pattern chosen; non-finite ones 0).
    Returns the result fields and every level's record."""
    steps = (s["pc_steps"], s["pc_steps"], s["pc_steps_z"])
    span = [s["pc_span"], s["pc_span"], s["pc_span_z"]]
    n_c = steps[0] * steps[1] * steps[2]
    if n_c * n_pat > 4 << 20:
        raise SearchTooLarge
    xy = steps[0] * steps[1]
    pc = [float(v) for v in pc0]
    res = {"start": list(pc), "n_patterns": n_pat, "n_candidates": 0, "levels": s["pc_levels"], "start_score": 0.0}
    history = []
    level, walked, best_c = 0, 0, 0
    while level < s["pc_levels"]:
        axes = [axis(pc[a], span[a], steps[a]) for a in range(3)]
        if not all(math.isfinite(v) for v in axes[0] + axes[1]):
            raise NoPcCandidates
        z0 = 0
        while z0 < len(axes[2]) and not valid_depth(axes[2][z0], s["pc_z_min"]):
            z0 += 1
        if z0 == len(axes[2]):
            raise NoPcCandidates
        z1 = z0 + 1
        while z1 < len(axes[2]) and valid_depth(axes[2][z1], s["pc_z_min"]):
            z1 += 1
        lo, hi = z0 * xy, z1 * xy
        cands = [(axes[0][c % steps[0]], axes[1][(c // steps[0]) % steps[1]], axes[2][c // xy]) for c in range(lo, hi)]
        got = np.asarray(score(np.array(cands, np.float64)), np.float32)
        pat_scores = np.zeros(n_pat * n_c, np.float32)
        for b in range(n_pat):
            for j, c in enumerate(range(lo, hi)):
                v = got[b, j]
                pat_scores[b * n_c + c] = v if math.isfinite(float(v)) else 0.0
        scores = np.zeros(n_c, np.float32)
        for c in range(lo, hi):
            acc = 0.0
            for b in range(n_pat):
                acc += float(pat_scores[b * n_c + c])
            scores[c] = np.float32(acc / n_pat)
        best_c = max_of(scores, lo, hi)
        res["n_candidates"] += hi - lo
        pat_best, pat_ncc = [], []
        for b in range(n_pat):
            top, at_c = -math.inf, lo
            for c in range(lo, hi):
                v = float(pat_scores[b * n_c + c])
                if v > top:
                    top, at_c = v, c
            pat_best.append(at_c)
            pat_ncc.append(top)
        lvl = {"axes": axes, "scores": scores, "pat_scores": pat_scores, "pat_best": pat_best, "pat_ncc": pat_ncc,
               "density": None, "ballots": 0, "inliers": 0, "walked": 0}
        history.append(lvl)
        voted = None
        if s["pc_vote"] == "ballots":
            step = [axes[a][1] - axes[a][0] if steps[a] > 1 else 0.0 for a in range(3)]
            voted, best_c, lvl["density"], (lvl["ballots"], lvl["inliers"]) = consensus(
                s, pat_scores, n_pat, steps, step, lo, hi)
        lvl["best"] = best_c
        bi = (best_c % steps[0], (best_c // steps[0]) % steps[1], best_c // xy)
        if voted is not None:
            peak = voted
        elif level + 1 == s["pc_levels"]:
            peak = peak_at(scores, lo, hi, steps, best_c)
        else:
            peak = [float(v) for v in bi]
        lvl["peak"] = peak
        if level == 0 and walked == 0:
            mid = (steps[0] // 2) + steps[0] * ((steps[1] // 2) + steps[1] * (steps[2] // 2))
            res["start_score"] = float(scores[mid])
        for a in range(3):
            st = axes[a][1] - axes[a][0] if steps[a] > 1 else 0.0
            pc[a] = axes[a][bi[a]] + (peak[a] - bi[a]) * st
        if not (math.isfinite(pc[0]) and math.isfinite(pc[1]) and valid_depth(pc[2], s["pc_z_min"])):
            raise NoPcCandidates
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
    res["best"] = best_c
    return res, history


def candidate_score(tables, ph, harmonics, pattern, t_candidate, offset, frame, mask, shape):
    """One pattern's score under one candidate (pcfit.zig:430-450): its coefficients sampled at
    the candidate's position less the pattern's beam offset, correlated with the master and
    normalized by the candidate window's denominators; the volume's largest value."""
    walm, wst = osp.coefficients(tables, None, t_candidate, frame, mask, flags=osp.FLAG_WINDOW, shape=shape)
    rden = osp.window_denominators(tables, ph, walm, wst[0])
    g, _ = osp.coefficients(tables, pattern, np.asarray(t_candidate) - np.asarray(offset), frame, mask)
    vol = osp.correlation_volume(tables, ph, harmonics.f, g) * rden
    return osp.peak(tables, ph, vol)
