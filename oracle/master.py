"""Master patterns: loading, symmetry, harmonics and weight tables (oracle restatement of
zebsdsolve `src/master.zig`)."""
import json
import math

import numpy as np

from . import lambert, rot, sh, sym


class Master:
    """master.zig:23-154 — two side × side Lambert sheets [north | south], normalized."""

    def __init__(self, side, raw, ops, point_group=0):
        self.side = int(side)
        self.raw = np.asarray(raw, dtype=np.float32).reshape(-1)
        self.ops = [np.asarray(o, dtype=np.float64).reshape(3, 3) for o in ops]
        self.point_group = point_group
        self.laue = sym.laue_of_point_group(point_group) or _laue_from_operators(self.ops)
        self.setting = sym.Setting()

    def rotations(self):
        return self.setting.rotations()

    def at(self, sheets, v):
        """master.zig:150-153 — bilinear intensity of `sheets` in crystal direction(s) v."""
        v = np.asarray(v, dtype=np.float64)
        uv = lambert.sphere_to_square(v)
        plane = self.side * self.side
        sheets = np.asarray(sheets).reshape(-1)
        north = lambert.sample(sheets[:plane], self.side, uv[..., 0], uv[..., 1])
        south = lambert.sample(sheets[plane:], self.side, uv[..., 0], uv[..., 1])
        return np.where(v[..., 2] >= 0, north, south)

    def measure_symmetry(self, seed=12345):
        """master.zig:77-138 — keep the candidate operators under which the raw master correlates
        with itself above 0.97 over 1500 random directions.  (The reference draws its directions
        from Zig's DefaultPrng; this restatement uses NumPy's generator: the kept set only differs
        where a correlation sits at the 0.97 threshold.)"""
        rng = np.random.default_rng(seed)
        n = 1500
        z = 2 * rng.random(n) - 1
        phi = 2 * math.pi * rng.random(n)
        st = np.sqrt(np.maximum(0.0, 1 - z * z))
        dirs = np.stack([st * np.cos(phi), st * np.sin(phi), z], -1)
        base = self.at(self.raw, dirs)
        mean = base.mean()
        var0 = ((base - mean) ** 2).sum()
        cands = list(self.ops)
        for q in sym.operators(self.laue):
            R = rot.to_mat(q)
            cands.append(R.copy())
            cands.append(-R)
        found = []
        for g in cands:
            if any(np.abs(f - g).sum() < 1e-6 for f in found):
                continue
            v = self.at(self.raw, dirs @ g.T)
            v = v - v.mean()
            cov = (v * (base - mean)).sum()
            var1 = (v * v).sum()
            if cov / math.sqrt(max(var0 * var1, 1e-300)) > 0.97:
                found.append(g)
        self.ops = found
        s = sym.setting_of(found)
        self.setting = s if s is not None else sym.Setting()
        self.laue = self.setting.laue


def normalize(sheets):
    """master.zig:157-166 — zero mean, unit variance over both sheets (f64 statistics)."""
    s = np.asarray(sheets, dtype=np.float64)
    mean = s.mean()
    sd = math.sqrt(((s - mean) ** 2).mean())
    k = 1 / sd if sd > 0 else 1.0
    return ((s - mean) * k).astype(np.float32)


def _laue_from_operators(ops):
    """master.zig:531-568"""
    seen = []
    has4 = has3z = has3d = False
    for g0 in ops:
        g = g0 if np.linalg.det(g0) >= 0 else -g0
        if any(np.abs(s - g).sum() < 1e-6 for s in seen):
            continue
        seen.append(g)
        tr = g[0, 0] + g[1, 1] + g[2, 2]
        if abs(tr - 1) < 1e-6:
            has4 = True
        if abs(tr) < 1e-6:
            if abs(g[2, 2] - 1) < 1e-6:
                has3z = True
            else:
                has3d = True
    n = len(seen)
    six = any(abs(g[0, 0] + g[1, 1] + g[2, 2] - 2) < 1e-6 for g in seen)
    return {1: "c1", 2: "c2", 3: "c3", 4: "c4" if has4 else "d2",
            6: ("c6" if six else "d3") if (has3z and not has4) else "d3",
            8: "d4", 12: "t" if has3d else "d6", 24: "o"}.get(n, "c1")


def _sample_stored(sheet, has, side, x, y):
    """master.zig:489-526 — bilinear over stored pixels only (weights renormalized)."""
    last = float(side - 1)
    fj = min(max((x + 1) * 0.5 * last, 0.0), last)
    fi = min(max((y + 1) * 0.5 * last, 0.0), last)
    c0 = int(math.floor(fj))
    r0 = int(math.floor(fi))
    c1 = min(c0 + 1, side - 1)
    r1 = min(r0 + 1, side - 1)
    tj = fj - c0
    ti = fi - r0
    idx = [r0 * side + c0, r0 * side + c1, r1 * side + c0, r1 * side + c1]
    wts = [(1 - ti) * (1 - tj), (1 - ti) * tj, ti * (1 - tj), ti * tj]
    acc = 0.0
    wsum = 0.0
    for i, w in zip(idx, wts):
        if has[i]:
            acc += w * sheet[i]
            wsum += w
    if wsum > 1e-9:
        return acc / wsum
    ci = int(round(fi))
    cj = int(round(fj))
    for r in range(1, 8):
        for di in range(-r, r + 1):
            for dj in range(-r, r + 1):
                ii, jj = ci + di, cj + dj
                if ii < 0 or jj < 0 or ii >= side or jj >= side:
                    continue
                if has[ii * side + jj]:
                    return sheet[ii * side + jj]
    return 0.0


def from_sector(vals, kij, hw, ops, normals, point_group=0):
    """master.zig:384-485 (without the grid-symmetry shortcut, which master.zig:755-773 shows
    gives the same sheets) — expand a fundamental sector to both hemispheres."""
    side = 2 * hw + 1
    plane = side * side
    sec = np.zeros(2 * plane, np.float32)
    has = np.zeros(2 * plane, bool)
    kij = np.asarray(kij, np.int64).reshape(-1, 3)
    vals = np.asarray(vals, np.float64).reshape(-1)
    ix = kij[:, 0] + hw
    iy = kij[:, 1] + hw
    ok = (ix >= 0) & (iy >= 0) & (ix < side) & (iy < side)
    south = kij[:, 2] <= 0
    needs_south = bool((south & ok).any())
    at = np.where(south, plane, 0) + iy * side + ix
    sec[at[ok]] = vals[ok]
    has[at[ok]] = True
    ops = [np.asarray(o, dtype=np.float64).reshape(3, 3) for o in ops]
    normals = np.asarray(normals, dtype=np.float64).reshape(-1, 3)
    eps = 1.0 / max(hw, 1)
    last = float(side - 1)
    rr, cc = np.meshgrid(np.arange(side), np.arange(side), indexing="ij")
    xs = np.tile((2 * cc / last - 1).ravel(), 2)
    ys = np.tile((2 * rr / last - 1).ravel(), 2)
    hemi = np.repeat([False, True], plane)
    d = lambert.square_to_sphere(xs, ys, hemi)
    rep = d.copy()
    best = np.full(d.shape[0], -np.inf)
    best_in = np.zeros(d.shape[0], bool)
    for g in ops:
        t = d @ g.T
        margin = (t @ normals.T).min(1) if len(normals) else np.full(d.shape[0], np.inf)
        inside = margin >= -eps
        take = (inside & ~best_in) | ((inside == best_in) & (margin > best))
        best = np.where(take, margin, best)
        best_in = np.where(take, inside, best_in)
        rep = np.where(take[:, None], t, rep)
        if len(normals) == 0:
            break
    use_south = (rep[:, 2] < 0) & needs_south
    uv = lambert.sphere_to_square(rep)
    sheets = np.zeros(2 * plane, np.float32)
    for hs in (False, True):
        sel = np.nonzero(use_south == hs)[0]
        off = plane if hs else 0
        sh_ = sec[off:off + plane]
        hs_ = has[off:off + plane]
        fj = np.clip((uv[sel, 0] + 1) * 0.5 * last, 0.0, last)
        fi = np.clip((uv[sel, 1] + 1) * 0.5 * last, 0.0, last)
        c0 = np.floor(fj).astype(np.int64)
        r0 = np.floor(fi).astype(np.int64)
        c1 = np.minimum(c0 + 1, side - 1)
        r1 = np.minimum(r0 + 1, side - 1)
        tj = fj - c0
        ti = fi - r0
        idx = [r0 * side + c0, r0 * side + c1, r1 * side + c0, r1 * side + c1]
        wts = [(1 - ti) * (1 - tj), (1 - ti) * tj, ti * (1 - tj), ti * tj]
        acc = np.zeros(sel.size)
        wsum = np.zeros(sel.size)
        for i, w in zip(idx, wts):
            hv = hs_[i]
            acc += np.where(hv, w * sh_[i], 0.0)
            wsum += np.where(hv, w, 0.0)
        val = np.where(wsum > 1e-9, acc / np.where(wsum > 1e-9, wsum, 1.0), 0.0)
        for k in np.nonzero(wsum <= 1e-9)[0]:
            val[k] = _sample_stored(sh_, hs_, side, uv[sel[k], 0], uv[sel[k], 1])
        sheets[sel] = val
    return Master(side, normalize(sheets), ops, point_group)


def load_ebsdsim(path):
    """master.zig:276-335 — an ebsdsim .npz (fundamental sector + point-group operators)."""
    z = np.load(path)
    fs = z["fundamental_sector"] if "fundamental_sector" in z.files else z["integrated_fundamental_sector"]
    kij = np.asarray(z["fundamental_kij"]).astype(np.int64)
    n_k = kij.shape[0]
    if fs.ndim == 3:
        vals = fs.reshape(-1)[:n_k].astype(np.float64)
    else:
        n_sites = fs.shape[1] if fs.ndim == 2 else 1
        vals = fs.reshape(n_k, n_sites).astype(np.float64).mean(1)
    hw = int(np.max(np.abs(kij[:, :2]))) if n_k else 0
    meta = {}
    if "meta_json" in z.files:
        try:
            meta = json.loads(bytes(np.asarray(z["meta_json"], np.uint8)).decode())
        except Exception:
            meta = {}
    if "halfw" in meta:
        hw = int(meta["halfw"])
    ops = np.asarray(z["pg_operators"], np.float64).reshape(-1, 3, 3)
    nrm = np.asarray(z["fs_normals"], np.float64)
    normals = nrm.reshape(-1, 3) if nrm.ndim == 2 else np.zeros((0, 3))
    pg = int(meta.get("pg_num", 0) or 0)
    m = from_sector(vals, kij, hw, ops, normals, pg)
    m.measure_symmetry()
    return m


class Harmonics:
    """master.zig:665-711 — f and f² coefficients of the band-limited zero-mean master."""

    def __init__(self, master, sheets, L):
        nt = max(4 * L, 512)
        grid = sh.Grid(L, nt, 2 * nt)
        dirs = grid.directions().reshape(-1, 3)
        samples = master.at(sheets, dirs)
        f = grid.analyze(samples)
        f[0] = 0
        self.rules = sh.Rules.detect(L, f, 1e-5)
        ms, ls = sh.pair_table(L)
        for p in range(len(f)):
            if not self.rules.allows(int(ls[p]), int(ms[p])):
                f[p] = 0
        g2 = sh.Grid(L, 2 * L, 4 * L)
        s2 = g2.synthesize(f)
        self.f = f
        self.f2 = g2.analyze(s2 * s2)
        self.L = L


def fold_of(rules):
    """master.zig:715-721"""
    return {4: 4, 2: 2, 6: 2}.get(rules.n_fold, 1)


def weights(L, coef, tab, fold):
    """master.zig:727-753 — W[μ + μmax, l, k] = i^{−m} f_{l,m} d^l_{k,m}(π/2), m = fold·μ (complex)."""
    mu_max = (L - 1) // fold
    mc = 2 * mu_max + 1
    out = np.zeros((mc, L, L), np.complex128)
    for mi in range(mc):
        mu = mi - mu_max
        m = mu * fold
        ph = sh.ipow(-m)
        for k in range(L):
            for l in range(max(k, abs(m)), L):
                c = sh.signed_coef(L, coef, l, m)
                d = sh.d_half_pi(tab, l, k, m)
                out[mi, l, k] = c * ph * d
    return out
