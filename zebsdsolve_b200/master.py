"""A candidate phase's master pattern: loading (ebsdsim .npz), its symmetry, and the tables the
device kernels read (zebsdsolve src/master.zig).

The master is two side × side equal-area Lambert sheets [north | south] normalized to zero mean
and unit variance (master.zig:7-10, 157-166).  Everything per-pattern runs on the device; the
per-phase tables (harmonics of the master and of its square, the weight table, the correlation
table) are built once per bandwidth in FP64 on the device.
"""
import io
import json
import math
from pathlib import Path

import numpy as np

from . import rotations as R


class MasterError(ValueError):
    pass


def square_to_sphere(x, y, south):
    """lambert.zig:9-25 in float64, vectorised."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    sc = math.sqrt(math.pi / 2)
    xa, ya = np.abs(x) * sc, np.abs(y) * sc
    swap = xa >= ya
    xn, yn = np.where(swap, xa, ya), np.where(swap, ya, xa)
    r = (2 * xn / math.pi) * np.sqrt(np.maximum(math.pi - xn * xn, 0.0))
    ang = math.pi * yn / (4 * np.where(xn == 0, 1.0, xn))
    xh, yh = r * np.cos(ang), r * np.sin(ang)
    hx = np.where(swap, xh, yh) * np.where(x < 0, -1.0, 1.0)
    hy = np.where(swap, yh, xh) * np.where(y < 0, -1.0, 1.0)
    z = 1 - 2 * xn * xn / math.pi
    v = np.stack([hx, hy, np.where(south, -z, z)], -1)
    v /= np.linalg.norm(v, axis=-1, keepdims=True)
    pole = np.stack([np.zeros_like(z), np.zeros_like(z), np.where(south, -1.0, 1.0) + np.zeros_like(z)], -1)
    return np.where((xn == 0)[..., None], pole, v)


def sphere_to_square(v):
    """lambert.zig:28-45 in float64, vectorised."""
    v = np.asarray(v, np.float64)
    kz = np.abs(v[..., 2])
    xn = np.sqrt(np.maximum(math.pi * (1 - kz) / 2, 0.0))
    ax, ay = np.abs(v[..., 0]), np.abs(v[..., 1])
    sc = math.sqrt(math.pi / 2)
    big = ax >= ay
    u = np.where(big, xn, (4 * xn / math.pi) * np.arctan2(ax, np.maximum(ay, 1e-300)))
    w = np.where(big, (4 * xn / math.pi) * np.arctan2(ay, np.maximum(ax, 1e-300)), xn)
    out = np.stack([u / sc * np.where(v[..., 0] < 0, -1.0, 1.0), w / sc * np.where(v[..., 1] < 0, -1.0, 1.0)], -1)
    return np.where((kz >= 1 - 1e-14)[..., None], 0.0, out)


def bilinear(sheet, side, x, y):
    """lambert.zig:48-64"""
    last = side - 1.0
    fj = np.clip((x + 1) * 0.5 * last, 0.0, last)
    fi = np.clip((y + 1) * 0.5 * last, 0.0, last)
    c0 = np.floor(fj).astype(np.int64)
    r0 = np.floor(fi).astype(np.int64)
    c1 = np.minimum(c0 + 1, side - 1)
    r1 = np.minimum(r0 + 1, side - 1)
    tj, ti = fj - c0, fi - r0
    s = np.asarray(sheet, np.float64).reshape(-1)
    return (s[r0 * side + c0] * (1 - tj) + s[r0 * side + c1] * tj) * (1 - ti) + \
        (s[r1 * side + c0] * (1 - tj) + s[r1 * side + c1] * tj) * ti


class Master:
    """master.zig:23-154"""

    def __init__(self, name, side, sheets, ops, point_group=0, space_group=0, voltage_kv=0.0, source="ebsdsim"):
        self.name = name
        self.side = int(side)
        self.raw = np.ascontiguousarray(sheets, np.float32).reshape(-1)
        if self.raw.size != 2 * self.side * self.side:
            raise MasterError("master sheets do not match their side")
        self.ops = [np.asarray(o, np.float64).reshape(3, 3) for o in ops]
        self.lattice = None  # a, b, c (Å), α, β, γ (degrees) when the file says
        self.point_group = int(point_group)
        self.space_group = int(space_group)
        self.voltage_kv = float(voltage_kv)
        self.source = source
        self.laue = R.laue_of_point_group(self.point_group) or _laue_of_operators(self.ops)
        self.setting = R.Setting()

    def rotations(self):
        """The rotations that leave the master unchanged: what orientations are reduced by."""
        return self.setting.rots

    def at(self, v, sheets=None):
        """The master (bilinear) in crystal directions v [..., 3]."""
        s = self.raw if sheets is None else np.asarray(sheets).reshape(-1)
        plane = self.side * self.side
        uv = sphere_to_square(v)
        n = bilinear(s[:plane], self.side, uv[..., 0], uv[..., 1])
        so = bilinear(s[plane:], self.side, uv[..., 0], uv[..., 1])
        return np.where(np.asarray(v)[..., 2] >= 0, n, so)

    def measure_symmetry(self, seed=12345):
        """master.zig:77-138 — the candidate operators (the file's, and the Laue class's rotations
        with and without the inversion) under which the master correlates with itself above 0.97
        over 1500 random directions; then its setting."""
        rng = np.random.default_rng(seed)
        n = 1500
        z = 2 * rng.random(n) - 1
        phi = 2 * math.pi * rng.random(n)
        st = np.sqrt(np.maximum(0.0, 1 - z * z))
        dirs = np.stack([st * np.cos(phi), st * np.sin(phi), z], -1)
        base = self.at(dirs)
        b0 = base - base.mean()
        var0 = (b0 * b0).sum()
        cands = list(self.ops)
        for q in R.group(self.laue):
            m = R.to_matrix(q)
            cands += [m, -m]
        found = []
        for g in cands:
            if any(np.abs(f - g).sum() < 1e-6 for f in found):
                continue
            v = self.at(dirs @ g.T)
            v = v - v.mean()
            if (v * b0).sum() / math.sqrt(max(var0 * (v * v).sum(), 1e-300)) > 0.97:
                found.append(g)
        self.ops = found
        s = R.setting_of(found)
        self.setting = s if s is not None else R.Setting()
        self.laue = self.setting.laue


def normalize(sheets):
    """Zero mean and unit variance over both sheets, statistics in float64 (master.zig:157-166)."""
    s = np.asarray(sheets, np.float64)
    mean = s.mean()
    sd = math.sqrt(((s - mean) ** 2).mean())
    return ((s - mean) * (1.0 / sd if sd > 0 else 1.0)).astype(np.float32)


def _laue_of_operators(ops):
    """master.zig:531-568 — the Laue class from the operators' proper parts."""
    seen = []
    for g0 in ops:
        g = g0 if np.linalg.det(g0) >= 0 else -g0
        if not any(np.abs(s - g).sum() < 1e-6 for s in seen):
            seen.append(g)
    tr = [float(np.trace(g)) for g in seen]
    has4 = any(abs(t - 1) < 1e-6 for t in tr)
    has3z = any(abs(t) < 1e-6 and abs(g[2, 2] - 1) < 1e-6 for t, g in zip(tr, seen))
    has3d = any(abs(t) < 1e-6 and not abs(g[2, 2] - 1) < 1e-6 for t, g in zip(tr, seen))
    six = any(abs(t - 2) < 1e-6 for t in tr)
    return {1: "c1", 2: "c2", 3: "c3", 4: "c4" if has4 else "d2", 6: ("c6" if six else "d3") if (has3z and not has4) else "d3",
            8: "d4", 12: "t" if has3d else "d6", 24: "o"}.get(len(seen), "c1")


def expand_sector(vals, kij, hw, ops, normals):
    """master.zig:384-485 — a fundamental sector (values at Lambert pixels `kij`: column, row from
    −hw, hemisphere sign) expanded to both full sheets: each pixel takes the value at its
    symmetry-equivalent direction deepest inside the sector (bilinear over stored pixels only)."""
    side = 2 * hw + 1
    plane = side * side
    kij = np.asarray(kij, np.int64).reshape(-1, 3)
    vals = np.asarray(vals, np.float64).reshape(-1)
    sec = np.zeros(2 * plane)
    has = np.zeros(2 * plane, bool)
    ix, iy = kij[:, 0] + hw, kij[:, 1] + hw
    ok = (ix >= 0) & (iy >= 0) & (ix < side) & (iy < side)
    south = kij[:, 2] <= 0
    at = np.where(south, plane, 0) + iy * side + ix
    sec[at[ok]] = vals[ok].astype(np.float32)
    has[at[ok]] = True
    needs_south = bool((south & ok).any())
    last = side - 1.0
    rr, cc = np.divmod(np.arange(plane), side)
    xs = np.tile(2 * cc / last - 1, 2)
    ys = np.tile(2 * rr / last - 1, 2)
    d = square_to_sphere(xs, ys, np.repeat([False, True], plane))
    normals = np.asarray(normals, np.float64).reshape(-1, 3)
    eps = 1.0 / max(hw, 1)
    rep = d.copy()
    best = np.full(len(d), -np.inf)
    best_in = np.zeros(len(d), bool)
    for g in ops:
        t = d @ np.asarray(g, np.float64).reshape(3, 3).T
        margin = (t @ normals.T).min(1) if len(normals) else np.full(len(d), np.inf)
        inside = margin >= -eps
        take = (inside & ~best_in) | ((inside == best_in) & (margin > best))
        best = np.where(take, margin, best)
        best_in = np.where(take, inside, best_in)
        rep = np.where(take[:, None], t, rep)
        if len(normals) == 0:
            break
    uv = sphere_to_square(rep)
    use_s = (rep[:, 2] < 0) & needs_south
    out = np.zeros(2 * plane)
    for hs in (False, True):
        idx = np.nonzero(use_s == hs)[0]
        base = plane if hs else 0
        fj = np.clip((uv[idx, 0] + 1) * 0.5 * last, 0, last)
        fi = np.clip((uv[idx, 1] + 1) * 0.5 * last, 0, last)
        c0, r0 = np.floor(fj).astype(np.int64), np.floor(fi).astype(np.int64)
        c1, r1 = np.minimum(c0 + 1, side - 1), np.minimum(r0 + 1, side - 1)
        tj, ti = fj - c0, fi - r0
        acc = np.zeros(len(idx))
        ws = np.zeros(len(idx))
        for p, wgt in ((r0 * side + c0, (1 - ti) * (1 - tj)), (r0 * side + c1, (1 - ti) * tj),
                       (r1 * side + c0, ti * (1 - tj)), (r1 * side + c1, ti * tj)):
            hv = has[base + p]
            acc += np.where(hv, wgt * sec[base + p], 0.0)
            ws += np.where(hv, wgt, 0.0)
        val = np.where(ws > 1e-9, acc / np.where(ws > 1e-9, ws, 1.0), 0.0)
        for k in np.nonzero(ws <= 1e-9)[0]:  # the nearest stored pixel (master.zig:508-525)
            ci, cj = int(round(fi[k])), int(round(fj[k]))
            val[k] = 0.0
            found = False
            for rad in range(1, 8):
                for di in range(-rad, rad + 1):
                    for dj in range(-rad, rad + 1):
                        ii, jj = ci + di, cj + dj
                        if 0 <= ii < side and 0 <= jj < side and has[base + ii * side + jj]:
                            val[k] = sec[base + ii * side + jj]
                            found = True
                            break
                    if found:
                        break
                if found:
                    break
        out[idx] = val
    return side, out


def load_npz(path):
    """master.zig:276-335 — an ebsdsim .npz master: fundamental sector, its Lambert pixels, the
    point group's operators and the sector's normals, expanded to full sheets; then its symmetry."""
    path = Path(path)
    try:
        z = np.load(path, allow_pickle=False)
    except Exception as e:
        raise MasterError(f"NotAMasterPattern: {path}: {e}") from None
    files = set(z.files)
    key = "fundamental_sector" if "fundamental_sector" in files else "integrated_fundamental_sector"
    for k in (key, "fundamental_kij", "pg_operators", "fs_normals"):
        if k not in files:
            raise MasterError(f"NotAMasterPattern: {path} has no {k}")
    fs = np.asarray(z[key])
    kij = np.asarray(z["fundamental_kij"]).astype(np.int64)
    n_k = kij.shape[0]
    if fs.ndim == 3:
        if fs.shape[2] != n_k:
            raise MasterError("NotAMasterPattern: sector and pixels differ")
        vals = fs.reshape(-1)[:n_k].astype(np.float64)
    else:
        sites = fs.shape[1] if fs.ndim == 2 else 1
        vals = fs.reshape(n_k, sites).astype(np.float64).mean(1)
    meta = {}
    if "meta_json" in files:
        try:
            meta = json.loads(bytes(np.asarray(z["meta_json"], np.uint8)).decode())
        except Exception:
            meta = {}
    hw = int(meta["halfw"]) if "halfw" in meta else int(np.abs(kij[:, :2]).max(initial=0))
    ops = np.asarray(z["pg_operators"], np.float64).reshape(-1, 3, 3)
    nrm = np.asarray(z["fs_normals"], np.float64)
    normals = nrm.reshape(-1, 3) if nrm.ndim == 2 else np.zeros((0, 3))
    side, sheets = expand_sector(vals, kij, hw, ops, normals)
    pg = int(meta.get("pg_num") or 0)
    sg = int(meta.get("space_group") or 0)
    m = Master(path.stem, side, normalize(sheets), ops, pg, sg, float(meta.get("voltage_kv") or 0.0))
    m.lattice = lattice_of(meta)
    m.measure_symmetry()
    return m


def lattice_of(meta):
    """master.zig:255-274 — the cell (a, b, c in Å; α, β, γ in degrees) from the metadata's "cell",
    or None when it is absent or not a cell."""
    cell = meta.get("cell") if isinstance(meta, dict) else None
    if not isinstance(cell, dict):
        return None
    try:
        v = [float(cell[k]) for k in ("a_angstrom", "b_angstrom", "c_angstrom", "alpha_deg", "beta_deg", "gamma_deg")]
    except (KeyError, TypeError, ValueError):
        return None
    ok = all(math.isfinite(x) and x > 0 for x in v) and all(x < 180 for x in v[3:])
    return v if ok else None


def write_npz(path, sheets, side, ops, point_group, meta=None):
    """Write full sheets in the ebsdsim layout `load_npz` reads: every pixel of both hemispheres
    in `fundamental_kij` (south with k[2] = −1), the operators identity first, no sector normals,
    so that each pixel samples itself (master.zig:440-452)."""
    hw = (side - 1) // 2
    rr, cc = np.divmod(np.arange(side * side), side)
    kij = np.concatenate([np.stack([cc - hw, rr - hw, np.full(side * side, s)], -1) for s in (1, -1)]).astype(np.int32)
    m = {"halfw": hw, "pg_num": int(point_group)}
    m.update(meta or {})
    buf = io.BytesIO()
    np.savez(buf, fundamental_sector=np.asarray(sheets, np.float32).reshape(1, 1, -1), fundamental_kij=kij,
             pg_operators=np.asarray(ops, np.float64).reshape(-1, 3, 3), fs_normals=np.zeros((0, 3)),
             meta_json=np.frombuffer(json.dumps(m).encode(), np.uint8))
    Path(path).write_bytes(buf.getvalue())


def fold_of(n_fold):
    """master.zig:715-721 — the power of two dividing the rotation order about z."""
    return {4: 4, 2: 2, 6: 2}.get(n_fold, 1)
