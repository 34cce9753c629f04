"""The plane of source points (the reference's src/plane.zig): where the beam stood for every map
cell, as a transformation of the scan's indices fitted through source points measured on a few
patterns (Winkelmann, Nolze, Cios, Tokarski and Bała, Materials 13 (2020) 2816; kikuchipy's
EBSDDetector.fit_pc).

P (4 × 3, row-major): P · (column, row, 1) = w · (PCx, PCy, PCz, 1). The models, simplest first,
each inside the next: one centre, a tilt line (PCx fixed, PCy and PCz along the rows), the affine
plane (nine numbers), the projective one (eleven). Points are arrays over the fit patterns: row,
col, y = (PCx · aspect, PCy, PCz), w (3 × 3 weights, the inverse covariance up to a factor),
used. Host arithmetic in FP64.
"""
import math

import numpy as np

from . import rotations as R

N = 11
SLOPE_PRIOR = 0.1  # plane.zig:162
MODELS = ("centre", "line", "affine", "projective")
FREE = {"centre": (2, 5, 8), "line": (2, 4, 5, 7, 8), "affine": tuple(range(9)), "projective": tuple(range(11))}


class Points:
    """Source points measured on the fit patterns (plane.zig:49-59)."""

    def __init__(self, row, col, y, w=None, used=None):
        self.row = np.asarray(row, np.float64).reshape(-1)
        self.col = np.asarray(col, np.float64).reshape(-1)
        n = len(self.row)
        self.y = np.asarray(y, np.float64).reshape(n, 3).copy()
        self.w = np.tile(np.eye(3), (n, 1, 1)) if w is None else np.asarray(w, np.float64).reshape(n, 3, 3).copy()
        self.used = np.ones(n, bool) if used is None else np.asarray(used, bool).copy()

    def __len__(self):
        return len(self.row)

    def copy(self):
        return Points(self.row, self.col, self.y, self.w, self.used)


class Frame:
    """plane.zig:101-118 — the map's indices brought to about ±1."""

    def __init__(self, rows, cols, aspect):
        self.c0 = 0.5 * (cols - 1)
        self.r0 = 0.5 * (rows - 1)
        self.sc = max(self.c0, 1.0)
        self.sr = max(self.r0, 1.0)
        self.aspect = aspect


def solve(n, A, b):
    """plane.zig:63-97 — A x = b (n × n) by elimination with partial pivoting; None when a pivot
    is below 1e-300."""
    A = np.array(A, np.float64).reshape(-1)
    side = int(round(math.sqrt(A.size)))
    A = A.reshape(side, side)[:n, :n].copy()
    b = np.array(b, np.float64).reshape(-1)[:n].copy()
    for c in range(n):
        p = c + int(np.argmax(np.abs(A[c:, c])))
        if not abs(A[p, c]) > 1e-300:
            return None
        if p != c:
            A[[c, p]] = A[[p, c]]
            b[[c, p]] = b[[p, c]]
        for r in range(c + 1, n):
            f = A[r, c] / A[c, c]
            if f == 0:
                continue
            A[r, c:] -= f * A[c, c:]
            b[r] -= f * b[c]
    x = np.zeros(n)
    for r in range(n - 1, -1, -1):
        acc = b[r]
        for k in range(r + 1, n):
            acc -= A[r, k] * x[k]
        x[r] = acc / A[r, r]
    return x


def _cr(fr, row, col):
    return (np.asarray(col, np.float64) - fr.c0) / fr.sc, (np.asarray(row, np.float64) - fr.r0) / fr.sr


def _model(theta, c, r):
    w = theta[9] * c + theta[10] * r + 1
    y = np.stack([(theta[3 * k] * c + theta[3 * k + 1] * r + theta[3 * k + 2]) / w for k in range(3)], -1)
    return y, w


def _jacobian(theta, c, r):
    """The place (…, 3) and its Jacobian (…, 3, N) against θ at frame coordinates c, r."""
    y, w = _model(theta, c, r)
    c = np.asarray(c, np.float64)
    J = np.zeros(c.shape + (3, N))
    b = (c / w, r / w, 1 / w)
    for k in range(3):
        for j in range(3):
            J[..., k, 3 * k + j] = b[j]
        J[..., k, 9] = -y[..., k] * c / w
        J[..., k, 10] = -y[..., k] * r / w
    return y, J


def model_at(theta, fr, row, col):
    """plane.zig:123-135 — the model's place for map cells and its Jacobian (…, 3, N)."""
    c, r = _cr(fr, row, col)
    return _jacobian(np.asarray(theta, np.float64), c, r)


def bounded(theta):
    """plane.zig:236-240 — the denominator above a tenth of its middle's over the whole map."""
    return abs(theta[9]) + abs(theta[10]) <= 0.9


def slope_weight(chi2, dof):
    """plane.zig:245-248"""
    return 0.0 if dof == 0 else chi2 / dof / (SLOPE_PRIOR * SLOPE_PRIOR)


def fit_theta(which, pts, fr):
    """plane.zig:168-233 — the model's unknowns θ fitted to the used points by weighted least
    squares (projective: Gauss–Newton from the affine fit, its slopes held to SLOPE_PRIOR against
    the points' scatter). None with too few points, a singular system, or an unbounded plane."""
    every = FREE[which]
    theta = np.zeros(N)
    u = pts.used
    count = int(u.sum())
    if count * 3 < len(every) + 1:
        return None
    c, r = _cr(fr, pts.row[u], pts.col[u])
    Y, W = pts.y[u], pts.w[u]
    most = 40 if which == "projective" else 1
    for it in range(most):
        F = list(FREE["affine"] if (which == "projective" and it == 0) else every)
        f, J = _jacobian(theta, c, r)
        res = Y - f
        chi2 = float(np.einsum("pk,pkl,pl->", res, W, res))
        yy = float(np.einsum("pk,pkl,pl->", Y, W, Y))
        JF = J[:, :, F]  # [p][3][m]
        WJ = np.einsum("pkl,plm->pkm", W, JF)
        g = np.einsum("pkm,pk->m", WJ, res)
        A = np.einsum("pkm,pkn->mn", WJ, JF)
        if which == "projective" and it > 0:
            if chi2 <= 1e-20 * yy:
                break
            lam = slope_weight(chi2, count * 3 - len(every))
            for i, fi in enumerate(F):
                if fi >= 9:
                    A[i, i] += lam
                    g[i] -= lam * theta[fi]
        d = solve(len(F), A, g)
        if d is None:
            return None
        theta[F] += d
        if it > 0 and np.abs(d).max() < 1e-13:
            break
    if which == "projective" and not bounded(theta):
        return None
    return theta


def to_plane(which, theta, fr):
    """plane.zig:252-273 — θ as the plane P of the scan's own indices; None where undefined."""
    P = np.zeros(12)
    for k in range(4):
        a = theta[3 * k] if k < 3 else theta[9]
        b = theta[3 * k + 1] if k < 3 else theta[10]
        c = theta[3 * k + 2] if k < 3 else 1.0
        s = 1 / fr.aspect if k == 0 else 1.0
        P[3 * k] = s * a / fr.sc
        P[3 * k + 1] = s * b / fr.sr
        P[3 * k + 2] = s * (c - a * fr.c0 / fr.sc - b * fr.r0 / fr.sr)
    if not abs(P[11]) > 1e-12:
        return None
    P = P * (1 / P[11])
    if which != "projective":
        P[9] = P[10] = 0.0
    return P


def fit_model(which, pts, fr):
    theta = fit_theta(which, pts, fr)
    return None if theta is None else to_plane(which, theta, fr)


def fit(kind, pts, fr):
    """plane.zig:164-166"""
    return fit_model("projective" if kind == "projective" else "affine", pts, fr)


def at(P, row, col):
    """plane.zig:288-295 — the plane's source point(s) for map cells, pattern-centre coordinates."""
    row = np.asarray(row, np.float64)
    col = np.asarray(col, np.float64)
    w = P[9] * col + P[10] * row + P[11]
    return np.stack([(P[0] * col + P[1] * row + P[2]) / w, (P[3] * col + P[4] * row + P[5]) / w,
                     (P[6] * col + P[7] * row + P[8]) / w], -1)


def misfit(P, pts, aspect):
    """plane.zig:276-285 — each point's rᵀ W r from the plane."""
    pc = at(P, pts.row, pts.col)
    r = pts.y - pc * np.array([aspect, 1.0, 1.0])
    return np.einsum("pk,pkl,pl->p", r, pts.w, r)


def said(P, geo, rows, cols, aspect, h_px, sx, sy):
    """plane.zig:315-364 — what a plane says of the geometry at the map's middle: the source
    there (pc), the sample's frame against the nominal one (rot: a rotation vector in the
    detector's axes), the beam's travel for a row and for a column against the steps and the
    pixel size (step), and the scan's directions off a right angle (skew, radians)."""
    c0, r0 = 0.5 * (cols - 1), 0.5 * (rows - 1)

    def place(pc):
        return np.array([0.5 - pc[1], (0.5 - pc[0]) * aspect, pc[2]])

    h = 0.5
    a = (place(at(P, r0 + h, c0)) - place(at(P, r0 - h, c0))) * (1 / (2 * h))
    b = (place(at(P, r0, c0 + h)) - place(at(P, r0, c0 - h))) * (1 / (2 * h))
    xs, ys = a * (-float(sy)), b * (-float(sx))
    lx, ly = math.sqrt(float(xs @ xs)), math.sqrt(float(ys @ ys))
    out = {"pc": at(P, r0, c0).tolist(), "rot": [0.0, 0.0, 0.0], "step": [0.0, 0.0], "skew": 0.0}
    if geo.px_um > 0 and h_px > 0:
        out["step"] = [lx * h_px * geo.px_um / geo.step_y_um, ly * h_px * geo.px_um / geo.step_x_um]
    if not lx > 0:
        return out
    x = xs * (1 / lx)
    R0 = geo.nominal()
    if ly > 0:
        yn = ys * (1 / ly)
    else:  # a tilt line says nothing across the rows: the nominal y, square to x
        v = R0[1] - x * float(R0[1] @ x)
        lv = math.sqrt(float(v @ v))
        if not lv > 1e-9:
            return out
        yn = v * (1 / lv)
    z = np.cross(x, yn)
    lz = math.sqrt(float(z @ z))
    if not lz > 1e-9:
        return out
    z = z * (1 / lz)
    Rm = np.array([x, np.cross(z, x), z])
    out["rot"] = R.log_map(R.from_matrix(R0.T @ Rm)).tolist()
    out["skew"] = math.asin(min(max(float(x @ yn), -1.0), 1.0))
    return out
