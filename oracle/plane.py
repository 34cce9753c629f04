"""The plane of source points: oracle restatement of zebsdsolve `src/plane.zig` (test
infrastructure — what zebsdsolve_b200.plane is tested against, never part of the product path).

Scalar loops in the reference's order: Frame.of (plane.zig:106-118), model_at / model (123-142),
fit_theta (168-233), bounded (236-240), slope_weight (245-248), to_plane (252-273), misfit
(276-285), at (288-295), said (315-364), solve (63-97). A point is a dict with row, col, y (PCx ·
aspect, PCy, PCz), w (3 × 3, row-major 9) and used.
"""
import math

import numpy as np

from . import rot

N = 11
SLOPE_PRIOR = 0.1
FREE = {"centre": (2, 5, 8), "line": (2, 4, 5, 7, 8), "affine": tuple(range(9)), "projective": tuple(range(11))}


def point(row, col, y, w=None, used=True):
    return {"row": float(row), "col": float(col), "y": [float(v) for v in y],
            "w": list(w) if w is not None else [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0], "used": bool(used)}


def solve(n, A0, b0):
    """plane.zig:63-97 — A is N × N row-major (only the first n rows and columns read)."""
    A = list(A0)
    b = list(b0)
    for c in range(n):
        p = c
        for r in range(c + 1, n):
            if abs(A[r * N + c]) > abs(A[p * N + c]):
                p = r
        if not abs(A[p * N + c]) > 1e-300:
            return None
        if p != c:
            for k in range(n):
                A[c * N + k], A[p * N + k] = A[p * N + k], A[c * N + k]
            b[c], b[p] = b[p], b[c]
        for r in range(c + 1, n):
            f = A[r * N + c] / A[c * N + c]
            if f == 0:
                continue
            for k in range(c, n):
                A[r * N + k] -= f * A[c * N + k]
            b[r] -= f * b[c]
    x = [0.0] * N
    for r in range(n - 1, -1, -1):
        acc = b[r]
        for k in range(r + 1, n):
            acc -= A[r * N + k] * x[k]
        x[r] = acc / A[r * N + r]
    return x


def frame_of(rows, cols, aspect):
    """plane.zig:106-118"""
    c0 = 0.5 * (cols - 1)
    r0 = 0.5 * (rows - 1)
    return {"c0": c0, "r0": r0, "sc": max(c0, 1.0), "sr": max(r0, 1.0), "aspect": aspect}


def model(theta, c, r):
    w = theta[9] * c + theta[10] * r + 1
    return [(theta[3 * k] * c + theta[3 * k + 1] * r + theta[3 * k + 2]) / w for k in range(3)], w


def jacobian(theta, c, r):
    y, w = model(theta, c, r)
    b = (c, r, 1.0)
    J = [0.0] * (3 * N)
    for k in range(3):
        for j in range(3):
            J[k * N + 3 * k + j] = b[j] / w
        J[k * N + 9] = -y[k] * c / w
        J[k * N + 10] = -y[k] * r / w
    return y, J


def model_at(theta, fr, row, col):
    """plane.zig:123-135"""
    c = (col - fr["c0"]) / fr["sc"]
    r = (row - fr["r0"]) / fr["sr"]
    return jacobian(theta, c, r)


def bounded(theta):
    return abs(theta[9]) + abs(theta[10]) <= 0.9


def slope_weight(chi2, dof):
    if dof == 0:
        return 0.0
    return chi2 / dof / (SLOPE_PRIOR * SLOPE_PRIOR)


def fit_theta(which, pts, fr):
    """plane.zig:168-233"""
    every = FREE[which]
    theta = [0.0] * N
    count = sum(1 for p in pts if p["used"])
    if count * 3 < len(every) + 1:
        return None
    most = 40 if which == "projective" else 1
    for it in range(most):
        F = FREE["affine"] if (which == "projective" and it == 0) else every
        m = len(F)
        A = [0.0] * (N * N)
        g = [0.0] * N
        chi2 = 0.0
        yy = 0.0
        for p in pts:
            if not p["used"]:
                continue
            c = (p["col"] - fr["c0"]) / fr["sc"]
            r = (p["row"] - fr["r0"]) / fr["sr"]
            f, J = jacobian(theta, c, r)
            res = [p["y"][k] - f[k] for k in range(3)]
            w = p["w"]
            for k in range(3):
                for l in range(3):
                    chi2 += res[k] * w[k * 3 + l] * res[l]
                    yy += p["y"][k] * w[k * 3 + l] * p["y"][l]
            for i, fi in enumerate(F):
                wj = [0.0, 0.0, 0.0]
                for k in range(3):
                    for l in range(3):
                        wj[k] += w[k * 3 + l] * J[l * N + fi]
                for k in range(3):
                    g[i] += wj[k] * res[k]
                for j, fj in enumerate(F):
                    for k in range(3):
                        A[i * N + j] += wj[k] * J[k * N + fj]
        if which == "projective" and it > 0:
            if chi2 <= 1e-20 * yy:
                break
            lam = slope_weight(chi2, count * 3 - len(every))
            for i, fi in enumerate(F):
                if fi < 9:
                    continue
                A[i * N + i] += lam
                g[i] -= lam * theta[fi]
        d = solve(m, A, g)
        if d is None:
            return None
        moved = 0.0
        for i, fi in enumerate(F):
            theta[fi] += d[i]
            moved = max(moved, abs(d[i]))
        if it > 0 and moved < 1e-13:
            break
    if which == "projective" and not bounded(theta):
        return None
    return theta


def to_plane(which, theta, fr):
    """plane.zig:252-273"""
    P = [0.0] * 12
    for k in range(4):
        a = theta[3 * k] if k < 3 else theta[9]
        b = theta[3 * k + 1] if k < 3 else theta[10]
        c = theta[3 * k + 2] if k < 3 else 1.0
        s = 1 / fr["aspect"] if k == 0 else 1.0
        P[3 * k] = s * a / fr["sc"]
        P[3 * k + 1] = s * b / fr["sr"]
        P[3 * k + 2] = s * (c - a * fr["c0"] / fr["sc"] - b * fr["r0"] / fr["sr"])
    if not abs(P[11]) > 1e-12:
        return None
    scale = 1 / P[11]
    P = [v * scale for v in P]
    if which != "projective":
        P[9] = 0.0
        P[10] = 0.0
    return P


def fit_model(which, pts, fr):
    theta = fit_theta(which, pts, fr)
    return None if theta is None else to_plane(which, theta, fr)


def fit(kind, pts, fr):
    return fit_model("projective" if kind == "projective" else "affine", pts, fr)


def at(P, row, col):
    """plane.zig:288-295"""
    w = P[9] * col + P[10] * row + P[11]
    return [(P[0] * col + P[1] * row + P[2]) / w, (P[3] * col + P[4] * row + P[5]) / w,
            (P[6] * col + P[7] * row + P[8]) / w]


def misfit(P, p, aspect):
    """plane.zig:276-285"""
    pc = at(P, p["row"], p["col"])
    r = [p["y"][0] - pc[0] * aspect, p["y"][1] - pc[1], p["y"][2] - pc[2]]
    q = 0.0
    for i in range(3):
        for j in range(3):
            q += r[i] * p["w"][i * 3 + j] * r[j]
    return q


def said(P, geo, rows, cols, aspect, h_px, sx, sy):
    """plane.zig:315-364 — (pc, rot, step, skew) at the map's middle; geo an oracle Geometry."""
    c0 = 0.5 * (cols - 1)
    r0 = 0.5 * (rows - 1)

    def place(pc):
        return np.array([0.5 - pc[1], (0.5 - pc[0]) * aspect, pc[2]])

    h = 0.5
    a = (place(at(P, r0 + h, c0)) - place(at(P, r0 - h, c0))) * (1 / (2 * h))
    b = (place(at(P, r0, c0 + h)) - place(at(P, r0, c0 - h))) * (1 / (2 * h))
    xs = a * (-float(sy))
    ys = b * (-float(sx))
    lx = math.sqrt(float(np.dot(xs, xs)))
    ly = math.sqrt(float(np.dot(ys, ys)))
    out = {"pc": at(P, r0, c0), "rot": [0.0, 0.0, 0.0], "step": [0.0, 0.0], "skew": 0.0}
    if geo.px_um > 0 and h_px > 0:
        out["step"] = [lx * h_px * geo.px_um / geo.step_y_um, ly * h_px * geo.px_um / geo.step_x_um]
    if not lx > 0:
        return out
    x = xs * (1 / lx)
    R0 = geo.nominal()
    if ly > 0:
        yn = ys * (1 / ly)
    else:
        y0 = np.array([R0[1, 0], R0[1, 1], R0[1, 2]])
        v = y0 - x * float(np.dot(y0, x))
        lv = math.sqrt(float(np.dot(v, v)))
        if not lv > 1e-9:
            return out
        yn = v * (1 / lv)
    z = np.cross(x, yn)
    lz = math.sqrt(float(np.dot(z, z)))
    if not lz > 1e-9:
        return out
    z = z * (1 / lz)
    y = np.cross(z, x)
    Rm = np.array([x, y, z])
    out["rot"] = list(rot.so3_log(rot.from_mat(R0.T @ Rm)))
    out["skew"] = math.asin(min(max(float(np.dot(x, yn)), -1.0), 1.0))
    return out
