"""Equal-area square ↔ hemisphere map (oracle restatement of zebsdsolve `src/lambert.zig`).

Pixel (row, col) of a side × side sheet is at (x, y) = (2col/(side−1) − 1, 2row/(side−1) − 1)
(lambert.zig:1-4).  Vectorised over leading axes.
"""
import math

import numpy as np


def square_to_sphere(x, y, southern):
    """lambert.zig:9-25"""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    sc = math.sqrt(math.pi / 2.0)
    xa = np.abs(x) * sc
    ya = np.abs(y) * sc
    swap = xa >= ya
    xn = np.where(swap, xa, ya)
    yn = np.where(swap, ya, xa)
    safe = np.where(xn == 0, 1.0, xn)
    r = (2 * xn / math.pi) * np.sqrt(np.maximum(math.pi - xn * xn, 0.0))
    ang = math.pi * yn / (4 * safe)
    xh = r * np.cos(ang)
    yh = r * np.sin(ang)
    z = 1 - 2 * xn * xn / math.pi
    hx = np.where(swap, xh, yh) * np.where(x < 0, -1.0, 1.0)
    hy = np.where(swap, yh, xh) * np.where(y < 0, -1.0, 1.0)
    zz = np.where(southern, -z, z)
    v = np.stack([hx, hy, zz], -1)
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    v = v / np.where(n > 0, n, 1.0)
    pole = np.stack([np.zeros_like(z), np.zeros_like(z), np.where(southern, -1.0, 1.0)], -1)
    return np.where((xn == 0)[..., None], pole, v)


def sphere_to_square(v):
    """lambert.zig:28-45 — unit vector(s) [..., 3] → square coordinates of their own hemisphere."""
    v = np.asarray(v, dtype=np.float64)
    kz = np.abs(v[..., 2])
    xn = np.sqrt(np.maximum(math.pi * (1 - kz) / 2, 0.0))
    ax = np.abs(v[..., 0])
    ay = np.abs(v[..., 1])
    sc = math.sqrt(math.pi / 2.0)
    big = ax >= ay
    u = np.where(big, xn, (4 * xn / math.pi) * np.arctan2(ax, np.maximum(ay, 1e-300)))
    w = np.where(big, (4 * xn / math.pi) * np.arctan2(ay, np.maximum(ax, 1e-300)), xn)
    out = np.stack([(u / sc) * np.where(v[..., 0] < 0, -1.0, 1.0), (w / sc) * np.where(v[..., 1] < 0, -1.0, 1.0)], -1)
    return np.where((kz >= 1 - 1e-14)[..., None], 0.0, out)


def sample(sheet, side, x, y):
    """lambert.zig:48-64 — bilinear sample of a side × side sheet at square coordinates."""
    sheet = np.asarray(sheet).reshape(-1)
    last = float(side - 1)
    fj = np.clip((np.asarray(x) + 1) * 0.5 * last, 0.0, last)
    fi = np.clip((np.asarray(y) + 1) * 0.5 * last, 0.0, last)
    c0 = np.floor(fj).astype(np.int64)
    r0 = np.floor(fi).astype(np.int64)
    c1 = np.minimum(c0 + 1, side - 1)
    r1 = np.minimum(r0 + 1, side - 1)
    tj = fj - c0
    ti = fi - r0
    a = sheet[r0 * side + c0].astype(np.float64)
    b = sheet[r0 * side + c1].astype(np.float64)
    c = sheet[r1 * side + c0].astype(np.float64)
    d = sheet[r1 * side + c1].astype(np.float64)
    return (a * (1 - tj) + b * tj) * (1 - ti) + (c * (1 - tj) + d * tj) * ti
