"""Rotations in float64 (oracle restatement of zebsdsolve `src/rot.zig`).

A quaternion is (w, x, y, z), acts as q v q*; an orientation maps sample directions to crystal
directions (rot.zig:3-7).  Functions accept a single quaternion or arrays [..., 4].
"""
import math

import numpy as np


def qmul(a, b):
    """rot.zig:46-53"""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    w = a[..., 0] * b[..., 0] - a[..., 1] * b[..., 1] - a[..., 2] * b[..., 2] - a[..., 3] * b[..., 3]
    x = a[..., 0] * b[..., 1] + a[..., 1] * b[..., 0] + a[..., 2] * b[..., 3] - a[..., 3] * b[..., 2]
    y = a[..., 0] * b[..., 2] - a[..., 1] * b[..., 3] + a[..., 2] * b[..., 0] + a[..., 3] * b[..., 1]
    z = a[..., 0] * b[..., 3] + a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1] + a[..., 3] * b[..., 0]
    return np.stack([w, x, y, z], -1)


def qconj(q):
    """rot.zig:55-57"""
    q = np.asarray(q, dtype=np.float64)
    return q * np.array([1.0, -1.0, -1.0, -1.0])


def qstd(q):
    """rot.zig:60-64 — unit norm with a non-negative real part."""
    q = np.asarray(q, dtype=np.float64)
    n = np.sqrt((q * q).sum(-1, keepdims=True))
    n = np.where(n == 0, 1.0, n)
    s = np.where(q[..., :1] < 0, -1.0, 1.0)
    return q * s / n


def qapply(q, v):
    """rot.zig:67-71 — q v q*"""
    q = np.asarray(q, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    u = q[..., 1:4]
    t = 2 * np.cross(u, v)
    return v + q[..., :1] * t + np.cross(u, t)


def to_mat(q):
    """rot.zig:74-84 — matrix of v ↦ q v q* (row-major 3×3)."""
    w, x, y, z = (float(c) for c in q)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
    ])


def from_mat(m):
    """rot.zig:87-104 — Shepperd's method."""
    m = np.asarray(m, dtype=np.float64).reshape(9)
    tr = m[0] + m[4] + m[8]
    if tr > 0:
        s = math.sqrt(tr + 1.0) * 2
        q = [0.25 * s, (m[7] - m[5]) / s, (m[2] - m[6]) / s, (m[3] - m[1]) / s]
    elif m[0] > m[4] and m[0] > m[8]:
        s = math.sqrt(1.0 + m[0] - m[4] - m[8]) * 2
        q = [(m[7] - m[5]) / s, 0.25 * s, (m[1] + m[3]) / s, (m[2] + m[6]) / s]
    elif m[4] > m[8]:
        s = math.sqrt(1.0 + m[4] - m[0] - m[8]) * 2
        q = [(m[2] - m[6]) / s, (m[1] + m[3]) / s, 0.25 * s, (m[5] + m[7]) / s]
    else:
        s = math.sqrt(1.0 + m[8] - m[0] - m[4]) * 2
        q = [(m[3] - m[1]) / s, (m[2] + m[6]) / s, (m[5] + m[7]) / s, 0.25 * s]
    return qstd(np.array(q))


def from_bunge(e):
    """rot.zig:142-148"""
    sigma = 0.5 * (e[0] + e[2])
    delta = 0.5 * (e[0] - e[2])
    c = math.cos(0.5 * e[1])
    s = math.sin(0.5 * e[1])
    return qstd(np.array([c * math.cos(sigma), -s * math.cos(delta), -s * math.sin(delta), -c * math.sin(sigma)]))


def to_bunge(q0):
    """rot.zig:151-173 — Bunge (phi1, Phi, phi2), phi1, phi2 in [0, 2π), Phi in [0, π]."""
    q = qstd(np.asarray(q0, dtype=np.float64))
    q03 = q[0] * q[0] + q[3] * q[3]
    q12 = q[1] * q[1] + q[2] * q[2]
    chi = math.sqrt(q03 * q12)
    if chi < 1e-14:
        if q12 <= q03:
            e = [math.atan2(-2 * q[0] * q[3], q[0] * q[0] - q[3] * q[3]), 0.0, 0.0]
        else:
            e = [math.atan2(2 * q[1] * q[2], q[1] * q[1] - q[2] * q[2]), math.pi, 0.0]
    else:
        e = [
            math.atan2((q[1] * q[3] - q[0] * q[2]) / chi, (-q[0] * q[1] - q[2] * q[3]) / chi),
            math.atan2(2 * chi, q03 - q12),
            math.atan2((q[0] * q[2] + q[1] * q[3]) / chi, (q[2] * q[3] - q[0] * q[1]) / chi),
        ]
    if e[0] < 0:
        e[0] += 2 * math.pi
    if e[2] < 0:
        e[2] += 2 * math.pi
    return np.array(e)


def from_zyz(a, b, c):
    """rot.zig:176-181 — Rz(a) Ry(b) Rz(c) (active)."""
    qa = np.array([math.cos(0.5 * a), 0, 0, math.sin(0.5 * a)])
    qb = np.array([math.cos(0.5 * b), 0, math.sin(0.5 * b), 0])
    qc = np.array([math.cos(0.5 * c), 0, 0, math.sin(0.5 * c)])
    return qmul(qa, qmul(qb, qc))


def so3_exp(phi):
    """rot.zig:192-198"""
    phi = np.asarray(phi, dtype=np.float64)
    th2 = float(np.dot(phi, phi))
    th = math.sqrt(th2)
    k = 0.5 - th2 / 48.0 if th < 1e-6 else math.sin(0.5 * th) / th
    return np.array([math.cos(0.5 * th), k * phi[0], k * phi[1], k * phi[2]])


def so3_log(q0):
    """rot.zig:201-207"""
    q = qstd(q0)
    s = math.sqrt(q[1] ** 2 + q[2] ** 2 + q[3] ** 2)
    k = 2.0 if s < 1e-9 else 2.0 * math.atan2(s, q[0]) / s
    return np.array([k * q[1], k * q[2], k * q[3]])


def angle_between(a, b):
    """rot.zig:184-187"""
    d = abs(float(np.dot(a, b)))
    return 2 * math.acos(min(d, 1.0))
