"""Host-side rotation math: quaternions (w, x, y, z; v ↦ q v q*; an orientation maps sample to
crystal directions), Bunge angles, the eleven proper rotation groups, fundamental-zone
representatives and disorientations (zebsdsolve src/rot.zig, src/sym.zig).  Vectorised over
leading axes."""
import math

import numpy as np


def qmul(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    aw, ax, ay, az = np.moveaxis(a, -1, 0)
    bw, bx, by, bz = np.moveaxis(b, -1, 0)
    return np.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], -1)


def qconj(q):
    return np.asarray(q, np.float64) * np.array([1.0, -1.0, -1.0, -1.0])


def qstd(q):
    """unit norm, non-negative w (rot.zig:60-64)"""
    q = np.asarray(q, np.float64)
    n = np.linalg.norm(q, axis=-1, keepdims=True)
    n = np.where(n == 0, 1.0, n)
    return q / n * np.where(q[..., :1] < 0, -1.0, 1.0)


def qapply(q, v):
    q = np.asarray(q, np.float64)
    u = q[..., 1:]
    t = 2.0 * np.cross(u, v)
    return v + q[..., :1] * t + np.cross(u, t)


def to_matrix(q):
    w, x, y, z = (float(c) for c in q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def from_matrix(m):
    """Shepperd (rot.zig:87-104)"""
    m = np.asarray(m, np.float64)
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0:
        s = 2 * math.sqrt(tr + 1.0)
        q = (0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s)
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = 2 * math.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2])
        q = ((m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s)
    elif m[1, 1] > m[2, 2]:
        s = 2 * math.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2])
        q = ((m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s)
    else:
        s = 2 * math.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1])
        q = ((m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s)
    return qstd(np.array(q))


def exp_map(phi):
    """so(3) exp of rotation vectors [..., 3] (rot.zig:192-198)"""
    phi = np.asarray(phi, np.float64)
    th = np.linalg.norm(phi, axis=-1, keepdims=True)
    k = np.where(th < 1e-6, 0.5 - th * th / 48.0, np.sin(0.5 * th) / np.where(th < 1e-6, 1.0, th))
    return np.concatenate([np.cos(0.5 * th), k * phi], -1)


def log_map(q):
    """so(3) log: the rotation vector of quaternions [..., 4] (rot.zig:201-207)"""
    q = qstd(q)
    s = np.linalg.norm(q[..., 1:], axis=-1, keepdims=True)
    k = np.where(s < 1e-9, 2.0, 2.0 * np.arctan2(s, q[..., :1]) / np.where(s < 1e-9, 1.0, s))
    return k * q[..., 1:]


def to_bunge(q):
    """Bunge (φ1, Φ, φ2) radians of quaternions [..., 4] (rot.zig:151-173)"""
    q = qstd(q)
    w, x, y, z = np.moveaxis(q, -1, 0)
    q03 = w * w + z * z
    q12 = x * x + y * y
    chi = np.sqrt(q03 * q12)
    safe = np.where(chi < 1e-14, 1.0, chi)
    e1 = np.arctan2((x * z - w * y) / safe, (-w * x - y * z) / safe)
    e2 = np.arctan2(2 * chi, q03 - q12)
    e3 = np.arctan2((w * y + x * z) / safe, (y * z - w * x) / safe)
    small = chi < 1e-14
    lo = q12 <= q03
    e1 = np.where(small, np.where(lo, np.arctan2(-2 * w * z, w * w - z * z), np.arctan2(2 * x * y, x * x - y * y)), e1)
    e2 = np.where(small, np.where(lo, 0.0, math.pi), e2)
    e3 = np.where(small, 0.0, e3)
    e1 = np.where(e1 < 0, e1 + 2 * math.pi, e1)
    e3 = np.where(e3 < 0, e3 + 2 * math.pi, e3)
    return np.stack([e1, e2, e3], -1)


_r2 = math.sqrt(0.5)
_r3 = math.sqrt(3.0) / 2
_GROUPS = {}
_GROUPS["c1"] = [(1, 0, 0, 0)]
_GROUPS["c2"] = _GROUPS["c1"] + [(0, 0, 0, 1)]
_GROUPS["d2"] = _GROUPS["c2"] + [(0, 1, 0, 0), (0, 0, 1, 0)]
_GROUPS["c4"] = _GROUPS["c2"] + [(_r2, 0, 0, _r2), (_r2, 0, 0, -_r2)]
_GROUPS["d4"] = _GROUPS["c4"] + [(0, 1, 0, 0), (0, 0, 1, 0), (0, _r2, _r2, 0), (0, -_r2, _r2, 0)]
_GROUPS["c3"] = [(1, 0, 0, 0), (0.5, 0, 0, _r3), (0.5, 0, 0, -_r3)]
_GROUPS["d3"] = _GROUPS["c3"] + [(0, 1, 0, 0), (0, -0.5, _r3, 0), (0, 0.5, _r3, 0)]
_GROUPS["c6"] = _GROUPS["c3"] + [(0, 0, 0, 1), (_r3, 0, 0, 0.5), (_r3, 0, 0, -0.5)]
_GROUPS["d6"] = _GROUPS["c6"] + [(0, 1, 0, 0), (0, -0.5, _r3, 0), (0, 0.5, _r3, 0), (0, _r3, 0.5, 0),
                                 (0, -_r3, 0.5, 0), (0, 0, 1, 0)]
_GROUPS["t"] = _GROUPS["d2"] + [(0.5, s1 * 0.5, s2 * 0.5, s3 * 0.5) for s1, s2, s3 in
                                ((1, -1, 1), (1, 1, -1), (1, -1, -1), (-1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1),
                                 (1, 1, 1))]
_GROUPS["o"] = _GROUPS["t"] + [(_r2, 0, 0, _r2), (_r2, 0, 0, -_r2), (0, _r2, _r2, 0), (0, -_r2, _r2, 0),
                               (_r2, _r2, 0, 0), (_r2, -_r2, 0, 0), (_r2, 0, _r2, 0), (_r2, 0, -_r2, 0),
                               (0, _r2, 0, _r2), (0, -_r2, 0, _r2), (0, 0, _r2, _r2), (0, 0, -_r2, _r2)]

LAUE_NAMES = {"c1": "-1", "c2": "2/m", "d2": "mmm", "c4": "4/m", "d4": "4/mmm", "c3": "-3", "d3": "-3m", "c6": "6/m",
              "d6": "6/mmm", "t": "m-3", "o": "m-3m"}
LAUE_NUMBERS = {k: i + 1 for i, k in enumerate(("c1", "c2", "d2", "c4", "d4", "c3", "d3", "c6", "d6", "t", "o"))}


def group(kind):
    """The rotations of one of the eleven groups, identity first (sym.zig:74-113)."""
    return np.array(_GROUPS[kind], np.float64)


def to_fz(q, ops):
    """The symmetry-equivalent g·q with the largest w, ties keeping the first (sym.zig:120-131)."""
    q = np.asarray(q, np.float64)
    best = qstd(q)
    bw = best[..., 0].copy()
    for g in np.asarray(ops, np.float64):
        c = qstd(qmul(np.broadcast_to(g, q.shape), q))
        take = c[..., 0] > bw + 1e-12
        best = np.where(take[..., None], c, best)
        bw = np.where(take, c[..., 0], bw)
    return best


def disorientation(a, b, ops):
    """Smallest rotation angle between a and b over the group `ops`, radians (sym.zig:135-145)."""
    m = qmul(a, qconj(b))
    best = m
    for g in np.asarray(ops, np.float64):
        c = qmul(np.broadcast_to(g, m.shape), m)
        best = np.where((np.abs(c[..., 0]) > np.abs(best[..., 0]))[..., None], c, best)
    return 2 * np.arctan2(np.linalg.norm(best[..., 1:], axis=-1), np.abs(best[..., 0]))


# ── a master's symmetry in its own setting (sym.zig:148-344) ──

def _axis_order(q):
    s = float(np.linalg.norm(q[1:]))
    if s < 1e-9:
        return np.array([0.0, 0.0, 1.0]), 1
    return np.asarray(q[1:]) / s, int(round(2 * math.pi / (2 * math.atan2(s, abs(q[0])))))


def _contains(lst, q):
    return any(abs(float(np.dot(s, q))) > 1 - 1e-6 for s in lst)


def _closure(lst):
    out = [np.array([1.0, 0, 0, 0])] + [q for q in lst if not abs(float(q[0])) > 1 - 1e-6]
    grew = True
    while grew:
        grew = False
        for a in list(out):
            for b in list(out):
                c = qstd(qmul(a, b))
                if not _contains(out, c):
                    if len(out) >= 24:
                        return None
                    out.append(c)
                    grew = True
    return out


def _kind(lst):
    top = max(_axis_order(q)[1] for q in lst)
    return {1: "c1", 2: "c2", 3: "c3", 4: "c4" if top == 4 else "d2", 6: "c6" if top == 6 else "d3", 8: "d4",
            12: "d6" if top == 6 else "t", 24: "o"}.get(len(lst))


class Setting:
    """The rotations a master obeys (its orientations are reduced by these), its Laue class and the
    frame that takes the tables' standard setting to the master's."""

    def __init__(self, rotation="c1", laue="c1", frame=(1.0, 0, 0, 0), rots=None):
        self.rotation = rotation
        self.laue = laue
        self.frame = np.array(frame, np.float64)
        self.rots = np.array(rots if rots is not None else [(1.0, 0, 0, 0)], np.float64)


def setting_of(mats):
    """The setting of the point-group operators `mats` (3 × 3; proper and improper), or None when
    they make no crystallographic group (sym.zig:275-344)."""
    p, l = [], []
    for m in mats:
        m = np.asarray(m, np.float64).reshape(3, 3)
        proper = np.linalg.det(m) > 0
        q = qstd(from_matrix(m if proper else -m))
        if proper and not _contains(p, q):
            p.append(q)
        if not _contains(l, q):
            l.append(q)
    p, l = _closure(p), _closure(l)
    if p is None or l is None:
        return None
    kp, kl = _kind(p), _kind(l)
    if kp is None or kl is None:
        return None
    out = Setting(kp, kl, rots=p)
    if kl == "c1":
        return out
    principal = {"c1": 1, "c2": 2, "d2": 2, "t": 2, "c3": 3, "d3": 3, "c4": 4, "d4": 4, "o": 4, "c6": 6, "d6": 6}[kl]
    want_x = {"o": 4, "t": 2, "d2": 2, "d3": 2, "d4": 2, "d6": 2}.get(kl, 0)

    def frame_from(zv, xv):
        yv = np.cross(zv, xv)
        return qstd(from_matrix(np.stack([xv, yv, zv], 1)))

    def fits(lst, k, f):
        ops = group(k)
        return len(ops) == len(lst) and all(_contains(lst, qmul(qmul(f, g), qconj(f))) for g in ops)

    best_w = -1.0
    for qz in l:
        az, oz = _axis_order(qz)
        if oz != principal:
            continue
        for sz in (1.0, -1.0):
            zv = az * sz
            cands = []
            if want_x == 0:
                e = np.array([1.0, 0, 0]) if abs(zv[0]) < 0.9 else np.array([0, 1.0, 0])
                xv = e - zv * np.dot(e, zv)
                cands.append(frame_from(zv, xv / np.linalg.norm(xv)))
            else:
                for qx in l:
                    ax, ox = _axis_order(qx)
                    if ox == want_x and abs(np.dot(ax, zv)) <= 1e-6:
                        cands += [frame_from(zv, ax), frame_from(zv, -ax)]
            for f in cands:
                if abs(f[0]) > best_w + 1e-12 and fits(l, kl, f) and fits(p, kp, f):
                    best_w = abs(f[0])
                    out.frame = qstd(f)
    return out if best_w >= 0 else None


def laue_of_point_group(pg):
    for lo, hi, k in ((1, 2, "c1"), (3, 5, "c2"), (6, 8, "d2"), (9, 11, "c4"), (12, 15, "d4"), (16, 17, "c3"),
                      (18, 20, "d3"), (21, 23, "c6"), (24, 27, "d6"), (28, 29, "t"), (30, 32, "o")):
        if lo <= pg <= hi:
            return k
    return None


POINT_GROUP_NAMES = ["1", "-1", "2", "m", "2/m", "222", "mm2", "mmm", "4", "-4", "4/m", "422", "4mm", "-42m", "4/mmm",
                     "3", "-3", "32", "3m", "-3m", "6", "-6", "6/m", "622", "6mm", "-6m2", "6/mmm", "23", "m-3", "432",
                     "-43m", "m-3m"]
