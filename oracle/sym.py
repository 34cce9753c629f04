"""Crystal rotation groups, fundamental zone, disorientation (oracle restatement of `src/sym.zig`)."""
import math

import numpy as np

from . import rot

r2 = 0.70710678118654752440
r3 = 0.86602540378443864676

# sym.zig:74-96 (identity first)
C1 = [(1, 0, 0, 0)]
C2 = [(1, 0, 0, 0), (0, 0, 0, 1)]
D2 = [(1, 0, 0, 0), (0, 0, 0, 1), (0, 1, 0, 0), (0, 0, 1, 0)]
C4 = [(1, 0, 0, 0), (0, 0, 0, 1), (r2, 0, 0, r2), (r2, 0, 0, -r2)]
D4 = C4 + [(0, 1, 0, 0), (0, 0, 1, 0), (0, r2, r2, 0), (0, -r2, r2, 0)]
C3 = [(1, 0, 0, 0), (0.5, 0, 0, r3), (0.5, 0, 0, -r3)]
D3 = C3 + [(0, 1, 0, 0), (0, -0.5, r3, 0), (0, 0.5, r3, 0)]
C6 = C3 + [(0, 0, 0, 1), (r3, 0, 0, 0.5), (r3, 0, 0, -0.5)]
D6 = C6 + [(0, 1, 0, 0), (0, -0.5, r3, 0), (0, 0.5, r3, 0), (0, r3, 0.5, 0), (0, -r3, 0.5, 0), (0, 0, 1, 0)]
T = D2 + [(0.5, 0.5, -0.5, 0.5), (0.5, 0.5, 0.5, -0.5), (0.5, 0.5, -0.5, -0.5), (0.5, -0.5, -0.5, -0.5),
          (0.5, -0.5, 0.5, 0.5), (0.5, -0.5, 0.5, -0.5), (0.5, -0.5, -0.5, 0.5), (0.5, 0.5, 0.5, 0.5)]
O = T + [(r2, 0, 0, r2), (r2, 0, 0, -r2), (0, r2, r2, 0), (0, -r2, r2, 0),
         (r2, r2, 0, 0), (r2, -r2, 0, 0), (r2, 0, r2, 0), (r2, 0, -r2, 0),
         (0, r2, 0, r2), (0, -r2, 0, r2), (0, 0, r2, r2), (0, 0, -r2, r2)]

# sym.zig:17-39 — Laue enum values
LAUE = {"c1": 1, "c2": 2, "d2": 3, "c4": 4, "d4": 5, "c3": 6, "d3": 7, "c6": 8, "d6": 9, "t": 10, "o": 11}
_GROUPS = {"c1": C1, "c2": C2, "d2": D2, "c4": C4, "d4": D4, "c3": C3, "d3": D3, "c6": C6, "d6": D6, "t": T, "o": O}


def operators(kind):
    """sym.zig:99-113"""
    return np.array(_GROUPS[kind], dtype=np.float64)


def to_fz(q, ops):
    """sym.zig:120-131 — g·q with the largest w (ties keep the first)."""
    best = rot.qstd(q)
    best_w = best[0]
    for g in ops:
        c = rot.qstd(rot.qmul(g, q))
        if c[0] > best_w + 1e-12:
            best_w = c[0]
            best = c
    return best


def disorientation(a, b, ops):
    """sym.zig:135-145 — smallest rotation angle between a and b over `ops` (radians).
    Vectorised over leading axes of a and b."""
    m = rot.qmul(a, rot.qconj(b))
    best = m
    for g in ops:
        c = rot.qmul(np.broadcast_to(g, m.shape), m)
        take = np.abs(c[..., 0]) > np.abs(best[..., 0])
        best = np.where(take[..., None], c, best)
    return 2 * np.arctan2(np.sqrt((best[..., 1:] ** 2).sum(-1)), np.abs(best[..., 0]))


def _axis_order(q):
    """sym.zig:172-177"""
    s = math.sqrt(q[1] ** 2 + q[2] ** 2 + q[3] ** 2)
    if s < 1e-9:
        return np.array([0.0, 0.0, 1.0]), 1
    t = 2 * math.atan2(s, abs(q[0]))
    return np.array([q[1], q[2], q[3]]) / s, int(round(2 * math.pi / t))


def _same(a, b):
    return abs(float(np.dot(a, b))) > 1 - 1e-6


def _has(lst, q):
    return any(_same(s, q) for s in lst)


def _close(lst):
    """sym.zig:190-225 — the group generated (identity first)."""
    ident = np.array([1.0, 0, 0, 0])
    out = [np.asarray(q, dtype=np.float64) for q in lst]
    if not _has(out, ident):
        out.append(ident)
    for i, q in enumerate(out):
        if _same(q, ident):
            out[i] = out[0]
            out[0] = ident
            break
    grew = True
    while grew:
        grew = False
        i = 0
        while i < len(out):
            j = 0
            while j < len(out):
                c = rot.qstd(rot.qmul(out[i], out[j]))
                if not _has(out, c):
                    if len(out) == 24:
                        return None
                    out.append(c)
                    grew = True
                j += 1
            i += 1
    return out


def _kind_of(lst):
    """sym.zig:228-243"""
    top = max(_axis_order(q)[1] for q in lst)
    n = len(lst)
    return {1: "c1", 2: "c2", 3: "c3", 4: "c4" if top == 4 else "d2", 6: "c6" if top == 6 else "d3",
            8: "d4", 12: "d6" if top == 6 else "t", 24: "o"}.get(n)


def _principal_order(k):
    """sym.zig:247-255"""
    return {"c1": 1, "c2": 2, "d2": 2, "t": 2, "c3": 3, "d3": 3, "c4": 4, "d4": 4, "o": 4, "c6": 6, "d6": 6}[k]


def _frame_from(zv, xv):
    """sym.zig:258-262"""
    yv = np.cross(zv, xv)
    return rot.qstd(rot.from_mat(np.array([[xv[0], yv[0], zv[0]], [xv[1], yv[1], zv[1]], [xv[2], yv[2], zv[2]]])))


def _is_in(lst, k, f):
    """sym.zig:265-270"""
    ops = operators(k)
    if len(ops) != len(lst):
        return False
    for g in ops:
        if not _has(lst, rot.qmul(rot.qmul(f, g), rot.qconj(f))):
            return False
    return True


class Setting:
    """sym.zig:155-169"""

    def __init__(self, rotation="c1", laue="c1", frame=(1.0, 0, 0, 0), rots=None):
        self.rotation = rotation
        self.laue = laue
        self.frame = np.array(frame, dtype=np.float64)
        self.rots = np.array(rots if rots is not None else [(1.0, 0, 0, 0)], dtype=np.float64)

    def rotations(self):
        return self.rots


def setting_of(mats):
    """sym.zig:275-344 — the master's symmetry from the operators it obeys (None: no group)."""
    p = []
    lq = []
    for m in mats:
        m = np.asarray(m, dtype=np.float64).reshape(3, 3)
        proper = np.linalg.det(m) > 0
        r = m if proper else -m
        q = rot.qstd(rot.from_mat(r))
        if proper and not _has(p, q):
            p.append(q)
        if not _has(lq, q):
            lq.append(q)
    p = _close(p)
    lq = _close(lq)
    if p is None or lq is None:
        return None
    kp = _kind_of(p)
    kl = _kind_of(lq)
    if kp is None or kl is None:
        return None
    out = Setting(kp, kl, rots=p)
    if kl == "c1":
        return out
    want_x = {"o": 4, "t": 2, "d2": 2, "d3": 2, "d4": 2, "d6": 2}.get(kl, 0)
    best_w = -1.0

    def attempt(f):
        nonlocal best_w
        if abs(f[0]) <= best_w + 1e-12:
            return
        if not _is_in(lq, kl, f) or not _is_in(p, kp, f):
            return
        best_w = abs(f[0])
        out.frame = rot.qstd(f)

    for qz in lq:
        az, oz = _axis_order(qz)
        if oz != _principal_order(kl):
            continue
        for sz in (1.0, -1.0):
            zv = az * sz
            if want_x == 0:
                e = np.array([1.0, 0, 0]) if abs(zv[0]) < 0.9 else np.array([0, 1.0, 0])
                xv = e - zv * np.dot(e, zv)
                xv = xv / np.linalg.norm(xv)
                attempt(_frame_from(zv, xv))
                continue
            for qx in lq:
                ax, ox = _axis_order(qx)
                if ox != want_x or abs(np.dot(ax, zv)) > 1e-6:
                    continue
                for sx in (1.0, -1.0):
                    attempt(_frame_from(zv, ax * sx))
    return out if best_w >= 0 else None


def laue_of_point_group(pg):
    """sym.zig:347-362"""
    table = [(1, 2, "c1"), (3, 5, "c2"), (6, 8, "d2"), (9, 11, "c4"), (12, 15, "d4"), (16, 17, "c3"),
             (18, 20, "d3"), (21, 23, "c6"), (24, 27, "d6"), (28, 29, "t"), (30, 32, "o")]
    for lo, hi, k in table:
        if lo <= pg <= hi:
            return k
    return None


def rotations_of_point_group(pg):
    """sym.zig:367-383"""
    t = {1: "c1", 2: "c1", 4: "c1", 3: "c2", 5: "c2", 7: "c2", 10: "c2", 6: "d2", 8: "d2", 14: "d2",
         9: "c4", 11: "c4", 13: "c4", 12: "d4", 15: "d4", 16: "c3", 17: "c3", 19: "c3", 22: "c3",
         18: "d3", 20: "d3", 26: "d3", 21: "c6", 23: "c6", 25: "c6", 24: "d6", 27: "d6",
         28: "t", 29: "t", 31: "t", 30: "o", 32: "o"}
    return t.get(pg)
