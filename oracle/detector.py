"""The detector side in float64 (oracle restatement of zebsdsolve `src/detector.zig`,
`shaders/detector.wgsl`, `shaders/mastersph.wgsl`, `shaders/common.wgsl` and the per-pattern steps
of `src/planefit.zig`): master lookups,
simulated patterns, rotation-only Gauss–Newton refinement, NMI, chance decoys."""
import math

import numpy as np

from . import rot

PI = math.pi
TAU = 2 * math.pi


def sphere_to_square(v):
    """common.wgsl:44-57 — 1 − |z| taken as (x² + y²)/(1 + |z|)."""
    v = np.asarray(v, np.float64)
    ax = np.abs(v[..., 0])
    ay = np.abs(v[..., 1])
    xn = np.sqrt(np.maximum(PI * 0.5 * (ax * ax + ay * ay) / (1.0 + np.abs(v[..., 2])), 0.0))
    big = ax >= ay
    u = np.where(big, xn, (4.0 * xn / PI) * np.arctan2(ax, np.maximum(ay, 1e-30)))
    w = np.where(big, (4.0 * xn / PI) * np.arctan2(ay, np.maximum(ax, 1e-30)), xn)
    sc = 0.79788456080286536
    return np.stack([u * sc * np.where(v[..., 0] < 0, -1.0, 1.0), w * sc * np.where(v[..., 1] < 0, -1.0, 1.0)], -1)


def square_to_sphere(p, south):
    """mastersph.wgsl:40-62"""
    p = np.asarray(p, np.float64)
    sc = 1.2533141373155003
    xa = np.abs(p[..., 0]) * sc
    ya = np.abs(p[..., 1]) * sc
    swap = xa >= ya
    xn = np.maximum(xa, ya)
    yn = np.minimum(xa, ya)
    safe = np.where(xn > 0, xn, 1.0)
    r = (2.0 * xn / PI) * np.sqrt(np.maximum(PI - xn * xn, 0.0))
    ang = PI * yn / (4.0 * safe)
    hx = r * np.cos(ang)
    hy = r * np.sin(ang)
    hx, hy = np.where(swap, hx, hy), np.where(swap, hy, hx)
    v = np.stack([hx * np.where(p[..., 0] < 0, -1.0, 1.0), hy * np.where(p[..., 1] < 0, -1.0, 1.0), 1.0 - 2.0 * xn * xn / PI], -1)
    v = v / np.linalg.norm(v, axis=-1, keepdims=True)
    v = np.where((xn > 0)[..., None], v, np.array([0.0, 0.0, 1.0]))
    south = np.broadcast_to(np.asarray(south, bool), v.shape[:-1])
    return np.where(south[..., None], v * np.array([1.0, 1.0, -1.0]), v)


def sheet_lookup(table, side, v):
    """detector.wgsl:102-133 (master_at / grad_at) — bilinear over the hemisphere's sheet; `table`
    is [2·side·side] or [2·side·side, 4]."""
    uv = sphere_to_square(v)
    last = float(side - 1)
    fj = np.clip((uv[..., 0] + 1.0) * 0.5 * last, 0.0, last)
    fi = np.clip((uv[..., 1] + 1.0) * 0.5 * last, 0.0, last)
    c0 = np.minimum(np.floor(fj).astype(np.int64), side - 2)
    r0 = np.minimum(np.floor(fi).astype(np.int64), side - 2)
    o = r0 * side + c0 + np.where(np.asarray(v)[..., 2] < 0.0, side * side, 0)
    tj = fj - c0
    ti = fi - r0
    tab = np.asarray(table, np.float64)
    if tab.ndim == 2:
        tj = tj[..., None]
        ti = ti[..., None]
    top = tab[o] * (1 - tj) + tab[o + 1] * tj
    bot = tab[o + side] * (1 - tj) + tab[o + side + 1] * tj
    return top * (1 - ti) + bot * ti


def pixel_dirs(side):
    """mastersph.wgsl:79-85 — direction of every sheet pixel [2·side·side, 3]."""
    plane = side * side
    pix = np.arange(plane)
    last = float(side - 1)
    p = np.stack([2.0 * (pix % side) / last - 1.0, 2.0 * (pix // side) / last - 1.0], -1)
    north = square_to_sphere(p, False)
    south = square_to_sphere(p, True)
    return np.concatenate([north, south])


def symmetrize(sheets, side, ops):
    """mastersph.wgsl:111-122 — the master's mean over its point group: at each sheet pixel's
    direction d, the mean of the master (bilinear) at g·d over the operators g (3 × 3)."""
    d = pixel_dirs(side)
    acc = np.zeros(len(d))
    for g in ops:
        v = d @ np.asarray(g, np.float64).T
        acc += sheet_lookup(sheets, side, v / np.linalg.norm(v, axis=-1, keepdims=True))
    return acc / max(len(ops), 1)


def _tangent_frame(c):
    ref = np.where((np.abs(c[..., 0]) > 0.8)[..., None], np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    e1 = np.cross(c, ref)
    e1 = e1 / np.linalg.norm(e1, axis=-1, keepdims=True)
    e2 = np.cross(c, e1)
    return e1, e2


def _normalize(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def gradient_table(sheets, side):
    """mastersph.wgsl:124-138 — tangent gradient by central differences a sheet pixel apart
    (h = sqrt(2π)/side) with the master's value in .w: [2·side·side, 4]."""
    src = np.asarray(sheets, np.float64).reshape(-1)
    c = pixel_dirs(side)
    e1, e2 = _tangent_frame(c)
    h = math.sqrt(2.0 * PI) / side
    g1 = (sheet_lookup(src, side, _normalize(c + h * e1)) - sheet_lookup(src, side, _normalize(c - h * e1))) / (2.0 * h)
    g2 = (sheet_lookup(src, side, _normalize(c + h * e2)) - sheet_lookup(src, side, _normalize(c - h * e2))) / (2.0 * h)
    g = g1[:, None] * e1 + g2[:, None] * e2
    return np.concatenate([g, src[:, None]], -1)


def sphere_blur(sheets, side, sigma):
    """prep.zig:215-237, mastersph.wgsl:87-109 — Gaussian smoothing on the sphere by passes of
    doubling width over a 9 × 9 tangent lattice (step 0.6σ)."""
    if not (sigma > 0.05):
        return np.asarray(sheets, np.float64).reshape(-1)
    src = np.asarray(sheets, np.float64).reshape(-1)
    px_rad = math.sqrt(2.0 * PI) / side
    left = sigma * sigma
    s = min(sigma, 2.0)
    d = pixel_dirs(side)
    ref = np.where((np.abs(d[..., 0]) > 0.8)[..., None], np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    e1 = _normalize(np.cross(d, ref))
    e2 = np.cross(d, e1)
    while left > 1e-6:
        if s * s > left or left - s * s < 0.02 * left:
            s = math.sqrt(left)
        left -= s * s
        sr = s * px_rad
        step = 0.6 * sr
        k = 1.0 / (2 * sr * sr)
        acc = np.zeros(src.size)
        wsum = 0.0
        for i in range(-4, 5):
            for j in range(-4, 5):
                a = i * step
                b = j * step
                w = math.exp(-(a * a + b * b) * k)
                acc += w * sheet_lookup(src, side, _normalize(d + a * e1 + b * e2))
                wsum += w
        src = acc / wsum
        s *= 2
    return src


def rays(h, w, frame, t):
    """detector.wgsl:250-252 — u = c0·row + c1·col + t for every pixel [h, w, 3]."""
    c0, c1, _ = (np.asarray(c, np.float64) for c in frame)
    rr, cc = np.meshgrid(np.arange(h, dtype=np.float64), np.arange(w, dtype=np.float64), indexing="ij")
    return rr[..., None] * c0 + cc[..., None] * c1 + np.asarray(t, np.float64)


def project(sheets, side, frame, t, q, h, w):
    """detector.wgsl:254-263 — the master at q·normalize(u) for every pixel."""
    u = _normalize(rays(h, w, frame, t))
    return sheet_lookup(np.asarray(sheets).reshape(-1), side, rot.qapply(np.asarray(q, np.float64), u))


def in_mask(h, w, mask):
    """detector.wgsl:95-99"""
    rr, cc = np.meshgrid(np.arange(h, dtype=np.float64), np.arange(w, dtype=np.float64), indexing="ij")
    if mask[2] <= 0:
        return np.ones((h, w), bool)
    return (rr - mask[0]) ** 2 + (cc - mask[1]) ** 2 <= mask[2]


def rot_sums(grad, side, frame, t, q, pattern, mask):
    """detector.wgsl:329-363 — the 19 sums of orientation refinement over the masked pixels."""
    h, w = pattern.shape
    m_ = in_mask(h, w, mask)
    u = _normalize(rays(h, w, frame, t))[m_]
    c = rot.qapply(np.asarray(q, np.float64), u)
    g = sheet_lookup(grad, side, c)
    d = np.cross(c, g[:, :3])
    mv = g[:, 3]
    e = np.asarray(pattern, np.float64)[m_]
    return {
        "s0": np.array([float(m_.sum()), mv.sum(), (mv * mv).sum(), (mv * e).sum()]),
        "sd": d.sum(0), "sv": (mv[:, None] * d).sum(0), "se": (e[:, None] * d).sum(0),
        "hd": (d * d).sum(0), "ho": (d[:, [0, 0, 1]] * d[:, [1, 2, 2]]).sum(0),
    }


def _solve3(h, g):
    """detector.wgsl:519-527 — symmetric 3×3 (xx, xy, xz, yy, yz, zz) by Cramer's rule."""
    m = np.array([[h[0], h[1], h[2]], [h[1], h[3], h[4]], [h[2], h[4], h[5]]])
    det = np.linalg.det(m)
    if abs(det) < 1e-30:
        return np.zeros(3)
    return np.linalg.solve(m, g)


def ncc_grad_hess(t):
    """detector.wgsl:561-584 — NCC, its gradient and Gauss–Newton matrix from the 19 sums."""
    n = max(t["s0"][0], 1.0)
    mean = t["s0"][1] / n
    var_n = t["s0"][2] - n * mean * mean
    ncc = -2.0
    grad = np.zeros(3)
    hess = np.zeros(6)
    if var_n > 1e-12:
        inv = 1.0 / math.sqrt(var_n)
        ncc = t["s0"][3] * inv
        sd = t["sd"]
        au = (t["sv"] - mean * sd) * inv
        grad = (t["se"] - ncc * au) * inv
        iv = inv * inv
        hd, ho = t["hd"], t["ho"]
        hess = np.array([
            (hd[0] - sd[0] * sd[0] / n - au[0] * au[0]) * iv,
            (ho[0] - sd[0] * sd[1] / n - au[0] * au[1]) * iv,
            (ho[1] - sd[0] * sd[2] / n - au[0] * au[2]) * iv,
            (hd[1] - sd[1] * sd[1] / n - au[1] * au[1]) * iv,
            (ho[2] - sd[1] * sd[2] / n - au[1] * au[2]) * iv,
            (hd[2] - sd[2] * sd[2] / n - au[2] * au[2]) * iv,
        ])
    return ncc, grad, hess


def refine(grad, side, frame, t, q0, pattern, mask, iters=8, max_step=math.radians(2.0), scale0=1.0,
           scale_min=0.02, scale_max=1e4):
    """detector.zig:178-202, detector.wgsl:529-542, 561-659 — iters + 1 passes of sums and a
    step from the best point, accepted when the next sums score higher, the curvature scale μ
    adapted by the gain ratio.  Returns (q_best, best NCC, last improving step size)."""
    q_cur = np.asarray(q0, np.float64)
    q_best = q_cur.copy()
    best = -2.0
    mu = scale0
    g_best = np.zeros(3)
    h_best = np.zeros(6)
    last_good = 0.0
    promised = 0.0
    step_len = 0.0
    accepted = 0
    for it in range(iters + 1):
        ncc, g, hess = ncc_grad_hess(rot_sums(grad, side, frame, t, q_cur, pattern, mask))
        if ncc > best:
            if accepted > 0 and promised > 1e-6:
                rho = (ncc - best) / promised
                mu = min(max(mu * (2.0 - rho), mu / 3.0), mu * 3.0)
            q_best = q_cur.copy()
            best = ncc
            g_best = g
            h_best = hess
            last_good = step_len
            accepted += 1
        else:
            mu = mu * 3.0
        mu = min(max(mu, scale_min), scale_max)
        if it == iters:
            break
        hh = h_best * mu
        tr = max(hh[0] + hh[3] + hh[5], 1e-20)
        hh = hh.copy()
        hh[0] += 1e-6 * tr
        hh[3] += 1e-6 * tr
        hh[5] += 1e-6 * tr
        step = _solve3(hh, g_best)
        ln = float(np.linalg.norm(step))
        if ln > max_step:
            step = step * (max_step / ln)
        quad = hh[0] * step[0] ** 2 + hh[3] * step[1] ** 2 + hh[5] * step[2] ** 2 + \
            2.0 * (hh[1] * step[0] * step[1] + hh[2] * step[0] * step[2] + hh[4] * step[1] * step[2])
        promised = float(np.dot(g_best, step)) - 0.5 * quad
        step_len = float(np.linalg.norm(step))
        qn = rot.qmul(rot.so3_exp(step), q_best)
        q_cur = qn / np.linalg.norm(qn)
    return q_best, best, last_good


def nmi(sheets, side, frame, t, q, pattern, mask, n_bins=16):
    """detector.wgsl:744-832 — 2 I(A;B)/(H(A)+H(B)) with each image binned between its own
    extremes under the mask."""
    h, w = pattern.shape
    m_ = in_mask(h, w, mask)
    e = np.asarray(pattern, np.float64)[m_]
    s = project(sheets, side, frame, t, q, h, w)[m_]
    ke = n_bins / max(e.max() - e.min(), 1e-20)
    ks = n_bins / max(s.max() - s.min(), 1e-20)
    be = np.minimum(((e - e.min()) * ke).astype(np.int64), n_bins - 1)
    bs = np.minimum(((s - s.min()) * ks).astype(np.int64), n_bins - 1)
    hist = np.zeros((n_bins, n_bins))
    np.add.at(hist, (be, bs), 1)
    nn = max(hist.sum(), 1.0)

    def ent(c):
        c = c[c > 0]
        return -(c * np.log(c)).sum()

    h_joint = math.log(nn) - (-ent(hist)) / nn
    h_marg = 2 * math.log(nn) - (-ent(hist.sum(1)) - ent(hist.sum(0))) / nn
    return 2.0 * (h_marg - h_joint) / h_marg if h_marg > 1e-12 else 0.0


def hash_u32(x):
    """detector.wgsl:284-288 (wrapping u32 arithmetic)."""
    x = np.asarray(x, np.uint64) & 0xFFFFFFFF
    v = (x * 747796405 + 2891336453) & 0xFFFFFFFF
    w = (((v >> ((v >> 28) + 4)) ^ v) * 277803737) & 0xFFFFFFFF
    return ((w >> 22) ^ w) & 0xFFFFFFFF


def unit_rand(x):
    """detector.wgsl:290-292"""
    return (hash_u32(x) >> 8).astype(np.float64) / 16777216.0


def decoy(b, draw):
    """detector.wgsl:296-308 — Shoemake's uniform rotation from the item and draw numbers."""
    b = np.asarray(b, np.uint64)
    s = hash_u32(b + 1) ^ ((np.uint64(draw) * np.uint64(0x9E3779B9)) & np.uint64(0xFFFFFFFF))
    u1 = unit_rand(s)
    a2 = unit_rand(s + 1) * TAU
    a3 = unit_rand(s + 2) * TAU
    ra = np.sqrt(1.0 - u1)
    rb = np.sqrt(u1)
    return np.stack([ra * np.sin(a2), ra * np.cos(a2), rb * np.sin(a3), rb * np.cos(a3)], -1)


# ── six unknowns per pattern: the source's shift and the crystal's rotation ──

def _catmull_rom(t):
    """Catmull–Rom weights of the texels at −1, 0, 1, 2 and their slopes (detector.wgsl:161-164)."""
    w = 0.5 * np.stack([((-t + 2) * t - 1) * t, (3 * t - 5) * t * t + 2, ((-3 * t + 4) * t + 1) * t, (t - 1) * t * t], -1)
    d = 0.5 * np.stack([(-3 * t + 4) * t - 1, (9 * t - 10) * t, (-9 * t + 8) * t + 1, (3 * t - 2) * t], -1)
    return w, d


def _keys(a):
    """Keys' six-point kernel at a ≥ 0 and its slope (detector.wgsl:193-198)."""
    v = np.where(a < 1, ((4 / 3) * a - 7 / 3) * a * a + 1,
                 np.where(a < 2, ((-7 / 12 * a + 3) * a - 59 / 12) * a + 2.5,
                          np.where(a < 3, ((1 / 12 * a - 2 / 3) * a + 1.75) * a - 1.5, 0.0)))
    d = np.where(a < 1, (4 * a - 14 / 3) * a,
                 np.where(a < 2, (-1.75 * a + 6) * a - 59 / 12, np.where(a < 3, (0.25 * a - 4 / 3) * a + 1.75, 0.0)))
    return v, d


def grad_smooth(sheets, side, v, kind):
    """detector.wgsl:141-248 (grad_at_cubic, kind 1; grad_at_keys6, kind 2) — the master at
    directions v [n, 3] by a smooth kernel over the sheet's texels (indices held inside the sheet),
    with that surface's gradient carried onto the sphere by central differences of the square-
    Lambert map (1e-3 rad along two tangent directions). Returns [n, 4]: gradient, intensity."""
    v = np.asarray(v, np.float64)
    tab = np.asarray(sheets, np.float64).reshape(2, side, side)
    uv = sphere_to_square(v)
    last = float(side - 1)
    fj = np.clip((uv[:, 0] + 1.0) * 0.5 * last, 0.0, last)
    fi = np.clip((uv[:, 1] + 1.0) * 0.5 * last, 0.0, last)
    c0 = np.minimum(np.floor(fj).astype(np.int64), side - 2)
    r0 = np.minimum(np.floor(fi).astype(np.int64), side - 2)
    sh = (v[:, 2] < 0).astype(np.int64)
    tj, ti = fj - c0, fi - r0
    if kind == 1:
        wj, dj = _catmull_rom(tj)
        wi, di = _catmull_rom(ti)
        offs = np.arange(-1, 3)
    else:
        sj = tj[:, None] - (np.arange(6) - 2)[None, :]
        si = ti[:, None] - (np.arange(6) - 2)[None, :]
        wj, dj = _keys(np.abs(sj))
        wi, di = _keys(np.abs(si))
        dj, di = dj * np.sign(sj), di * np.sign(si)
        offs = np.arange(-2, 4)
    rr = np.clip(r0[:, None] + offs[None, :], 0, side - 1)
    cc = np.clip(c0[:, None] + offs[None, :], 0, side - 1)
    T = tab[sh[:, None, None], rr[:, :, None], cc[:, None, :]]  # [n][a][b]
    val = np.einsum("na,nb,nab->n", wi, wj, T)
    gj = np.einsum("na,nb,nab->n", wi, dj, T)
    gi = np.einsum("na,nb,nab->n", di, wj, T)
    e1 = np.cross(v, np.array([0.0, 0.0, 1.0]))
    small = (e1 * e1).sum(-1) < 1e-4
    e1[small] = np.cross(v[small], np.array([1.0, 0.0, 0.0]))
    e1 /= np.linalg.norm(e1, axis=-1, keepdims=True)
    e2 = np.cross(v, e1)
    h = 1e-3
    k = 0.5 * last / (2 * h)

    def s2s(x):
        return sphere_to_square(x / np.linalg.norm(x, axis=-1, keepdims=True))

    d1 = (s2s(v + h * e1) - s2s(v - h * e1)) * k
    d2 = (s2s(v + h * e2) - s2s(v - h * e2)) * k
    g = e1 * (gj * d1[:, 0] + gi * d1[:, 1])[:, None] + e2 * (gj * d2[:, 0] + gi * d2[:, 1])[:, None]
    return np.concatenate([g, val[:, None]], 1)


def sums6(grad, side, frame, t, q, shift, pattern, mask, interp=0, sheets=None):
    """detector.wgsl:435-499 (sums) — the 43 sums over the masked pixels at orientation q with the
    rays' origin moved by `shift` (pixels, sample axes): with u = c0·row + c1·col + t + shift,
    c = q·u/|u| and (∇M, M) = grad(c), the directions d = (q⁻¹·∇M/|u|, c × ∇M); sums
    n, ΣM, ΣM², ΣM·e, Σd (6), ΣM·d (6), Σe·d (6), Σd_i d_j (i ≤ j, 21). interp 1 or 2: the
    master by grad_smooth of the raw sheets instead of the gradient table (plane_interp)."""
    h, w = pattern.shape
    m_ = in_mask(h, w, mask)
    u = (rays(h, w, frame, np.asarray(t, np.float64) + np.asarray(shift, np.float64)))[m_]
    dist = np.linalg.norm(u, axis=-1, keepdims=True)
    q = np.asarray(q, np.float64)
    c = rot.qapply(q, u / dist)
    g = sheet_lookup(grad, side, c) if interp == 0 else grad_smooth(sheets, side, c, interp)
    val = g[:, 3]
    a = np.cross(c, g[:, :3])
    wv = rot.qapply(rot.qconj(q), g[:, :3]) / dist
    d = np.concatenate([wv, a], 1)
    e = np.asarray(pattern, np.float64)[m_]
    s = np.zeros(43)
    s[0] = float(m_.sum())
    s[1] = val.sum()
    s[2] = (val * val).sum()
    s[3] = (val * e).sum()
    s[4:10] = d.sum(0)
    s[10:16] = (val[:, None] * d).sum(0)
    s[16:22] = (e[:, None] * d).sum(0)
    o = 22
    for i in range(6):
        for j in range(i, 6):
            s[o] = (d[:, i] * d[:, j]).sum()
            o += 1
    return s


def local_of(s):
    """planefit.zig:176-200 (localOf) — NCC, its gradient g (6) and Gauss–Newton matrix H (6×6)
    from the 43 sums; None where the simulation has no variance."""
    n = max(s[0], 1.0)
    mean = s[1] / n
    var_n = s[2] - n * mean * mean
    if not var_n > 1e-12:
        return None
    inv = 1.0 / math.sqrt(var_n)
    ncc = s[3] * inv
    sd = s[4:10]
    au = (s[10:16] - mean * sd) * inv
    g = (s[16:22] - ncc * au) * inv
    H = np.zeros((6, 6))
    o = 22
    for i in range(6):
        for j in range(i, 6):
            v = (s[o] - sd[i] * sd[j] / n - au[i] * au[j]) * inv * inv
            H[i, j] = H[j, i] = v
            o += 1
    return ncc, g, H


def solve_pivot(A, b):
    """planefit.zig:203-233 (solve) — elimination with partial pivoting; None when singular."""
    A = np.array(A, np.float64, copy=True)
    b = np.array(b, np.float64, copy=True)
    N = len(b)
    for c in range(N):
        piv = c
        for r in range(c + 1, N):
            if abs(A[r, c]) > abs(A[piv, c]):
                piv = r
        if abs(A[piv, c]) < 1e-300:
            return None
        if piv != c:
            A[[c, piv]] = A[[piv, c]]
            b[[c, piv]] = b[[piv, c]]
        for r in range(c + 1, N):
            f = A[r, c] / A[c, c]
            if f == 0:
                continue
            A[r, c:] -= f * A[c, c:]
            b[r] -= f * b[c]
    x = np.zeros(N)
    for r in range(N - 1, -1, -1):
        x[r] = (b[r] - A[r, r + 1:] @ x[r + 1:]) / A[r, r]
    return x


def damped(H, g, lam):
    """planefit.zig:237-248 (damped, k = 6) — A = H with its diagonal × (1 + λ) + 1e-9·tr + 1e-30."""
    A = np.array(H, np.float64, copy=True)
    tr = np.trace(A)
    A[np.diag_indices(6)] = A[np.diag_indices(6)] * (1 + lam) + 1e-9 * tr + 1e-30
    return A, np.array(g, np.float64)


def settle6(grad, side, frame, t, q0, pattern, mask, trust, most, interp=0, sheets=None):
    """planefit.zig:570-622 (settle, k = 6) for one pattern: Levenberg–Marquardt on its own score
    over the source's shift and its rotation: λ from 1e-3, a step kept where the score rose
    (λ ← max(λ/3, 1e-4)), else λ ← min(5λ, 1e8); the shift clamped to ±trust pixels; stops when
    a round gains less than 1e-7 (a round whose step overshot goes again while λ < 1e8) or after
    `most` rounds. interp / sheets: the master as sums6 takes it. Returns (q, shift, ncc, rounds)."""
    q = rot.qstd(np.asarray(q0, np.float64))
    shift = np.zeros(3)
    keep = local_of(sums6(grad, side, frame, t, q, shift, pattern, mask, interp, sheets))
    lam = 1e-3
    it = 0
    while it < most:
        A, b = damped(keep[2], keep[1], lam)
        d = solve_pivot(A, b)
        qt, st = q, shift
        if d is not None:
            st = np.clip(shift + d[:3], -trust, trust)
            qt = rot.qstd(rot.qmul(rot.so3_exp(d[3:]), q))
        now = local_of(sums6(grad, side, frame, t, qt, st, pattern, mask, interp, sheets))
        gain = 0.0
        kept = damp = 0
        if now is not None and now[0] > keep[0]:
            gain = now[0] - keep[0]
            kept = 1
            q, shift, keep = qt, st, now
            lam = max(lam / 3, 1e-4)
        else:
            if lam < 1e8:
                damp = 1
            lam = min(lam * 5, 1e8)
        if kept == 0 and damp > 0:
            it += 1
            continue
        if gain < 1e-7:  # (planefit.zig:570-622: the loop's continue expression counts rounds; a break does not)
            break
        it += 1
    return q, shift, keep[0], it
