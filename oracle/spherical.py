"""Spherical indexing in float64 (oracle restatement of zebsdsolve `src/spherical.zig`,
`shaders/sphere.wgsl` and `shaders/so3.wgsl`).

coefficients: a pattern on the sphere (window-mean centred, windowed) → SH coefficients of unit
norm; correlate: coefficients × a master → the normalized correlation volume over the Euler grid
and its peak.  Where the kernels use ring/mirror-paired FFTs and half-length real transforms,
this restatement uses the plain definitions (numpy FFTs over the same grids), which the kernels
compute exactly in exact arithmetic.
"""
import math

import numpy as np

from . import rot, sh

FLAG_CENTER = 1
FLAG_NORM = 2
FLAG_WINDOW = 4


def fft_size(L):
    """spherical.zig:100-104"""
    n = 16
    while n < 2 * L - 1:
        n *= 2
    return n


class Tables:
    """spherical.zig:106-190 — what depends on the bandwidth only (in float64)."""

    def __init__(self, L):
        self.L = L
        self.n = fft_size(L)
        self.n_theta = self.n
        self.n_phi = 2 * self.n
        self.grid = sh.Grid(L, self.n_theta, self.n_phi)
        self.n_pairs = sh.pair_count(L)
        self.wigner = sh.wigner_half_pi(L)


def sample_grid(tables, pattern, t, frame, mask, window=False):
    """sphere.wgsl:128-163 — every GL direction's ray onto the detector: (value, window) [nθ, nφ]."""
    c0, c1, c2 = (np.asarray(c, np.float64) for c in frame)
    t = np.asarray(t, np.float64)
    h, w = (pattern.shape if pattern is not None else (0, 0))
    if window and pattern is None:
        raise ValueError("window sampling needs the pattern shape")
    d = tables.grid.directions()
    nd = d @ c2
    ok = nd > 1e-4
    safe = np.where(ok, nd, 1.0)
    hv = (float(np.dot(c2, t)) / safe)[..., None] * d - t
    row = hv @ c0
    col = hv @ c1
    inb = ok & (row >= 0) & (row <= h - 1) & (col >= 0) & (col <= w - 1)
    if mask[2] > 0:
        dr = row - mask[0]
        dc = col - mask[1]
        inb &= dr * dr + dc * dc <= mask[2]
    win = inb.astype(np.float64)
    if window:
        return win.copy(), win
    rr = np.where(inb, row, 0.0)
    cc = np.where(inb, col, 0.0)
    r0 = np.minimum(np.floor(rr).astype(np.int64), h - 2)
    q0 = np.minimum(np.floor(cc).astype(np.int64), w - 2)
    fr = rr - r0
    fc = cc - q0
    p = np.asarray(pattern, np.float64)
    top = p[r0, q0] * (1 - fc) + p[r0, q0 + 1] * fc
    bot = p[r0 + 1, q0] * (1 - fc) + p[r0 + 1, q0 + 1] * fc
    val = np.where(inb, top * (1 - fr) + bot * fr, 0.0)
    return val, win


def coefficients(tables, pattern, t, frame, mask, flags=FLAG_CENTER | FLAG_NORM, shape=None):
    """spherical.zig:319-361 with sphere.wgsl sphere_sums / rings / legendre / sh_norm.
    Returns (alm complex [pairs], stats (area, mean, norm, a00))."""
    window = (flags & FLAG_WINDOW) != 0
    if window:
        pattern = np.zeros(shape)
    val, win = sample_grid(tables, pattern, t, frame, mask, window=window)
    if window:
        val = win
    g = tables.grid
    wq = g.w[:, None]
    tot_v = float((val * win * wq).sum())
    tot_w = float((win * wq).sum())
    mean = tot_v / max(tot_w, 1e-20) if flags & FLAG_CENTER else 0.0
    samples = (val - mean) * win
    alm = g.analyze(samples)
    nrm = math.sqrt(max(sh.power(tables.L, alm), 1e-30))
    if flags & FLAG_NORM:
        alm = alm / nrm
    stats = np.array([tot_w * 2 * math.pi / g.n_phi, mean, nrm, alm[0].real])
    return alm, stats


class PhaseTables:
    """spherical.zig:192-242 — what a phase adds at a bandwidth."""

    def __init__(self, tables, harmonics, fold):
        self.fold = fold
        self.nc = tables.n // fold
        self.mu_max = (tables.L - 1) // fold
        self.mc = 2 * self.mu_max + 1
        self.l_step = 2 if harmonics.rules.inversion else 1
        self.f = harmonics.f
        self.f2 = harmonics.f2
        self.nb = tables.n // 2 + 1


def _wigner_blocks(tables):
    """d^l_{k,x}(π/2) for signed k, x in [−l, l], one (2l+1)² block per degree l, kept on the tables
    (sh.zig:296-302 element by element, as correlation_volume reads them)."""
    blocks = getattr(tables, "_blocks", None)
    if blocks is None:
        tab = tables.wigner
        blocks = []
        for l in range(tables.L):
            ks = range(-l, l + 1)
            blocks.append(np.array([[sh.d_half_pi(tab, l, k, x) for x in ks] for k in ks]))
        tables._blocks = blocks
    return blocks


def correlation_volume(tables, ph, f, g):
    """so3.wgsl:1-43 — C[j, iq, ia] = Σ T[k,m',m] e^{−i(k b_j + m' a + m c)} on the Euler grid
    (b_j = 2πj/n for j ≤ n/2, a = 2π ia/n, c = 2π iq/n), from
    T[k,m',m] = i^{m'−m} Σ_l f_lm conj(g_lm') d^l_{km'}(π/2) d^l_{km}(π/2) over every signed k, m'
    and the master's orders m = fold·μ (sh.zig:352-379)."""
    L, n = tables.L, tables.n
    fold, nc, mu_max = ph.fold, ph.nc, ph.mu_max
    tab = tables.wigner
    A = np.zeros((n, n, nc), np.complex128)
    blocks = _wigner_blocks(tables)
    for l in range(L):
        ks = np.arange(-l, l + 1)
        # d^l_{k, x} for signed k, x in [−l, l] (the same values for every pattern: built once)
        D = blocks[l]
        gl = np.array([sh.signed_coef(L, g, l, int(x)) for x in ks])
        mus = [mu for mu in range(-mu_max, mu_max + 1) if abs(mu * fold) <= l]
        for mu in mus:
            m = mu * fold
            fl = sh.signed_coef(L, f, l, m)
            if fl == 0:
                continue
            dkm = D[:, m + l]  # over k
            # T[k, m'] += f_lm conj(g_lm') d_km' d_km · i^{m' − m}
            ph_mp = np.array([sh.ipow(int(x) - m) for x in ks])
            term = fl * np.conj(gl)[None, :] * D * dkm[:, None] * ph_mp[None, :]
            A[np.ix_(ks % n, ks % n, [mu % nc])] += term[:, :, None]
    # e^{−i k b_j}: axis 0 (k) → j; e^{−i m' a}: axis 1 (m') → ia; e^{−i fold μ c}: axis 2 (μ) → iq
    C = np.fft.fftn(A).real
    # [k→j, m'→ia, μ→iq] → [j ≤ n/2, iq, ia]
    return np.transpose(C[: n // 2 + 1], (0, 2, 1)).copy()


def window_denominators(tables, ph, window_alm, area):
    """spherical.zig:448-464, so3.wgsl:614-626 — 1/sqrt(⟨w,f²⟩ − ⟨w,f⟩²/area), 0 where the
    variance is below 1e-6·area."""
    vf = correlation_volume(tables, ph, ph.f, window_alm)
    vf2 = correlation_volume(tables, ph, ph.f2, window_alm)
    a = max(area, 1e-12)
    v = vf2 - vf * vf / a
    return np.where(v > 1e-6 * a, 1.0 / np.sqrt(np.where(v > 1e-6 * a, v, 1.0)), 0.0)


def vertex(lo, mid, hi):
    """so3.wgsl:689-693"""
    den = lo - 2.0 * mid + hi
    if den >= -1e-12:
        return 0.0
    return min(max(0.5 * (lo - hi) / den, -0.5), 0.5)


def peak(tables, ph, ncc):
    """so3.wgsl:351-394, 631-663, 695-709, 776-796 — the volume's largest value (ties: lowest
    index (j·nc + iq)·n + ia), the parabolic vertex along a, c and (inside) b, and the orientation
    conj(Rz(a)Ry(b)Rz(c)) with w ≥ 0.  Returns (q, v0, (a, b, c), (j, iq, ia))."""
    n, nc = tables.n, ph.nc
    flat = ncc.reshape(-1)
    idx = int(np.argmax(flat))  # first of equal ones
    j, rest = divmod(idx, nc * n)
    iq, ia = divmod(rest, n)
    v0 = flat[idx]
    da = vertex(ncc[j, iq, (ia - 1) % n], v0, ncc[j, iq, (ia + 1) % n])
    dc = vertex(ncc[j, (iq - 1) % nc, ia], v0, ncc[j, (iq + 1) % nc, ia])
    dj = 0.0
    if 0 < j < n // 2:
        dj = vertex(ncc[j - 1, iq, ia], v0, ncc[j + 1, iq, ia])
    step = 2 * math.pi / n
    a = (ia + da) * step
    b = (j + dj) * step
    c = (iq + dc) * step
    q = rot.qconj(rot.from_zyz(a, b, c))
    if q[0] < 0:
        q = -q
    return q, float(v0), (a, b, c), (j, iq, ia)
