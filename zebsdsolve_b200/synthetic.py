"""Seeded synthetic inputs of the benchmark workloads: master patterns and scans.

Master: a real band-limited function on the sphere (SH degree ≤ lmax, Gaussian coefficients of
variance ∝ (1+l)⁻²), averaged over the proper rotations of a point group (432 or 622), sampled in
FP32 at every pixel of a side × side square-Lambert grid per hemisphere and normalized to zero
mean and unit variance.  The average is taken in SH space: each group element's Wigner D
(d(β) from the factorization through d(π/2)) applied to the coefficients.

Scan: orientations (uniform, or Voronoi grains with a Gaussian spread), patterns simulated by the
engine's own projection kernel from the master as the engine smooths it, intensity
1000·(0.6 + 0.4·m)·B with B a 2-D Gaussian background (σ = 0.4 of the width, mean 1), Poisson
counts, stored as uint16.
"""
import math

import numpy as np
import torch

from . import rotations as R
from .master import square_to_sphere


def wigner_half_pi(L):
    """d^l_{k,m}(π/2) at [k, m, l], the Jacobi three-term recursion vectorised over m."""
    d = np.zeros((L, L, L))
    lf = np.concatenate([[0.0], np.cumsum(np.log(np.arange(1, 2 * L + 2)))])
    for k in range(L):
        m = np.arange(k + 1)
        a, b = (k - m).astype(np.float64), (k + m).astype(np.float64)
        p2 = np.zeros(k + 1)
        p1 = np.zeros(k + 1)
        for nn in range(L - k):
            if nn == 0:
                p = np.ones(k + 1)
            elif nn == 1:
                p = (a - b) / 2
            else:
                c = 2 * nn + a + b
                p = ((c - 1) * (a * a - b * b) * p1 - 2 * (nn + a - 1) * (nn + b - 1) * c * p2) / (2 * nn * (nn + a + b) * (c - 2))
            j = nn + k
            v = np.exp(0.5 * (lf[nn + 2 * k] + lf[nn] - lf[j + m] - lf[j - m])) * 2.0 ** (-k) * p
            d[m, k, j] = v
            d[k, m, j] = np.where((k - m) % 2 == 0, v, -v)
            p2, p1 = p1, p
    return d


def _d_signed(tab, l):
    """d^l_{k,m}(π/2) for signed k, m ∈ [−l, l] (sh.zig:283-302)."""
    ks = np.arange(-l, l + 1)
    K, Mm = np.meshgrid(ks, ks, indexing="ij")
    base = tab[np.abs(K), np.abs(Mm), l]
    sgn = np.ones_like(base)
    both = (K < 0) & (Mm < 0)
    sgn = np.where(both, np.where((K - Mm) % 2 == 1, -1.0, 1.0), sgn)
    sgn = np.where(~both & (Mm < 0), np.where((l + K) % 2 == 1, -1.0, 1.0), sgn)
    sgn = np.where(~both & (K < 0) & (Mm >= 0), np.where((l + Mm) % 2 == 1, -1.0, 1.0), sgn)
    return base * sgn


def _zyz(q):
    """(a, b, c) with q = Rz(a) Ry(b) Rz(c)."""
    w, x, y, z = q
    b = 2 * math.atan2(math.hypot(x, y), math.hypot(w, z))
    s = math.atan2(z, w)
    dd = math.atan2(-x, y)
    return s + dd, b, s - dd


def symmetrize(coef, lmax, ops):
    """(1/|G|) Σ_g f(g⁻¹ x) in SH space: coefficients [l][m ≥ 0] complex."""
    tab = wigner_half_pi(lmax + 1)
    out = np.zeros_like(coef)
    angles = [_zyz(np.asarray(g, np.float64)) for g in ops]
    for l in range(lmax + 1):
        ms = np.arange(-l, l + 1)
        dh = _d_signed(tab, l)  # [k, m]
        a_signed = np.where(ms >= 0, coef[l, np.abs(ms)], ((-1.0) ** np.abs(ms)) * np.conj(coef[l, np.abs(ms)]))
        acc = np.zeros(2 * l + 1, np.complex128)
        for a, b, c in angles:
            # d^l_{m'm}(b) = i^{m'−m} Σ_k d_{km'} d_{km} e^{−ikb}
            e = np.exp(-1j * ms * b)
            dbeta = (dh * e[:, None]).T @ dh  # [m', m] before the phase
            ph = (1j) ** ((ms[:, None] - ms[None, :]) % 4)
            D = np.exp(-1j * ms[:, None] * a) * (ph * dbeta) * np.exp(-1j * ms[None, :] * c)
            acc += D @ a_signed
        out[l, : l + 1] = acc[l:] / len(ops)
    return out


def synthesize_at(coef, lmax, dirs, device="cpu"):
    """f(x) = Σ_l [a_l0 P̄_l^0 + 2 Re Σ_{m>0} a_lm P̄_l^m e^{imφ}] at unit vectors dirs [n, 3]."""
    dv = torch.as_tensor(dirs, dtype=torch.float64, device=device)
    x = dv[:, 2].clamp(-1, 1)
    phi = torch.atan2(dv[:, 1], dv[:, 0])
    s = torch.sqrt(torch.clamp(1 - x * x, min=0.0))
    cf = torch.as_tensor(coef, dtype=torch.complex128, device=device)
    out = torch.zeros_like(x)
    pmm = torch.full_like(x, math.sqrt(1.0 / (4 * math.pi)))
    for m in range(lmax + 1):
        if m > 0:
            pmm = pmm * (-math.sqrt((2 * m + 1) / (2 * m))) * s
        acc = cf[m, m] * pmm
        p2, p1 = pmm, None
        if m + 1 <= lmax:
            p1 = math.sqrt(2 * m + 3) * x * pmm
            acc = acc + cf[m + 1, m] * p1
        for l in range(m + 2, lmax + 1):
            a = math.sqrt((4 * l * l - 1) / (l * l - m * m))
            bb = math.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
            p = a * (x * p1 - bb * p2)
            acc = acc + cf[l, m] * p
            p2, p1 = p1, p
        k = 1.0 if m == 0 else 2.0
        out += k * (acc * torch.exp(1j * m * phi)).real
    return out.cpu().numpy()


def master_sheets(seed, side=401, lmax=96, group="432", device="cpu"):
    """Normalized Lambert sheets (2, side, side) float32 of the seeded symmetrized master."""
    rng = np.random.default_rng(seed)
    coef = np.zeros((lmax + 1, lmax + 1), np.complex128)  # [l, m]
    for l in range(lmax + 1):
        sd = 1.0 / (1 + l)
        coef[l, 0] = rng.normal(0, sd)
        if l > 0:
            coef[l, 1:l + 1] = rng.normal(0, sd / math.sqrt(2), l) + 1j * rng.normal(0, sd / math.sqrt(2), l)
    ops = R.group({"432": "o", "622": "d6", "1": "c1"}[group])
    coef = symmetrize(coef, lmax, ops)
    last = side - 1.0
    rr, cc = np.divmod(np.arange(side * side), side)
    xs, ys = 2 * cc / last - 1, 2 * rr / last - 1
    dirs = np.concatenate([square_to_sphere(xs, ys, False), square_to_sphere(xs, ys, True)])
    vals = synthesize_at(coef, lmax, dirs, device).astype(np.float32)
    v = vals.astype(np.float64)
    v = (v - v.mean()) / v.std()
    return v.astype(np.float32).reshape(2, side, side)


def group_matrices(group):
    """The point group's proper rotations as 3 × 3 matrices, identity first."""
    return np.stack([R.to_matrix(q) for q in R.group({"432": "o", "622": "d6", "1": "c1"}[group])])


POINT_GROUP = {"432": 30, "622": 24, "1": 1}


def uniform_quaternions(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1
    return q


def grain_map(rng, rows, cols, n_grains, spread_deg):
    """Voronoi grains of n_grains uniform seeds, each a uniform orientation, every cell rotated
    from its grain's by a Gaussian rotation of RMS angle spread_deg.  Returns (quats, grain)."""
    seeds = rng.random((n_grains, 2)) * np.array([rows, cols])
    gq = uniform_quaternions(rng, n_grains)
    r, c = np.divmod(np.arange(rows * cols), cols)
    pts = np.stack([r + 0.5, c + 0.5], 1)
    grain = np.empty(rows * cols, np.int64)
    for i in range(0, len(pts), 65536):
        d = ((pts[i:i + 65536, None, :] - seeds[None]) ** 2).sum(-1)
        grain[i:i + 65536] = d.argmin(1)
    q = gq[grain]
    if spread_deg > 0:
        phi = rng.normal(0, math.radians(spread_deg) / math.sqrt(3), (rows * cols, 3))
        q = R.qstd(R.qmul(R.exp_map(phi), q))
    return q, grain


def counted_patterns(sims, seed, counts=1000.0, device="cuda"):
    """uint16 patterns from simulations [n, h, w] (the master's values): Poisson counts of
    counts·(0.6 + 0.4·m)·B, B a Gaussian background of σ = 0.4 of the width with mean 1."""
    n, h, w = sims.shape
    yy, xx = torch.meshgrid(torch.arange(h, dtype=torch.float32, device=device) + 0.5 - 0.5 * h,
                            torch.arange(w, dtype=torch.float32, device=device) + 0.5 - 0.5 * w, indexing="ij")
    sg = 0.4 * w
    B = torch.exp(-(xx * xx + yy * yy) / (2 * sg * sg))
    B = B * (h * w) / B.sum()
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    lam = torch.clamp(counts * (0.6 + 0.4 * torch.as_tensor(sims, device=device)) * B, min=0.0)
    return torch.clamp(torch.poisson(lam, generator=g), 0, 65535).to(torch.int32).to(torch.uint16)
