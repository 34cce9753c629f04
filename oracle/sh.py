"""Spherical harmonics in float64 (oracle restatement of zebsdsolve `src/sh.zig`).

Conventions (sh.zig:6-13): Y_lm = P̄_l^m(cos θ) e^{imφ}, orthonormal, Condon–Shortley phase;
coefficients stored for m ≥ 0 at pair(L, m, l) (m-major, l = m … L−1); a Gauss–Legendre grid
has nθ rings (θ ascending) of nφ points φ_j = 2πj/nφ; D^l_{m'm}(a,b,c) = e^{−im'a} d^l_{m'm}(b)
e^{−imc} for S = Rz(a) Ry(b) Rz(c).
"""
import math

import numpy as np


def pair_count(L):
    """sh.zig:21-23"""
    return L * (L + 1) // 2


def pair(L, m, l):
    """sh.zig:26-28 — index of (m, l), 0 ≤ m ≤ l < L."""
    return m * L - (m * (m - 1)) // 2 + (l - m)


def pair_table(L):
    """(m, l) of every stored pair, in storage order."""
    ms = []
    ls = []
    for m in range(L):
        for l in range(m, L):
            ms.append(m)
            ls.append(l)
    return np.array(ms), np.array(ls)


def gauss_legendre(n):
    """sh.zig:31-72 — nodes x descending (cos θ for θ ascending) and weights on [−1, 1]."""
    x = np.zeros(n)
    w = np.zeros(n)
    nf = float(n)

    def p_and_prev(z):
        p0, p1 = 1.0, z
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * z * p1 - (k - 1) * p0) / k
        return p0, p1

    for i in range((n + 1) // 2):
        z = math.cos(math.pi * (i + 0.75) / (nf + 0.5))
        for _ in range(100):
            p0, p1 = p_and_prev(z)
            dp = nf * (z * p1 - p0) / (z * z - 1)
            dz = p1 / dp
            z -= dz
            if abs(dz) < 1e-16:
                break
        p0, p1 = p_and_prev(z)
        dp = nf * (z * p1 - p0) / (z * z - 1)
        x[i] = z
        x[n - 1 - i] = -z
        w[i] = 2 / ((1 - z * z) * dp * dp)
        w[n - 1 - i] = w[i]
    return x, w


def legendre_all(L, x):
    """sh.zig:75-99 — P̄_l^m(x) for every pair below L; x scalar or array (pairs first axis)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((pair_count(L),) + x.shape)
    s = np.sqrt(np.maximum(0.0, 1 - x * x))
    pmm = np.full(x.shape, math.sqrt(1.0 / (4.0 * math.pi)))
    for m in range(L):
        if m > 0:
            pmm = pmm * (-math.sqrt((2 * m + 1) / (2 * m))) * s
        base = pair(L, m, m)
        out[base] = pmm
        if m + 1 < L:
            out[base + 1] = math.sqrt(2 * m + 3) * x * pmm
        for l in range(m + 2, L):
            a = math.sqrt((4 * l * l - 1) / (l * l - m * m))
            b = math.sqrt(((l - 1) * (l - 1) - m * m) / (4 * (l - 1) * (l - 1) - 1))
            out[base + l - m] = a * (x * out[base + l - m - 1] - b * out[base + l - m - 2])
    return out


class Grid:
    """sh.zig:102-223 — a Gauss–Legendre grid with its Legendre table plm[pair, ring]."""

    def __init__(self, L, n_theta, n_phi):
        self.L = L
        self.n_theta = n_theta
        self.n_phi = n_phi
        self.x, self.w = gauss_legendre(n_theta)
        self.plm = legendre_all(L, self.x)  # [pairs, rings]

    def points(self):
        return self.n_theta * self.n_phi

    def directions(self):
        """sh.zig:138-143 — unit vectors [nθ, nφ, 3]."""
        ct = self.x[:, None]
        st = np.sqrt(np.maximum(0.0, 1 - ct * ct))
        phi = 2.0 * math.pi * np.arange(self.n_phi) / self.n_phi
        return np.stack(np.broadcast_arrays(st * np.cos(phi)[None, :], st * np.sin(phi)[None, :], ct), -1)

    def analyze(self, samples):
        """sh.zig:146-186 — samples [nθ·nφ] → complex coefficients [pairs]."""
        L, nt, nphi = self.L, self.n_theta, self.n_phi
        s = np.asarray(samples, dtype=np.float64).reshape(nt, nphi)
        j = np.arange(nphi)
        m = np.arange(L)
        # F[y][m] = (2π/nφ) Σ_j f e^{−imφ_j}
        ang = 2.0 * math.pi * ((m[:, None] * j[None, :]) % nphi) / nphi
        F = (s @ np.exp(-1j * ang).T) * (2.0 * math.pi / nphi)
        out = np.zeros(pair_count(L), dtype=np.complex128)
        ms, ls = pair_table(L)
        k = self.w[None, :] * self.plm  # [pairs, rings]
        out[:] = np.sum(k * F[:, ms].T, axis=1)
        return out

    def synthesize(self, coef):
        """sh.zig:189-222 — coefficients → samples [nθ·nφ]."""
        L, nt, nphi = self.L, self.n_theta, self.n_phi
        ms, _ = pair_table(L)
        coef = np.asarray(coef, dtype=np.complex128)
        G = np.zeros((nt, L), dtype=np.complex128)
        for m in range(L):
            sel = ms == m
            G[:, m] = (self.plm[sel] * coef[sel][:, None]).sum(0)
        j = np.arange(nphi)
        m = np.arange(1, L)
        ang = 2.0 * math.pi * ((m[:, None] * j[None, :]) % nphi) / nphi
        out = G[:, 0].real[:, None] + 2 * (G[:, 1:].real @ np.cos(ang) - G[:, 1:].imag @ np.sin(ang))
        return out.reshape(-1)


def power(L, coef):
    """sh.zig:226-234 — Σ |a_lm|² over all signed orders."""
    ms, _ = pair_table(L)
    k = np.where(ms == 0, 1.0, 2.0)
    return float(np.sum(k * np.abs(coef) ** 2))


def wigner_half_pi(L):
    """sh.zig:239-280 — d^l_{k,m}(π/2) at [k, m, l] (zero where l < max(k, m)), by the Jacobi
    three-term recursion d^j_{m,k} = 2^{−k} sqrt((j+k)!(j−k)!/((j+m)!(j−m)!)) P_{j−k}^{(k−m,k+m)}(0)."""
    n = L
    d = np.zeros((n, n, n))
    lf = np.zeros(2 * n + 2)
    for i in range(1, lf.size):
        lf[i] = lf[i - 1] + math.log(i)
    for k in range(n):
        for m in range(k + 1):
            a = float(k - m)
            b = float(k + m)
            p2 = 0.0
            p1 = 0.0
            nn = 0
            while nn + k < n:
                if nn == 0:
                    p = 1.0
                elif nn == 1:
                    p = (a - b) / 2
                else:
                    c = 2 * nn + a + b
                    num1 = (c - 1) * (a * a - b * b)
                    num2 = 2 * (nn + a - 1) * (nn + b - 1) * c
                    den = 2 * nn * (nn + a + b) * (c - 2)
                    p = (num1 * p1 - num2 * p2) / den
                j = nn + k
                pref = math.exp(0.5 * (lf[nn + 2 * k] + lf[nn] - lf[j + m] - lf[j - m])) * 2.0 ** (-k)
                v = pref * p
                d[m, k, j] = v
                d[k, m, j] = v if (k - m) % 2 == 0 else -v
                p2 = p1
                p1 = p
                nn += 1
    return d


def d_sign(l, k, m):
    """sh.zig:283-293"""
    if k < 0 and m < 0:
        return -1.0 if (k - m) % 2 else 1.0
    if m < 0:
        return -1.0 if (l + k) % 2 else 1.0
    if k < 0:
        return -1.0 if (l + m) % 2 else 1.0
    return 1.0


def d_half_pi(tab, l, k, m):
    """sh.zig:296-302 — d^l_{k,m}(π/2) for signed k, m."""
    ak, am = abs(k), abs(m)
    if ak > l or am > l:
        return 0.0
    return d_sign(l, k, m) * tab[ak, am, l]


def wigner_small_d(l, mp, m, beta):
    """sh.zig:305-325 — d^l_{m',m}(β) by Wigner's sum (tests, small l)."""
    f = math.factorial
    c = math.cos(0.5 * beta)
    s = math.sin(0.5 * beta)
    pre = math.sqrt(f(l + mp) * f(l - mp) * f(l + m) * f(l - m))
    total = 0.0
    for t in range(max(0, m - mp), min(l + m, l - mp) + 1):
        den = f(l + m - t) * f(t) * f(mp - m + t) * f(l - mp - t)
        sgn = 1.0 if (mp - m + t) % 2 == 0 else -1.0
        total += sgn * c ** (2 * l + m - mp - 2 * t) * s ** (mp - m + 2 * t) / den
    return pre * total


def signed_coef(L, coef, l, m):
    """sh.zig:328-334 — a_{l,m} for signed m from m ≥ 0 storage."""
    am = abs(m)
    if am > l:
        return 0j
    c = coef[pair(L, am, l)]
    if m >= 0:
        return c
    return np.conj(c) if am % 2 == 0 else -np.conj(c)


def ipow(n):
    """sh.zig:341-348 — i^n"""
    return (1, 1j, -1, -1j)[n % 4]


def correlation_at(L, tab, f, g, a, b, c):
    """sh.zig:352-379 — C(a,b,c) = ∫ g(x) f(S⁻¹x) dΩ, S = Rz(a)Ry(b)Rz(c), from the coefficients."""
    total = 0.0
    for k in range(-(L - 1), L):
        for mp in range(-(L - 1), L):
            for m in range(-(L - 1), L):
                t = 0j
                lmin = max(abs(k), abs(mp), abs(m))
                for l in range(lmin, L):
                    fl = signed_coef(L, f, l, m)
                    gl = signed_coef(L, g, l, mp)
                    dd = d_half_pi(tab, l, k, mp) * d_half_pi(tab, l, k, m)
                    t += fl * np.conj(gl) * dd
                t *= ipow(mp - m)
                ang = -(k * b + mp * a + m * c)
                total += t.real * math.cos(ang) - t.imag * math.sin(ang)
    return total


class Rules:
    """sh.zig:383-423 — which coefficients a crystal's symmetry leaves non-zero."""

    def __init__(self, n_fold=1, mirror=False, inversion=False):
        self.n_fold = n_fold
        self.mirror = mirror
        self.inversion = inversion

    def allows(self, l, m):
        if m % self.n_fold != 0:
            return False
        if self.mirror and (l + m) % 2 != 0:
            return False
        if self.inversion and l % 2 != 0:
            return False
        return True

    @staticmethod
    def detect(L, coef, tol):
        total = 0.0
        odd_l = 0.0
        odd_lm = 0.0
        off = {2: 0.0, 3: 0.0, 4: 0.0, 6: 0.0}
        for m in range(L):
            for l in range(m, L):
                if l == 0:
                    continue
                c = coef[pair(L, m, l)]
                e = (1.0 if m == 0 else 2.0) * (c.real * c.real + c.imag * c.imag)
                total += e
                if l % 2:
                    odd_l += e
                if (l + m) % 2:
                    odd_lm += e
                for n in (2, 3, 4, 6):
                    if m % n:
                        off[n] += e
        if total <= 0:
            return Rules()
        r = Rules(inversion=odd_l < tol * total, mirror=odd_lm < tol * total)
        for n in (6, 4, 3, 2):
            if off[n] < tol * total:
                r.n_fold = n
                break
        return r
