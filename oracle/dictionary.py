"""Dictionary indexing in float64 (oracle restatement; test infrastructure only): the cubochoric
orientation grid of `src/rot.zig`, the dictionary of `Engine.prepareDictionary`
(`src/engine.zig:1851-1899`) with Zig's standard generator for its shuffle, the simulated and
normalized entries (`shaders/detector.wgsl` project_dict 266-273, sim_norm 662-699), the best
entry per pattern (dict_score 705-740, pca.wgsl nearest 114-168) and Oja's rule with the
Cholesky re-orthonormalization (`src/pca.zig:70-162`, `shaders/pca.wgsl`).

The shuffle follows Zig 0.16's `std.Random.DefaultPrng` (xoshiro256++ seeded through SplitMix64,
Blackman & Vigna) and `Random.uintLessThan` (Lemire's multiply-and-reject with O'Neill's
threshold), restated from those published algorithms.  Oja's starting basis in the reference is
`floatNorm` (Zig's ziggurat) draws from seed 0x7a6562; here the starting basis is an argument.
"""
import math

import numpy as np

from . import detector as od
from . import rot

CUBOCHORIC_HALF_EDGE = 1.0725146985555481  # rot.zig:212, (π^(2/3))/2
MASK64 = (1 << 64) - 1


def cu_to_ho(cu):
    """rot.zig:219-266 — cubochoric → homochoric (Roşca, Morawiec & De Graef 2014)."""
    pi = math.pi
    ax = [abs(c) for c in cu]
    if max(ax) == 0:
        return (0.0, 0.0, 0.0)
    p = (0, 1, 2)
    if ax[0] >= ax[1] and ax[0] >= ax[2]:
        p = (1, 2, 0)
    elif ax[1] >= ax[0] and ax[1] >= ax[2]:
        p = (2, 0, 1)
    sc = pi ** (1.0 / 6.0) / 6.0 ** (1.0 / 6.0)
    x, y, z = cu[p[0]] * sc, cu[p[1]] * sc, cu[p[2]] * sc
    pref = math.sqrt(6.0 / pi)
    h = [0.0, 0.0, 0.0]
    if x == 0 and y == 0:
        h[p[2]] = pref * z
        return tuple(h)
    sq2 = math.sqrt(2.0)
    beta = 0.5 * pi ** (5.0 / 6.0) / 6.0 ** (1.0 / 6.0)
    prek = (3.0 * pi / 4.0) ** (1.0 / 3.0) * 2.0 ** 0.25 / beta
    if abs(y) <= abs(x):
        q = (pi / 12.0) * y / x
        k = prek * x / math.sqrt(sq2 - math.cos(q))
        t1 = (sq2 * math.cos(q) - 1) * k
        t2 = sq2 * math.sin(q) * k
    else:
        q = (pi / 12.0) * x / y
        k = prek * y / math.sqrt(sq2 - math.cos(q))
        t1 = sq2 * math.sin(q) * k
        t2 = (sq2 * math.cos(q) - 1) * k
    c = t1 * t1 + t2 * t2
    s = math.sqrt(max(0.0, 1.0 - pi * c / (24.0 * z * z)))
    h[p[0]] = t1 * s
    h[p[1]] = t2 * s
    h[p[2]] = pref * z - math.sqrt(pi) * c / (math.sqrt(24.0) * z)
    return tuple(h)


def from_homochoric(h):
    """rot.zig:269-285 — |h|³ = (3/4)(θ − sin θ), solved by Newton from θ = 2|h|."""
    r = math.sqrt(sum(c * c for c in h))
    if r < 1e-12:
        return (1.0, 0.0, 0.0, 0.0)
    target = r ** 3
    th = min(math.pi, 2.0 * r)
    for _ in range(50):
        d = 0.75 * (1 - math.cos(th))
        if d < 1e-300:
            break
        step = (0.75 * (th - math.sin(th)) - target) / d
        th = min(max(th - step, 0.0), math.pi)
        if abs(step) < 1e-15:
            break
    s = math.sin(0.5 * th) / r
    return (math.cos(0.5 * th), h[0] * s, h[1] * s, h[2] * s)


def from_cubochoric(cu):
    """rot.zig:215-217"""
    return from_homochoric(cu_to_ho(cu))


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & MASK64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)


def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & MASK64


class Xoshiro256:
    """xoshiro256++, the state filled by four SplitMix64 outputs of the seed."""

    def __init__(self, seed):
        g = SplitMix64(seed)
        self.s = [g.next() for _ in range(4)]

    def next(self):
        s = self.s
        r = (_rotl((s[0] + s[3]) & MASK64, 23) + s[0]) & MASK64
        t = (s[1] << 17) & MASK64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        return r

    def uint_less_than(self, n):
        """A uniform integer in [0, n): the high word of x·n, rejecting the low words below
        2^64 mod n."""
        x = self.next()
        m = x * n
        lo = m & MASK64
        if lo < n:
            t = (-n) & MASK64
            if t >= n:
                t -= n
                if t >= n:
                    t %= n
            while lo < t:
                x = self.next()
                m = x * n
                lo = m & MASK64
        return m >> 64


def dictionary(N, rotations):
    """engine.zig:1851-1899 — the points a·(i, j, k)/N of the cubochoric cube (i, j, k in [−N, N],
    a the half edge) whose standard quaternion q is its own fundamental-zone representative
    (|g·q|.w ≤ q.w + 1e-9 for every rotation g but the first, the identity), in that raster order,
    then shuffled by the generator seeded 0x64696374; f32 [M][4]."""
    ops = [np.asarray(g, np.float64) for g in rotations]
    out = []
    a = CUBOCHORIC_HALF_EDGE
    for i in range(-N, N + 1):
        for j in range(-N, N + 1):
            for k in range(-N, N + 1):
                q = rot.qstd(np.array(from_cubochoric((a * i / N, a * j / N, a * k / N))))
                if all(abs(rot.qmul(g, q)[0]) <= q[0] + 1e-9 for g in ops[1:]):
                    out.append(q.astype(np.float32))
    d = np.array(out, np.float32).reshape(-1, 4)
    g = Xoshiro256(0x64696374)
    left = len(d)
    while left > 1:
        j = g.uint_less_than(left)
        d[[left - 1, j]] = d[[j, left - 1]]
        left -= 1
    return d


def sims(sheets, side, frame, t0, dict_q, h, w, mask):
    """detector.wgsl project_dict + sim_norm — every entry at position t0: zero mean and unit
    norm under the mask, zero outside [M][h·w]."""
    m = od.in_mask(h, w, mask).reshape(-1)
    out = np.zeros((len(dict_q), h * w))
    for e, q in enumerate(np.asarray(dict_q, np.float64)):
        v = od.project(sheets, side, frame, t0, q, h, w).reshape(-1)
        v = np.where(m, v - v[m].mean(), 0.0)
        out[e] = v / math.sqrt(max((v * v).sum(), 1e-30))
    return out


def best(x, d):
    """dict_score / nearest — per row of x the row of d with the largest inner product, ties to
    the lower index: (index [n], score [n])."""
    s = np.asarray(x, np.float64) @ np.asarray(d, np.float64).T
    i = np.argmax(s, 1)  # the first maximum
    return i, s[np.arange(len(i)), i]


def orthonormalize(w2):
    """pca.zig:88-136 — the rows of W2 made orthonormal: W2 W2ᵀ = L Lᵀ (Cholesky, the diagonal
    lifted by a jitter while a pivot is at most 1e-12·trace/k), W = L⁻¹ W2."""
    w2 = np.asarray(w2, np.float64)
    k = w2.shape[0]
    G = w2 @ w2.T
    trace = float(np.trace(G))
    jitter = 0.0
    while True:
        L = np.zeros((k, k))
        ok = True
        for i in range(k):
            for j in range(i + 1):
                s = G[i, j] + (jitter if i == j else 0.0) - float(L[i, :j] @ L[j, :j])
                if i == j:
                    if not s > 1e-12 * trace / k:
                        jitter = 1e-6 * trace / k if jitter == 0 else jitter * 10
                        if jitter > trace:
                            raise ValueError("PcaBasisDegenerate")
                        ok = False
                        break
                    L[i, i] = math.sqrt(s)
                else:
                    L[i, j] = s / L[j, j]
            if not ok:
                break
        if ok:
            break
    return np.linalg.solve(L, w2)


def oja_step(W, X, step):
    """pca.zig:140-155 — W ← orthonormalize(W + η/n · (X Wᵀ)ᵀ X), η = 16k / (1 + step/8)."""
    W = np.asarray(W, np.float64)
    X = np.asarray(X, np.float64)
    k, n = W.shape[0], X.shape[0]
    eta = 16.0 * k / (1.0 + step / 8.0)
    Y = X @ W.T
    return orthonormalize(W + (eta / n) * (Y.T @ X))


def learn(W0, X, epochs, chunk):
    """engine.zig:1917-1934 — `epochs` passes of Oja's rule over the dictionary's rows X in steps
    of `chunk` rows, a tail shorter than half a chunk skipped; η counts the steps taken
    (pca.zig:148-153)."""
    W = orthonormalize(W0)
    total = X.shape[0]
    taken = 0
    for _ in range(epochs):
        for d0 in range(0, total, chunk):
            nb = min(chunk, total - d0)
            if nb < chunk // 2 and d0 != 0:
                continue
            W = oja_step(W, X[d0:d0 + nb], taken)
            taken += 1
    return W
