"""Dictionary indexing (settings `method` "dictionary" and "pca"): each pattern matched against the
simulated patterns of a grid of orientations, or against their leading principal components, and
the best entry refined on the detector like a spherical peak.

The dictionary (Engine.prepareDictionary, engine.zig:1851-1899): the points a·(i, j, k)/N of the
cubochoric cube (rot.zig:212-285) whose orientation is its own fundamental-zone representative,
shuffled by Zig's default generator seeded 0x64696374 (xoshiro256++ through SplitMix64, the
index drawn by Lemire's multiply-and-reject), so that the entries and their order are the
reference's.

On the device the entries are simulated once at the map's reference detector position and kept
(FP32 rows, and BF16 panels for the tensor cores) until the master, the geometry or the grid
changes; the reference simulates them again for every batch.  "pca" learns k components by
Oja's rule as the dictionary streams by (pca.zig:70-162; the GEMMs of a learning step in FP32
through cuBLAS, the k × k Cholesky factor in FP64 on the host, as the reference) and keeps every
entry's k coefficients.  A batch is then scored by zeb_match_bf16 (BF16 tensor cores, each
pattern's eight best) and rescored in FP32 by zeb_match_best, or by zeb_match_f32 in the plain
FP32 form.
"""
import ctypes
import math

import numpy as np
import torch

from . import _native as N
from .device import ptr, stream_ptr

CUBOCHORIC_HALF_EDGE = 1.0725146985555481  # rot.zig:212
_M64 = (1 << 64) - 1


# ── the grid ──

def cu_to_ho(cu):
    """rot.zig:219-266 — cubochoric → homochoric for rows of cu [M, 3] (Roşca, Morawiec & De
    Graef 2014: the cube's six pyramids, each square → curved square → Lambert → ball)."""
    cu = np.asarray(cu, np.float64)
    pi = math.pi
    ax = np.abs(cu)
    px = (ax[:, 0] >= ax[:, 1]) & (ax[:, 0] >= ax[:, 2])
    py = ~px & (ax[:, 1] >= ax[:, 0]) & (ax[:, 1] >= ax[:, 2])
    perm = np.where(px[:, None], [1, 2, 0], np.where(py[:, None], [2, 0, 1], [0, 1, 2]))
    rows = np.arange(len(cu))[:, None]
    sc = pi ** (1.0 / 6.0) / 6.0 ** (1.0 / 6.0)
    x, y, z = (cu[rows[:, 0], perm[:, i]] * sc for i in range(3))
    pref = math.sqrt(6.0 / pi)
    sq2 = math.sqrt(2.0)
    beta = 0.5 * pi ** (5.0 / 6.0) / 6.0 ** (1.0 / 6.0)
    prek = (3.0 * pi / 4.0) ** (1.0 / 3.0) * 2.0 ** 0.25 / beta
    axis = (x == 0) & (y == 0)
    xs = np.where(axis, 1.0, x)
    ys = np.where(axis, 1.0, y)
    zs = np.where(axis | (z == 0), 1.0, z)
    first = np.abs(ys) <= np.abs(xs)
    with np.errstate(divide="ignore", invalid="ignore"):
        q = np.where(first, (pi / 12.0) * ys / xs, (pi / 12.0) * xs / ys)
        k = prek * np.where(first, xs, ys) / np.sqrt(sq2 - np.cos(q))
    t1 = np.where(first, (sq2 * np.cos(q) - 1) * k, sq2 * np.sin(q) * k)
    t2 = np.where(first, sq2 * np.sin(q) * k, (sq2 * np.cos(q) - 1) * k)
    c = t1 * t1 + t2 * t2
    s = np.sqrt(np.maximum(0.0, 1.0 - pi * c / (24.0 * zs * zs)))
    h0 = np.where(axis, 0.0, t1 * s)
    h1 = np.where(axis, 0.0, t2 * s)
    h2 = np.where(axis, pref * z, pref * z - math.sqrt(pi) * c / (math.sqrt(24.0) * zs))
    h = np.zeros_like(cu)
    h[rows[:, 0], perm[:, 0]] = h0
    h[rows[:, 0], perm[:, 1]] = h1
    h[rows[:, 0], perm[:, 2]] = h2
    h[ax.max(1) == 0] = 0.0
    return h


def from_homochoric(h):
    """rot.zig:269-285 — |h|³ = (3/4)(θ − sin θ) by Newton from θ = 2|h|, each row stopping
    where the scalar iteration would."""
    h = np.asarray(h, np.float64)
    r = np.sqrt((h * h).sum(1))
    target = r ** 3
    th = np.minimum(math.pi, 2.0 * r)
    idx = np.flatnonzero(r >= 1e-12)  # the rows still iterating
    for _ in range(50):
        if idx.size == 0:
            break
        t = th[idx]
        d = 0.75 * (1 - np.cos(t))
        ok = d >= 1e-300
        idx, t, d = idx[ok], t[ok], d[ok]
        step = (0.75 * (t - np.sin(t)) - target[idx]) / d
        th[idx] = np.minimum(np.maximum(t - step, 0.0), math.pi)
        idx = idx[np.abs(step) >= 1e-15]
    small = r < 1e-12
    s = np.sin(0.5 * th) / np.where(small, 1.0, r)
    q = np.concatenate([np.cos(0.5 * th)[:, None], h * s[:, None]], 1)
    q[small] = (1.0, 0.0, 0.0, 0.0)
    return q


def _splitmix(seed):
    s = seed & _M64
    while True:
        s = (s + 0x9E3779B97F4A7C15) & _M64
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        yield z ^ (z >> 31)


def shuffle_order(n, seed):
    """The permutation Zig's `Random.shuffle`-style loop of engine.zig:1886-1896 applies: for
    left = n … 2, swap entries left − 1 and uintLessThan(left) of xoshiro256++ (seeded by four
    SplitMix64 outputs of `seed`). Returns perm with out[i] = in[perm[i]]."""
    g = _splitmix(seed)
    s0, s1, s2, s3 = (next(g) for _ in range(4))
    perm = list(range(n))
    left = n
    while left > 1:
        while True:  # uintLessThan(left): the high word of x·left, low words below 2^64 mod left redrawn
            u = (s0 + s3) & _M64
            r = ((((u << 23) | (u >> 41)) & _M64) + s0) & _M64
            t = (s1 << 17) & _M64
            s2 ^= s0
            s3 ^= s1
            s1 ^= s2
            s0 ^= s3
            s2 ^= t
            s3 = ((s3 << 45) | (s3 >> 19)) & _M64
            m = r * left
            lo = m & _M64
            if lo >= left:
                break
            th = (-left) & _M64
            if th >= left:
                th -= left
                if th >= left:
                    th %= left
            if lo >= th:
                break
        j = m >> 64
        perm[left - 1], perm[j] = perm[j], perm[left - 1]
        left -= 1
    return np.asarray(perm, np.int64)


def cubochoric_grid(N, rotations):
    """engine.zig:1851-1899 — the dictionary of grid N for a master with these rotations
    (quaternions, the identity first): f32 [M, 4] in the reference's order."""
    r = np.arange(-N, N + 1, dtype=np.float64) * (CUBOCHORIC_HALF_EDGE / N)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    cu = np.stack([i.reshape(-1), j.reshape(-1), k.reshape(-1)], 1)
    q = from_homochoric(cu_to_ho(cu))
    n = np.sqrt((q * q).sum(1, keepdims=True))
    q = q / np.where(n == 0, 1.0, n) * np.where(q[:, :1] < 0, -1.0, 1.0)
    idx = np.arange(len(q))
    for g in rotations[1:]:  # (g·q).w, the rows still in the zone only
        g = np.asarray(g, np.float64)
        p = q[idx]
        w = g[0] * p[:, 0] - g[1] * p[:, 1] - g[2] * p[:, 2] - g[3] * p[:, 3]
        idx = idx[np.abs(w) <= p[:, 0] + 1e-9]
    d = q[idx].astype(np.float32)
    return d[shuffle_order(len(d), 0x64696374)]


# ── the device side ──

def simulate(fr, vpair, side, t0, q, out):
    """zeb_dict_sims of the entries q (device f32 [n, 4]) into out [n, h·w]."""
    t = (ctypes.c_float * 3)(*[float(v) for v in t0])
    N.call("zeb_dict_sims", ctypes.byref(fr), ptr(vpair), side, t, ptr(q), q.shape[0], ptr(out), stream_ptr())
    return out


def panel(rows):
    """The BF16 operand panel of FP32 rows [n, cols] (zeb_pack_panel)."""
    n, cols = rows.shape
    p = torch.empty(N.load().zeb_panel_bytes(n, cols), dtype=torch.uint8, device=rows.device)
    N.call("zeb_pack_panel", ptr(rows), n, cols, rows.stride(0), ptr(p), stream_ptr())
    return p


def _orthonormalize(w2):
    """pca.zig:88-136 — the rows of W2 made orthonormal: the Gram matrix (FP32 on the device),
    its Cholesky factor in FP64 on the host (the diagonal lifted by a jitter while a pivot is at
    most 1e-12·trace/k), W = L⁻¹ W2 on the device."""
    k = w2.shape[0]
    G = (w2 @ w2.T).double().cpu().numpy()
    trace = float(np.trace(G))
    floor = 1e-12 * trace / k  # a pivot L[i][i]² at or below this counts as a dependent row
    jitter = 0.0
    while True:
        try:
            L = np.linalg.cholesky(G + jitter * np.eye(k))
            ok = bool(np.all(np.diag(L) ** 2 > floor))
        except np.linalg.LinAlgError:
            ok = False
        if ok:
            break
        jitter = 1e-6 * trace / k if jitter == 0 else jitter * 10
        if jitter > trace:
            raise RuntimeError("PcaBasisDegenerate")
    inv = np.tril(np.linalg.inv(L))
    return torch.as_tensor(inv, dtype=torch.float32, device=w2.device) @ w2


class Dictionary:
    """One phase's dictionary at one grid on the device: the entries' quaternions, and per use the
    simulated rows (method "dictionary") or the learned components and coefficients ("pca")."""

    def __init__(self, q_host, device):
        self.q_host = q_host
        self.q = torch.as_tensor(q_host, device=device).contiguous()
        self.n = len(q_host)
        self.key = None
        self.rows = None     # FP32 rows the patterns are scored against: sims [n][h·w] or coefficients [n][k]
        self.panel = None    # their BF16 panel (tensor-core forms)
        self.W = None        # PCA components [k][h·w]
        self.w_split = None  # the components as a split BF16 panel (the BF16 form's projection)
        self.kept = None

    def chunk(self, px):
        """Entries per learning step: about 64 MiB of simulated patterns (engine.zig:1917-1918)."""
        return min(self.n, max(256, min(4096, (64 << 20) // (px * 4))))

    def prepare_sims(self, fr, vpair, side, t0):
        px = fr.h * fr.w
        rows = torch.empty(self.n, px, dtype=torch.float32, device=self.q.device)
        step = max(1, (1 << 30) // (px * 4))
        for d0 in range(0, self.n, step):
            simulate(fr, vpair, side, t0, self.q[d0:d0 + step], rows[d0:d0 + step])
        self.rows, self.W, self.w_split = rows, None, None

    def prepare_pca(self, fr, vpair, side, t0, k, epochs, log=None):
        """engine.zig:1905-1955 — components by Oja's rule over `epochs` passes (steps of chunk()
        entries, a tail under half a chunk skipped), then every entry's coefficients."""
        px = fr.h * fr.w
        dev = self.q.device
        k = min(k, px, self.n)
        gen = torch.Generator().manual_seed(0x7A6562)
        W = _orthonormalize(torch.randn(k, px, generator=gen, dtype=torch.float32).to(dev))
        chunk = self.chunk(px)
        X = torch.empty(chunk, px, dtype=torch.float32, device=dev)
        taken = 0
        for _ in range(epochs):
            for d0 in range(0, self.n, chunk):
                nb = min(chunk, self.n - d0)
                if nb < chunk // 2 and d0 != 0:
                    continue  # a short tail is no sample: it would pull the basis toward its few patterns
                x = simulate(fr, vpair, side, t0, self.q[d0:d0 + nb], X[:nb])
                eta = 16.0 * k / (1.0 + taken / 8.0)
                Y = x @ W.T
                W = _orthonormalize(torch.addmm(W, Y.T, x, alpha=float(np.float32(eta / nb))))
                taken += 1
        coef = torch.empty(self.n, k, dtype=torch.float32, device=dev)
        for d0 in range(0, self.n, chunk):
            nb = min(chunk, self.n - d0)
            x = simulate(fr, vpair, side, t0, self.q[d0:d0 + nb], X[:nb])
            torch.mm(x, W.T, out=coef[d0:d0 + nb])
        head = coef[: min(self.n, 2048)]
        self.kept = float((head.double() ** 2).sum() / head.shape[0])
        self.rows, self.W, self.w_split = coef, W, None
        if log:
            log(f"dictionary components: {k} of {px} pixels hold {100 * self.kept:.1f} % of {self.n} patterns' "
                f"variance ({taken} steps of Oja's rule)")

    def project(self, x, tensor_cores, status):
        """pca.zig:159-162 — the batch's coefficients on the components, x [n, h·w] → [n, k]: on the
        tcgen05 tensor cores from split BF16 panels (near FP32; zeb_project_bf16) or in plain FP32
        (zeb_project_f32)."""
        n, px = x.shape
        x, w = x.contiguous(), self.W.contiguous()
        k = w.shape[0]
        out = torch.empty(n, k, dtype=torch.float32, device=x.device)
        if tensor_cores:
            if self.w_split is None:
                self.w_split = torch.empty(N.load().zeb_panel_split_bytes(k, px), dtype=torch.uint8, device=x.device)
                N.call("zeb_pack_panel_split", ptr(w), k, px, px, 1, ptr(self.w_split), stream_ptr())
            xs = torch.empty(N.load().zeb_panel_split_bytes(n, px), dtype=torch.uint8, device=x.device)
            N.call("zeb_pack_panel_split", ptr(x), n, px, px, 0, ptr(xs), stream_ptr())
            N.call("zeb_project_bf16", ptr(xs), n, ptr(self.w_split), k, px, ptr(out), ptr(status), stream_ptr())
        else:
            N.call("zeb_project_f32", ptr(x), n, ptr(w), k, px, ptr(out), stream_ptr())
        return out

    def seeds(self, x, tensor_cores, status, out):
        """The best entry for each row of x [n, K] (patterns or their coefficients) as seeds
        out [n, 8] = (q, score, index, 0, 0)."""
        n, K = x.shape
        dev = x.device
        if tensor_cores:
            if self.panel is None:
                self.panel = panel(self.rows)
            xp = panel(x)
            sl = N.load().zeb_match_slices(n, self.n, K, 1)
            cv = torch.empty(n * sl * 8, dtype=torch.float32, device=dev)
            ci = torch.empty(n * sl * 8, dtype=torch.int32, device=dev)
            N.call("zeb_match_bf16", ptr(xp), n, ptr(self.panel), self.n, K, sl, ptr(cv), ptr(ci), ptr(status),
                   stream_ptr())
            nc = sl * 8
        else:
            sl = N.load().zeb_match_slices(n, self.n, K, 0)
            cv = torch.empty(n * sl, dtype=torch.float32, device=dev)
            ci = torch.empty(n * sl, dtype=torch.int32, device=dev)
            N.call("zeb_match_f32", ptr(x), n, ptr(self.rows), self.n, K, sl, ptr(cv), ptr(ci), stream_ptr())
            nc = sl
        N.call("zeb_match_best", ptr(x), n, ptr(self.rows), self.n, K, ptr(ci), nc, ptr(self.q), ptr(out),
               stream_ptr())
        return out
