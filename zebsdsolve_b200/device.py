"""Device-side tables and buffers of the indexing path (torch tensors for the memory; the C ABI
for every computation).

BandTables: what depends on the bandwidth L only (spherical.zig Tables.init, :119-180) — the
Gauss–Legendre rings, the weighted Legendre table, the twiddles, Wigner d(π/2) — all from FP64
kernels.  PhaseBand: what a phase adds at L (master.Harmonics.init :680-710, spherical.PhaseGpu
:204-225): the harmonics of the master and of its square in FP64, the symmetry rules, the fold of
the c axis, and the correlation tables of f and f² the spectrum GEMM reads.
"""
import ctypes
import math

import numpy as np
import torch

from . import _native as N

TW_LEN = 1024


def fft_size(L):
    """spherical.zig:100-104"""
    n = 16
    while n < 2 * L - 1:
        n *= 2
    return n


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def pair_orders(L):
    """(m, l) of every stored pair (m-major)."""
    ms = np.concatenate([np.full(L - m, m) for m in range(L)])
    ls = np.concatenate([np.arange(m, L) for m in range(L)])
    return ms, ls


class Rules:
    """sh.zig:383-423 — the selection rules read off a function's coefficients."""

    def __init__(self, n_fold=1, mirror=False, inversion=False):
        self.n_fold, self.mirror, self.inversion = n_fold, mirror, inversion

    def allows(self, l, m):
        ok = (m % self.n_fold) == 0
        if self.mirror:
            ok &= ((l + m) % 2) == 0
        if self.inversion:
            ok &= (l % 2) == 0
        return ok

    @staticmethod
    def detect(L, coef, tol):
        ms, ls = pair_orders(L)
        e = np.where(ms == 0, 1.0, 2.0) * np.abs(coef) ** 2
        e = np.where(ls == 0, 0.0, e)
        total = e.sum()
        if total <= 0:
            return Rules()
        r = Rules(inversion=bool(e[ls % 2 == 1].sum() < tol * total), mirror=bool(e[(ls + ms) % 2 == 1].sum() < tol * total))
        for nf in (6, 4, 3, 2):
            if e[ms % nf != 0].sum() < tol * total:
                r.n_fold = nf
                break
        return r


def gauss_legendre(n, dev):
    x = torch.empty(n, dtype=torch.float64, device=dev)
    w = torch.empty(n, dtype=torch.float64, device=dev)
    N.call("zeb_gauss_legendre", n, ptr(x), ptr(w), stream_ptr())
    return x, w


def legendre_table(L, x):
    out = torch.empty(x.numel(), L * (L + 1) // 2, dtype=torch.float64, device=x.device)
    N.call("zeb_legendre_table", L, x.numel(), ptr(x), ptr(out), stream_ptr())
    return out


class BandTables:
    def __init__(self, L, dev):
        self.L = L
        self.n = fft_size(L)
        self.n_theta = self.n
        self.n_phi = 2 * self.n
        self.n_pairs = L * (L + 1) // 2
        nt, nphi = self.n_theta, self.n_phi
        x, w = gauss_legendre(nt, dev)
        plm = legendre_table(L, x[: nt // 2].contiguous())
        self.ring = torch.stack([x, torch.sqrt(torch.clamp(1 - x * x, min=0.0)), w, torch.zeros_like(x)], 1).float().contiguous()
        phi = 2 * math.pi * torch.arange(nphi, dtype=torch.float64, device=dev) / nphi
        self.phi_cs = torch.stack([torch.cos(phi), torch.sin(phi)], 1).float().contiguous()
        self.wplm = (w[: nt // 2, None] * plm * (2 * math.pi / nphi)).float().contiguous()
        t = -2 * math.pi * torch.arange(TW_LEN, dtype=torch.float64, device=dev) / TW_LEN
        self.tw = torch.stack([torch.cos(t), torch.sin(t)], 1).float().contiguous()
        self.wigner = torch.empty(L * L * L, dtype=torch.float64, device=dev)
        N.call("zeb_wigner_half_pi", L, ptr(self.wigner), stream_ptr())
        self.st = N.SphereTables(L, nt, nphi, self.n_pairs, self.ring.data_ptr(), self.phi_cs.data_ptr(),
                                 self.wplm.data_ptr(), self.tw.data_ptr())


def analyze(samples, w, plm, L):
    """sh.zig:146-186 on the device in FP64: ring spectra by FFT along φ, then the Legendre sums."""
    nphi = samples.shape[1]
    F = torch.fft.rfft(samples, dim=1)[:, :L] * (2 * math.pi / nphi)
    ms, _ = pair_orders(L)
    msd = torch.as_tensor(ms, device=samples.device)
    return ((w[:, None] * plm).to(torch.complex128) * F[:, msd]).sum(0)


def synthesize(coef, plm, L, n_phi):
    """sh.zig:189-222 on the device in FP64."""
    ms, _ = pair_orders(L)
    msd = torch.as_tensor(ms, device=coef.device)
    G = torch.zeros(plm.shape[0], n_phi // 2 + 1, dtype=torch.complex128, device=coef.device)
    G.index_add_(1, msd, plm.to(torch.complex128) * coef[None, :])
    return torch.fft.irfft(G, n=n_phi, dim=1) * n_phi


def spectrum_scale(Y, L):
    """The power of two s with s·|U| <= 16384 for every spectrum of this table: |U[j][m'][c]| =
    |Σ_l conj(g_lm') Y[pair(m',l)][j·nc+c]| <= ||g|| · y (Cauchy–Schwarz; the coefficients have unit
    norm), y the largest column norm over l of any order m' (Y: complex [pair][column], pairs
    m-major). FP16 then keeps 11 significant bits of every value far from its range's ends."""
    ms, _ = pair_orders(L)
    rows = torch.as_tensor(ms, device=Y.device)
    sq = torch.zeros(L, Y.shape[1], dtype=torch.float64, device=Y.device)
    sq.index_add_(0, rows, (Y.real * Y.real + Y.imag * Y.imag))
    y = float(torch.sqrt(sq.max()))
    return float(2.0 ** math.floor(math.log2(16384.0 / max(y, 1e-30))))


class PhaseBand:
    """A phase at one bandwidth: harmonics, rules, fold, weight tables → correlation tables."""

    def __init__(self, bt, sheets, side, L, precision="f32"):
        dev = sheets.device
        self.L = L
        nt = max(4 * L, 512)
        x, w = gauss_legendre(nt, dev)
        samples = torch.empty(nt, 2 * nt, dtype=torch.float64, device=dev)
        N.call("zeb_master_sample_grid", ptr(sheets), side, ptr(x), nt, 2 * nt, ptr(samples), stream_ptr())
        plm = legendre_table(L, x)
        f = analyze(samples, w, plm, L)
        f[0] = 0
        fh = f.cpu().numpy()
        self.rules = Rules.detect(L, fh, 1e-5)
        ms, ls = pair_orders(L)
        keep = torch.as_tensor(self.rules.allows(ls, ms), device=dev)
        f = torch.where(keep, f, torch.zeros_like(f))
        x2, w2 = gauss_legendre(2 * L, dev)
        plm2 = legendre_table(L, x2)
        s2 = synthesize(f, plm2, L, 4 * L)
        f2 = analyze(s2 * s2, w2, plm2, L)
        self.f, self.f2 = f, f2
        self.fold = {4: 4, 2: 2, 6: 2}.get(self.rules.n_fold, 1)
        n = bt.n
        self.dims = N.So3Dims(L, n, n // 2 + 1, n // self.fold, self.fold, (L - 1) // self.fold, bt.n_pairs)
        self.Y_f, Y64 = self._table(bt, f, keep=True)
        self.Y_f2 = self._table(bt, f2)
        # the BF16 forms: the master's table split and packed once for the tensor-core spectrum
        # (hi/lo BF16 pairs from the FP64 table, in the shared-memory layout the MMA reads)
        from .settings import SPLIT_L

        self.A = None
        self.split = None
        if SPLIT_L.get(precision) is not None:
            self.split = min(SPLIT_L[precision], L - 1)
            nbytes = N.load().zeb_tc_master_bytes(ctypes.byref(self.dims), self.split)
            if nbytes == 0:
                raise N.NativeError(f"precision {precision}: bandwidth {L} is beyond the tensor-core spectrum")
            self.A = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            N.call("zeb_tc_pack_master", ctypes.byref(self.dims), self.split, ptr(torch.view_as_real(Y64)),
                   ptr(self.A), stream_ptr())
        # the BF16 form keeps the spectrum in FP16 (zeb_spectrum_bf16_h, zeb_correlate_peaks_h) where
        # the tensor-core transform along a takes the bandwidth; bf16x3 keeps FP32 (its point is
        # FP32-quality U)
        self.u_scale = None
        if precision == "bf16" and 16 <= L <= 64 and n == 2 * L and 2 * self.dims.nb * self.dims.nc >= 128:
            self.u_scale = spectrum_scale(Y64, L)
        del Y64
        self.rden = None
        self.rden_key = None

    def weights(self, bt, coef):
        """master.zig:727-753 — W[μ+μmax, l, k] = i^{−m} f_{l,m} d^l_{k,m}(π/2), m = fold·μ, FP64."""
        L, fold = self.L, self.fold
        dev = coef.device
        mu_max = (L - 1) // fold
        mus = np.arange(-mu_max, mu_max + 1)
        m = mus * fold
        am = np.abs(m)
        l = np.arange(L)
        # f_{l,m} for signed m from m ≥ 0 storage: a_{l,−m} = (−1)^m conj(a_lm)
        pidx = am[:, None] * L - (am[:, None] * (am[:, None] - 1)) // 2 + (l[None, :] - am[:, None])
        valid = l[None, :] >= am[:, None]
        pidx = np.where(valid, pidx, 0)
        F = coef[torch.as_tensor(pidx, device=dev)]
        neg = torch.as_tensor(m < 0, device=dev)[:, None]
        sgn = torch.as_tensor(np.where(am % 2 == 1, -1.0, 1.0), device=dev)[:, None]
        F = torch.where(neg, torch.conj(F) * sgn, F) * torch.as_tensor(valid, device=dev)
        tab = bt.wigner.view(L, L, L)  # [k][m][l]
        D = tab[:, torch.as_tensor(am, device=dev), :].permute(1, 0, 2)  # [mi][k][l]
        kk = torch.arange(L, device=dev)
        par = ((kk[:, None] + torch.arange(L, device=dev)[None, :]) % 2 == 1)
        flip = torch.where(par, -1.0, 1.0).to(torch.float64)  # (−1)^{l+k}
        D = torch.where(neg[:, :, None], D * flip[None], D)
        ph = torch.as_tensor(np.array([(1, -1j, -1, 1j)[int(v) % 4] for v in m]), device=dev)  # i^{−m}
        W = ph[:, None, None] * F[:, :, None] * D.permute(0, 2, 1).to(torch.complex128)  # [mi][l][k]
        return W.contiguous()

    def _table(self, bt, coef, keep=False):
        """The FP32 table (and with keep, the FP64 one it was rounded from)."""
        W = self.weights(bt, coef)
        d = self.dims
        Y = torch.empty(bt.n_pairs, d.nb * d.nc, dtype=torch.complex128, device=coef.device)
        N.call("zeb_correlation_table", ctypes.byref(d), ptr(torch.view_as_real(W)), ptr(bt.wigner),
               ptr(torch.view_as_real(Y)), stream_ptr())
        Yf = torch.view_as_real(Y.to(torch.complex64)).contiguous()
        return (Yf, Y) if keep else Yf

    def volume_cells(self):
        d = self.dims
        return d.nb * d.nc * d.n


def master_blur(sheets, side, sigma):
    """prep.zig:215-237 — Gaussian smoothing on the sphere by sigma sheet pixels at the pole, in
    passes of doubling width (each over a 9 × 9 tangent lattice of step 0.6σ)."""
    if not (sigma > 0.05):
        return sheets
    px_rad = math.sqrt(2 * math.pi) / side
    left = sigma * sigma
    s = min(sigma, 2.0)
    src = sheets
    dst = torch.empty_like(sheets)
    while left > 1e-6:
        if s * s > left or left - s * s < 0.02 * left:
            s = math.sqrt(left)
        left -= s * s
        sr = s * px_rad
        N.call("zeb_master_blur_pass", ptr(src), ptr(dst), side, 0.6 * sr, 1.0 / (2 * sr * sr), 4, stream_ptr())
        src, dst = dst, src
        s *= 2
    return src.clone()
