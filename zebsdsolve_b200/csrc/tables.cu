// FP64 tables on the device: Gauss–Legendre quadrature, normalized associated Legendre values,
// Wigner d(π/2) by its three-term recursion, and each phase's correlation table (the Wigner-d
// contraction of the master's weights with the transform along b folded in).
//
// These run once per bandwidth or per phase; their outputs are rounded to FP32 (or BF16 hi/lo)
// for the per-pattern kernels.
#include "abi_util.cuh"

namespace zeb {

// Newton's iteration on P_n for node i (and its mirror n−1−i), as sh.zig:31-72 states it.
__global__ void k_gauss_legendre(int n, double* x, double* w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (n + 1) / 2) return;
  const double nf = (double)n;
  double z = cos(3.14159265358979323846 * ((double)i + 0.75) / (nf + 0.5));
  double p0, p1;
  for (int it = 0; it < 100; ++it) {
    p0 = 1.0; p1 = z;
    for (int k = 2; k <= n; ++k) {
      double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1; p1 = p2;
    }
    double dp = nf * (z * p1 - p0) / (z * z - 1.0);
    double dz = p1 / dp;
    z -= dz;
    if (fabs(dz) < 1e-16) break;
  }
  p0 = 1.0; p1 = z;
  for (int k = 2; k <= n; ++k) {
    double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
    p0 = p1; p1 = p2;
  }
  double dp = nf * (z * p1 - p0) / (z * z - 1.0);
  x[i] = z;
  x[n - 1 - i] = -z;
  w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  w[n - 1 - i] = w[i];
}

__host__ __device__ inline int pair_index(int L, int m, int l) { return m * L - (m * (m - 1)) / 2 + (l - m); }

// One thread per (x_i, m): P̄_m^m then the recursion up in l (sh.zig:75-99).
__global__ void k_legendre(int L, int n_x, const double* __restrict__ x, double* __restrict__ plm) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_x * L) return;
  int i = t / L, m = t % L;
  const int np = L * (L + 1) / 2;
  double xv = x[i];
  double s = sqrt(fmax(0.0, 1.0 - xv * xv));
  double pmm = sqrt(1.0 / (4.0 * 3.14159265358979323846));
  for (int mm = 1; mm <= m; ++mm) pmm *= -sqrt((2.0 * mm + 1.0) / (2.0 * mm)) * s;
  double* out = plm + (size_t)i * np;
  int base = pair_index(L, m, m);
  out[base] = pmm;
  if (m + 1 >= L) return;
  double p1 = sqrt(2.0 * m + 3.0) * xv * pmm;
  out[base + 1] = p1;
  double p2 = pmm;
  for (int l = m + 2; l < L; ++l) {
    double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
    double b = sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
    double p = a * (xv * p1 - b * p2);
    out[base + l - m] = p;
    p2 = p1; p1 = p;
  }
}

// One thread per (k ≥ m): the Jacobi polynomial P_{j−k}^{(k−m, k+m)}(0) by its three-term
// recursion in degree, and the prefactor from log-factorials (sh.zig:239-280).
__global__ void k_wigner(int L, double* __restrict__ d) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L * L) return;
  int k = t / L, m = t % L;
  if (m > k) return;
  const double a = (double)(k - m), b = (double)(k + m);
  double p2 = 0.0, p1 = 0.0;
  for (int nn = 0; nn + k < L; ++nn) {
    double p;
    if (nn == 0) {
      p = 1.0;
    } else if (nn == 1) {
      p = (a - b) / 2.0;
    } else {
      double c = 2.0 * nn + a + b;
      double num1 = (c - 1.0) * (a * a - b * b);
      double num2 = 2.0 * (nn + a - 1.0) * (nn + b - 1.0) * c;
      double den = 2.0 * nn * (nn + a + b) * (c - 2.0);
      p = (num1 * p1 - num2 * p2) / den;
    }
    int j = nn + k;
    double lg = lgamma((double)(nn + 2 * k) + 1.0) + lgamma((double)nn + 1.0) - lgamma((double)(j + m) + 1.0) -
                lgamma((double)(j - m) + 1.0);
    double pref = exp(0.5 * lg) * ldexp(1.0, -k);
    double v = pref * p;
    d[((size_t)m * L + k) * L + j] = v;
    d[((size_t)k * L + m) * L + j] = ((k - m) % 2 == 0) ? v : -v;
    p2 = p1; p1 = p;
  }
}

// Y[pair(m',l)][j·nc + iq] = i^{m'} Σ_k d^l_{k,m'} W[μ,l,k] β(k, j): one thread per output.
__global__ void k_correlation_table(zeb_so3_dims_t dm, const double2* __restrict__ W, const double* __restrict__ dq,
                                    double2* __restrict__ Y) {
  const int L = dm.L, nc = dm.nc, nb = dm.nb;
  const long long cols = (long long)nb * nc;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)dm.n_pairs * cols) return;
  int p = (int)(t / cols);
  int col = (int)(t % cols);
  int j = col / nc, iq = col % nc;
  // (m', l) of pair p
  int mp = 0;
  while (mp + 1 < L && pair_index(L, mp + 1, mp + 1) <= p) ++mp;
  int l = p - pair_index(L, mp, mp) + mp;
  int mu = (iq >= (nc + 1) / 2) ? iq - nc : iq;
  double2 out = make_double2(0.0, 0.0);
  if (abs(mu) <= dm.mu_max) {
    int m = mu * dm.fold;
    bool odd = ((mp + abs(m)) & 1) != 0;  // T[−k] = (−1)^{m'+m} T[k]
    const double2* Wr = W + ((size_t)(mu + dm.mu_max) * L + l) * L;
    const double bj = 6.283185307179586476925 * (double)j / (double)dm.n;
    double re = 0.0, im = 0.0;
    int kmax = l;  // d^l_{k,m'} = 0 for k > l
    for (int k = 0; k <= kmax && k < L; ++k) {
      double dd = dq[((size_t)k * L + mp) * L + l];
      double2 w = Wr[k];
      double tr = dd * w.x, ti = dd * w.y;
      if (k == 0) {
        re += tr; im += ti;
      } else if (!odd) {
        double c = 2.0 * cos(bj * k);
        re += tr * c; im += ti * c;
      } else {
        double s = -2.0 * sin(bj * k);  // × (−2i sin): (tr + i ti)(i s) = −ti s + i tr s
        re += -ti * s; im += tr * s;
      }
    }
    // × i^{m'}
    switch (mp & 3) {
      case 0: out = make_double2(re, im); break;
      case 1: out = make_double2(-im, re); break;
      case 2: out = make_double2(-re, -im); break;
      default: out = make_double2(im, -re); break;
    }
  }
  Y[t] = out;
}

// The transform along c folded into the table: each (pair, j) row of nc slots (the master's
// order μ ≡ slot mod nc) becomes its DFT at the nc grid points of c,
//   Y'[pair][j·nc + c] = Σ_s Y[pair][j·nc + s] e^{−2πi s c / nc}
// (e^{−i m c} with m = fold·μ and c = 2π q/n, so3.wgsl:396-430), in place, FP64.  A block holds
// 256/nc whole rows (or one row of nc > 256) and the nc twiddles, from sincospi of exact fractions.
__global__ void k_table_cdft(double2* __restrict__ Y, long long rows, int nc) {
  extern __shared__ double2 cd_sm[];
  double2* tw = cd_sm;       // [nc]
  double2* row = cd_sm + nc;  // [rows per block][nc]
  const int per = blockDim.x / nc;
  const long long r0 = (long long)blockIdx.x * per;
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    double sn, cs;
    sincospi(-2.0 * (double)t / (double)nc, &sn, &cs);
    tw[t] = make_double2(cs, sn);
  }
  const int rl = threadIdx.x / nc, c = threadIdx.x - rl * nc;
  const bool live = rl < per && r0 + rl < rows;
  if (live) row[rl * nc + c] = Y[(r0 + rl) * nc + c];
  __syncthreads();
  if (!live) return;
  double re = 0.0, im = 0.0;
  const double2* in = row + rl * nc;
  for (int s = 0; s < nc; ++s) {
    const double2 v = in[s], w = tw[(s * c) & (nc - 1)];
    re += v.x * w.x - v.y * w.y;
    im += v.x * w.y + v.y * w.x;
  }
  Y[(r0 + rl) * nc + c] = make_double2(re, im);
}

}  // namespace zeb

using namespace zeb;

extern "C" int zeb_gauss_legendre(int n, double* x, double* w, void* stream) {
  ZEB_REQUIRE(n >= 1 && n <= 65536 && x && w, ZEB_EARG, "gauss_legendre: n=%d", n);
  int th = 128, bl = ((n + 1) / 2 + th - 1) / th;
  k_gauss_legendre<<<bl, th, 0, (cudaStream_t)stream>>>(n, x, w);
  return zeb_launch_check("gauss_legendre");
}

extern "C" int zeb_legendre_table(int L, int n_x, const double* x, double* plm, void* stream) {
  ZEB_REQUIRE(L >= 1 && L <= 512 && n_x >= 1 && x && plm, ZEB_EARG, "legendre_table: L=%d n_x=%d", L, n_x);
  int total = n_x * L, th = 128;
  k_legendre<<<(total + th - 1) / th, th, 0, (cudaStream_t)stream>>>(L, n_x, x, plm);
  return zeb_launch_check("legendre_table");
}

extern "C" int zeb_wigner_half_pi(int L, double* d, void* stream) {
  ZEB_REQUIRE(L >= 1 && L <= 512 && d, ZEB_EARG, "wigner_half_pi: L=%d", L);
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(double) * (size_t)L * L * L, (cudaStream_t)stream);
  ZEB_REQUIRE(e == cudaSuccess, ZEB_ECUDA, "wigner_half_pi: %s", cudaGetErrorString(e));
  int th = 128;
  k_wigner<<<(L * L + th - 1) / th, th, 0, (cudaStream_t)stream>>>(L, d);
  return zeb_launch_check("wigner_half_pi");
}

extern "C" int zeb_correlation_table(const zeb_so3_dims_t* d, const double* W, const double* wigner, double* Y,
                                     void* stream) {
  ZEB_REQUIRE(d && W && wigner && Y, ZEB_EARG, "correlation_table: null argument");
  ZEB_REQUIRE(d->L >= 2 && d->L <= 256 && d->nc >= 1 && d->nb >= 1 && d->fold >= 1 &&
                  d->n_pairs == d->L * (d->L + 1) / 2,
              ZEB_EARG, "correlation_table: bad dims L=%d nc=%d nb=%d", d->L, d->nc, d->nb);
  long long total = (long long)d->n_pairs * d->nb * d->nc;
  int th = 256;
  long long bl = (total + th - 1) / th;
  ZEB_REQUIRE((d->nc & (d->nc - 1)) == 0 && d->nc <= 1024, ZEB_EARG, "correlation_table: nc=%d", d->nc);
  k_correlation_table<<<(unsigned)bl, th, 0, (cudaStream_t)stream>>>(*d, (const double2*)W, wigner, (double2*)Y);
  int rc = zeb_launch_check("correlation_table");
  if (rc) return rc;
  const long long rows = (long long)d->n_pairs * d->nb;
  const int per = d->nc >= 256 ? 1 : 256 / d->nc;
  const int threads = per * d->nc;
  const size_t sm = (size_t)(d->nc + threads) * sizeof(double2);
  k_table_cdft<<<(unsigned)((rows + per - 1) / per), threads, sm, (cudaStream_t)stream>>>((double2*)Y, rows, d->nc);
  return zeb_launch_check("correlation_table (transform along c)");
}
