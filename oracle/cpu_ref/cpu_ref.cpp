// The reference's per-pattern indexing path restated in C++17, FP32, threads over patterns: the CPU
// baseline that the bench times on the host cores (test and measurement infrastructure, like the
// rest of oracle/: nothing here is part of the product, and the product never calls it).
//
// It follows the oracle's FP64 NumPy restatement (oracle/pipeline.py Scan.index) step by step,
// in single precision, with the tables the oracle builds (passed in as FP32 arrays), the patterns
// spread over host threads (std::thread, each taking the next pattern):
//   * the filters (oracle/prep.py run: static background, the direct Gaussian background with
//     its taps renormalized inside the image, zero mean and unit norm under the mask;
//     prep.zig:143-204, prep.wgsl);
//   * the pattern on the Gauss–Legendre grid and its harmonics (oracle/spherical.py sample_grid,
//     coefficients; oracle/sh.py Grid.analyze: a 256-point FFT per ring, then the weighted
//     Legendre sums; sphere.wgsl, sh.zig:146-186);
//   * the correlation volume (oracle/spherical.py correlation_volume: the Wigner-weighted
//     products over every degree accumulated on the (k, m', μ) grid, then a 3-D FFT; so3.wgsl,
//     sh.zig:352-379), times the map-centre window's denominators, its peak and the parabolic
//     vertex (peak; so3.wgsl:351-394, 631-709);
//   * the Gauss–Newton refinement from the gradient table and the NMI (oracle/detector.py
//     refine, rot_sums, ncc_grad_hess, nmi; detector.wgsl, detector.zig:178-202).
// The orientation's reduction to the fundamental zone stays with the caller (Python).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

using cf = std::complex<float>;
constexpr float kPi = 3.14159265358979323846f;

struct Tables {
  int h, w;
  const float* static_bg;  // [h·w] or null
  int dynamic;             // 0 none, 1 subtract, 2 divide
  float sigma;             // the background's deviation, pixels (direct blur: floor(σ/6) < 2)
  float mask[3];           // centre row, col, squared radius (<= 0: none)
  float c0[3], c1[3], c2[3];
  int L, n_theta, n_phi;
  const float* dirs;  // [n_theta][n_phi][3]
  const float* glw;   // [n_theta]
  const float* plm;   // [pairs][n_theta]
  int n, nc, fold, mu_max;
  const float* wig;     // per degree l, D^l[k][x] for signed k, x in [−l, l], row-major, concatenated
  const float* f;       // master coefficients [pairs] as (re, im)
  const float* rden;    // [n/2 + 1][nc][n]
  int side;
  const float* grad;    // [2·side·side][4]: tangent gradient (xyz), value (w)
  const float* sheets;  // [2·side·side]
  int iters;
  float max_step;
  int nmi_bins;
};

inline int pair_of(int L, int m, int l) { return m * L - (m * (m - 1)) / 2 + (l - m); }

// ── FFT: forward (e^{−2πi jk/n}), radix 2, in place, n a power of two up to 1024; the twiddles
// of each size computed once (FP64, rounded to FP32) ──
struct Twiddles {
  std::vector<cf> w[11];  // w[lg][k] = e^{−2πi k / 2^lg}, k < 2^(lg−1)
  Twiddles() {
    for (int lg = 1; lg <= 10; ++lg) {
      const int len = 1 << lg;
      w[lg].resize(len / 2);
      for (int k = 0; k < len / 2; ++k)
        w[lg][k] = cf((float)std::cos(-2.0 * M_PI * k / len), (float)std::sin(-2.0 * M_PI * k / len));
    }
  }
};
const Twiddles kTw;

void fft(cf* x, int n) {
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(x[i], x[j]);
  }
  for (int len = 2, lg = 1; len <= n; len <<= 1, ++lg) {
    const cf* tw = kTw.w[lg].data();
    const int half = len / 2;
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < half; ++k) {
        const cf u = x[i + k], v = x[i + k + half] * tw[k];
        x[i + k] = u + v;
        x[i + k + half] = u - v;
      }
  }
}

// ── the filters ──
void prep(const Tables& T, const uint16_t* raw, std::vector<float>& img) {
  const int h = T.h, w = T.w, hw = h * w;
  img.resize(hw);
  for (int i = 0; i < hw; ++i) img[i] = (float)raw[i] - (T.static_bg ? T.static_bg[i] : 0.f);
  if (T.dynamic && T.sigma > 0.f) {
    const int R = std::max(1, (int)std::ceil(3.f * T.sigma));
    const float k0 = 1.f / (2.f * T.sigma * T.sigma);
    std::vector<float> tap(R + 1), tmp(hw), bg(hw);
    for (int d = 0; d <= R; ++d) tap[d] = std::exp(-(float)(d * d) * k0);
    for (int r = 0; r < h; ++r)  // along the rows
      for (int c = 0; c < w; ++c) {
        float s = 0.f, g = 0.f;
        for (int x = std::max(0, c - R); x <= std::min(w - 1, c + R); ++x) {
          const float t = tap[std::abs(x - c)];
          s += t * img[r * w + x];
          g += t;
        }
        tmp[r * w + c] = s / g;
      }
    for (int r = 0; r < h; ++r)  // along the columns
      for (int c = 0; c < w; ++c) {
        float s = 0.f, g = 0.f;
        for (int y = std::max(0, r - R); y <= std::min(h - 1, r + R); ++y) {
          const float t = tap[std::abs(y - r)];
          s += t * tmp[y * w + c];
          g += t;
        }
        bg[r * w + c] = s / g;
      }
    for (int i = 0; i < hw; ++i) img[i] = T.dynamic == 1 ? img[i] - bg[i] : img[i] / std::max(bg[i], 1e-6f);
  }
  // zero mean and unit norm under the mask, zero outside
  double sum = 0.0;
  int cnt = 0;
  std::vector<char> m(hw);
  for (int r = 0; r < h; ++r)
    for (int c = 0; c < w; ++c) {
      const float dr = (float)r - T.mask[0], dc = (float)c - T.mask[1];
      const bool in = T.mask[2] <= 0.f || dr * dr + dc * dc <= T.mask[2];
      m[r * w + c] = in;
      if (in) {
        sum += img[r * w + c];
        ++cnt;
      }
    }
  const float mean = (float)(sum / std::max(cnt, 1));
  double ss = 0.0;
  for (int i = 0; i < hw; ++i) {
    img[i] = m[i] ? img[i] - mean : 0.f;
    ss += (double)img[i] * img[i];
  }
  const float inv = 1.f / (float)std::sqrt(std::max(ss, 1e-30));
  for (int i = 0; i < hw; ++i) img[i] *= inv;
}

// ── the pattern's harmonics ──
void coefficients(const Tables& T, const std::vector<float>& pat, const double* t, std::vector<cf>& alm) {
  const int h = T.h, w = T.w, nt = T.n_theta, np_ = T.n_phi, L = T.L;
  const float tx = (float)t[0], ty = (float)t[1], tz = (float)t[2];
  const float c2t = T.c2[0] * tx + T.c2[1] * ty + T.c2[2] * tz;
  std::vector<float> val((size_t)nt * np_), win((size_t)nt * np_);
  double sv = 0.0, sw = 0.0;
  for (int y = 0; y < nt; ++y) {
    double rv = 0.0, rw = 0.0;
    for (int j = 0; j < np_; ++j) {
      const float* d = T.dirs + ((size_t)y * np_ + j) * 3;
      const float nd = T.c2[0] * d[0] + T.c2[1] * d[1] + T.c2[2] * d[2];
      float v = 0.f, wv = 0.f;
      if (nd > 1e-4f) {
        const float s = c2t / nd;
        const float hx = s * d[0] - tx, hy = s * d[1] - ty, hz = s * d[2] - tz;
        const float row = hx * T.c0[0] + hy * T.c0[1] + hz * T.c0[2];
        const float col = hx * T.c1[0] + hy * T.c1[1] + hz * T.c1[2];
        bool in = row >= 0.f && row <= (float)(h - 1) && col >= 0.f && col <= (float)(w - 1);
        if (in && T.mask[2] > 0.f) {
          const float dr = row - T.mask[0], dc = col - T.mask[1];
          in = dr * dr + dc * dc <= T.mask[2];
        }
        if (in) {
          const int r0 = std::min((int)std::floor(row), h - 2), q0 = std::min((int)std::floor(col), w - 2);
          const float fr = row - (float)r0, fc = col - (float)q0;
          const float* p = pat.data() + r0 * w + q0;
          const float top = p[0] * (1.f - fc) + p[1] * fc, bot = p[w] * (1.f - fc) + p[w + 1] * fc;
          v = top * (1.f - fr) + bot * fr;
          wv = 1.f;
        }
      }
      val[(size_t)y * np_ + j] = v;
      win[(size_t)y * np_ + j] = wv;
      rv += (double)v * wv;
      rw += wv;
    }
    sv += rv * T.glw[y];
    sw += rw * T.glw[y];
  }
  const float mean = (float)(sv / std::max(sw, 1e-20));
  // F[y][m] = (2π/nφ) Σ_j s e^{−imφ_j}, then a_lm = Σ_y w_y P̄_lm(y) F[y][m]
  std::vector<cf> line(np_), F((size_t)nt * L);
  const float k2 = 2.f * kPi / (float)np_;
  for (int y = 0; y < nt; ++y) {
    for (int j = 0; j < np_; ++j) line[j] = cf((val[(size_t)y * np_ + j] - mean) * win[(size_t)y * np_ + j], 0.f);
    fft(line.data(), np_);
    for (int m = 0; m < L; ++m) F[(size_t)y * L + m] = line[m] * k2;
  }
  const int pairs = L * (L + 1) / 2;
  alm.assign(pairs, cf(0.f, 0.f));
  for (int m = 0; m < L; ++m)
    for (int l = m; l < L; ++l) {
      const int p = pair_of(L, m, l);
      cf acc(0.f, 0.f);
      for (int y = 0; y < nt; ++y) acc += F[(size_t)y * L + m] * (T.glw[y] * T.plm[(size_t)p * nt + y]);
      alm[p] = acc;
    }
  double pw = 0.0;
  for (int m = 0; m < L; ++m)
    for (int l = m; l < L; ++l) pw += (m == 0 ? 1.0 : 2.0) * std::norm(alm[pair_of(L, m, l)]);
  const float inv = 1.f / (float)std::sqrt(std::max(pw, 1e-30));
  for (auto& a : alm) a *= inv;
}

inline cf signed_coef(const cf* c, int L, int l, int m) {
  const int am = std::abs(m);
  if (am > l) return cf(0.f, 0.f);
  const cf v = c[pair_of(L, am, l)];
  if (m >= 0) return v;
  return (am % 2 == 0) ? std::conj(v) : -std::conj(v);
}

inline cf ipow(int n) {
  switch (((n % 4) + 4) % 4) {
    case 0: return cf(1.f, 0.f);
    case 1: return cf(0.f, 1.f);
    case 2: return cf(-1.f, 0.f);
    default: return cf(0.f, -1.f);
  }
}

struct Peak {
  float q[4];
  float score;
};

// conj(Rz(a) Ry(b) Rz(c)) with w >= 0
void zyz_quat(double a, double b, double c, float* q) {
  const double qa[4] = {std::cos(0.5 * a), 0, 0, std::sin(0.5 * a)};
  const double qb[4] = {std::cos(0.5 * b), 0, std::sin(0.5 * b), 0};
  const double qc[4] = {std::cos(0.5 * c), 0, 0, std::sin(0.5 * c)};
  auto mul = [](const double* x, const double* y, double* o) {
    o[0] = x[0] * y[0] - x[1] * y[1] - x[2] * y[2] - x[3] * y[3];
    o[1] = x[0] * y[1] + x[1] * y[0] + x[2] * y[3] - x[3] * y[2];
    o[2] = x[0] * y[2] - x[1] * y[3] + x[2] * y[0] + x[3] * y[1];
    o[3] = x[0] * y[3] + x[1] * y[2] - x[2] * y[1] + x[3] * y[0];
  };
  double bc[4], r[4];
  mul(qb, qc, bc);
  mul(qa, bc, r);
  double o[4] = {r[0], -r[1], -r[2], -r[3]};
  if (o[0] < 0) for (double& v : o) v = -v;
  for (int k = 0; k < 4; ++k) q[k] = (float)o[k];
}

inline float vertex(float lo, float mid, float hi) {
  const float den = lo - 2.f * mid + hi;
  if (den >= -1e-12f) return 0.f;
  return std::min(std::max(0.5f * (lo - hi) / den, -0.5f), 0.5f);
}

// An FFT along an axis of length n (a power of two) whose consecutive points are `stride` floats
// apart, done for `lanes` contiguous lanes at once (re and im in separate arrays): the bit-reversal
// swaps whole rows and each butterfly runs over the lanes, which the compiler vectorizes.
void fft_rows(float* re, float* im, int n, size_t stride, int lanes) {
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j)
      for (int e = 0; e < lanes; ++e) {
        std::swap(re[i * stride + e], re[j * stride + e]);
        std::swap(im[i * stride + e], im[j * stride + e]);
      }
  }
  for (int half = 1, lg = 1; half < n; half <<= 1, ++lg) {
    const cf* tw = kTw.w[lg].data();
    for (int i = 0; i < n; i += 2 * half)
      for (int k = 0; k < half; ++k) {
        const float wr = tw[k].real(), wi = tw[k].imag();
        float* ar = re + (size_t)(i + k) * stride;
        float* ai = im + (size_t)(i + k) * stride;
        float* br = re + (size_t)(i + k + half) * stride;
        float* bi = im + (size_t)(i + k + half) * stride;
        for (int e = 0; e < lanes; ++e) {
          const float vr = br[e] * wr - bi[e] * wi, vi = br[e] * wi + bi[e] * wr;
          br[e] = ar[e] - vr;
          bi[e] = ai[e] - vi;
          ar[e] += vr;
          ai[e] += vi;
        }
      }
  }
}

// The correlation volume on the Euler grid, times the denominators, and its peak. The oracle sums
// A[k, m', μ] = Σ_l f_lm conj(g_lm') d^l_{k,m'} d^l_{k,m} i^{m'−m} (m = fold·μ) and transforms all
// three axes; here the transform along μ is folded into the sums, A[k][m'][c] += Q_l[k][m'] ·
// P̂_l[k][c] with P̂_l[k][c] = Σ_μ f_lm d^l_{k,m} i^{−m} e^{−2πi μ c/nc} (the same DFT, taken per
// degree, so each update is a contiguous complex AXPY over c), then m' and k are transformed.
Peak correlate(const Tables& T, const std::vector<cf>& g, std::vector<float>& Are, std::vector<float>& Aim) {
  const int L = T.L, n = T.n, nc = T.nc, fold = T.fold, mu_max = T.mu_max;
  const cf* f = reinterpret_cast<const cf*>(T.f);
  const size_t total = (size_t)n * n * nc;
  Are.assign(total, 0.f);
  Aim.assign(total, 0.f);
  // e^{−2πi μ c / nc} for every μ and c
  std::vector<cf> om((size_t)(2 * mu_max + 1) * nc);
  for (int mu = -mu_max; mu <= mu_max; ++mu)
    for (int c = 0; c < nc; ++c) {
      const double a = -2.0 * M_PI * (double)(((long long)mu * c) % nc) / nc;
      om[(size_t)(mu + mu_max) * nc + c] = cf((float)std::cos(a), (float)std::sin(a));
    }
  std::vector<float> Pr, Pi, Qr, Qi;
  size_t off = 0;
  for (int l = 0; l < L; ++l) {
    const int s = 2 * l + 1;
    const float* D = T.wig + off;  // D[(k+l)·s + (x+l)]
    off += (size_t)s * s;
    Pr.assign((size_t)s * nc, 0.f);
    Pi.assign((size_t)s * nc, 0.f);
    bool any = false;
    for (int mu = -mu_max; mu <= mu_max; ++mu) {
      const int m = mu * fold;
      if (std::abs(m) > l) continue;
      const cf fl = signed_coef(f, L, l, m);
      if (fl == cf(0.f, 0.f)) continue;
      any = true;
      const cf ph = fl * ipow(-m);
      const cf* w = om.data() + (size_t)(mu + mu_max) * nc;
      for (int k = -l; k <= l; ++k) {
        const cf p = ph * D[(k + l) * s + (m + l)];
        float* pr = Pr.data() + (size_t)(k + l) * nc;
        float* pi = Pi.data() + (size_t)(k + l) * nc;
        for (int c = 0; c < nc; ++c) {
          pr[c] += p.real() * w[c].real() - p.imag() * w[c].imag();
          pi[c] += p.real() * w[c].imag() + p.imag() * w[c].real();
        }
      }
    }
    if (!any) continue;
    Qr.resize((size_t)s * s);
    Qi.resize((size_t)s * s);
    for (int x = -l; x <= l; ++x) {
      const cf gc = std::conj(signed_coef(g.data(), L, l, x)) * ipow(x);
      for (int k = -l; k <= l; ++k) {
        const float d = D[(k + l) * s + (x + l)];
        Qr[(size_t)(k + l) * s + (x + l)] = gc.real() * d;
        Qi[(size_t)(k + l) * s + (x + l)] = gc.imag() * d;
      }
    }
    for (int k = -l; k <= l; ++k) {
      const int ki = ((k % n) + n) % n;
      const float* pr = Pr.data() + (size_t)(k + l) * nc;
      const float* pi = Pi.data() + (size_t)(k + l) * nc;
      for (int x = -l; x <= l; ++x) {
        const float qr = Qr[(size_t)(k + l) * s + (x + l)], qi = Qi[(size_t)(k + l) * s + (x + l)];
        const size_t o = ((size_t)ki * n + (((x % n) + n) % n)) * nc;
        float* ar = Are.data() + o;
        float* ai = Aim.data() + o;
        for (int c = 0; c < nc; ++c) {
          ar[c] += qr * pr[c] - qi * pi[c];
          ai[c] += qr * pi[c] + qi * pr[c];
        }
      }
    }
  }
  // along m' (rows of nc lanes, one block per k), then along k (rows of n·nc lanes)
  for (int k = 0; k < n; ++k) fft_rows(Are.data() + (size_t)k * n * nc, Aim.data() + (size_t)k * n * nc, n, nc, nc);
  fft_rows(Are.data(), Aim.data(), n, (size_t)n * nc, n * nc);
  // C[k→j][m'→a][μ→c] → vol[j][c][a] for j <= n/2, times the denominators
  const int nb = n / 2 + 1;
  std::vector<float> vol((size_t)nb * nc * n);
  for (int j = 0; j < nb; ++j)
    for (int a = 0; a < n; ++a)
      for (int c = 0; c < nc; ++c) {
        const size_t o = ((size_t)j * nc + c) * n + a;
        vol[o] = Are[((size_t)j * n + a) * nc + c] * T.rden[o];
      }
  // the peak (first of equal values) and the vertex along a, c and (inside) b
  size_t best = 0;
  for (size_t i = 1; i < vol.size(); ++i)
    if (vol[i] > vol[best]) best = i;
  const int j = (int)(best / ((size_t)nc * n)), rest = (int)(best % ((size_t)nc * n));
  const int iq = rest / n, ia = rest % n;
  auto at = [&](int jj, int qq, int aa) { return vol[((size_t)jj * nc + qq) * n + aa]; };
  const float v0 = vol[best];
  const float da = vertex(at(j, iq, (ia + n - 1) % n), v0, at(j, iq, (ia + 1) % n));
  const float dc = vertex(at(j, (iq + nc - 1) % nc, ia), v0, at(j, (iq + 1) % nc, ia));
  float dj = 0.f;
  if (j > 0 && j < n / 2) dj = vertex(at(j - 1, iq, ia), v0, at(j + 1, iq, ia));
  const double step = 2.0 * M_PI / n;
  Peak pk;
  zyz_quat((ia + da) * step, (j + dj) * step, (iq + dc) * step, pk.q);
  pk.score = v0;
  return pk;
}

// ── the detector side: the square-Lambert lookup, the refinement, the NMI ──
inline void sphere_to_square(const float* v, float& u, float& w) {
  const float ax = std::fabs(v[0]), ay = std::fabs(v[1]);
  const float xn = std::sqrt(std::max(kPi * 0.5f * (ax * ax + ay * ay) / (1.f + std::fabs(v[2])), 0.f));
  float uu = xn, ww = xn;
  if (ax >= ay) ww = (4.f * xn / kPi) * std::atan2(ay, std::max(ax, 1e-30f));
  else uu = (4.f * xn / kPi) * std::atan2(ax, std::max(ay, 1e-30f));
  const float sc = 0.79788456080286536f;
  u = uu * sc * (v[0] < 0.f ? -1.f : 1.f);
  w = ww * sc * (v[1] < 0.f ? -1.f : 1.f);
}

// bilinear over the hemisphere's sheet of a table with `ch` channels a texel
inline void lookup(const float* tab, int ch, int side, const float* v, float* out) {
  float u, w;
  sphere_to_square(v, u, w);
  const float last = (float)(side - 1);
  const float fj = std::min(std::max((u + 1.f) * 0.5f * last, 0.f), last);
  const float fi = std::min(std::max((w + 1.f) * 0.5f * last, 0.f), last);
  const int c0 = std::min((int)std::floor(fj), side - 2), r0 = std::min((int)std::floor(fi), side - 2);
  const size_t o = (size_t)r0 * side + c0 + (v[2] < 0.f ? (size_t)side * side : 0);
  const float tj = fj - (float)c0, ti = fi - (float)r0;
  for (int k = 0; k < ch; ++k) {
    const float top = tab[o * ch + k] * (1.f - tj) + tab[(o + 1) * ch + k] * tj;
    const float bot = tab[(o + side) * ch + k] * (1.f - tj) + tab[(o + side + 1) * ch + k] * tj;
    out[k] = top * (1.f - ti) + bot * ti;
  }
}

inline void qapply(const double* q, const float* v, float* o) {
  const double u[3] = {q[1], q[2], q[3]};
  const double t[3] = {2 * (u[1] * v[2] - u[2] * v[1]), 2 * (u[2] * v[0] - u[0] * v[2]), 2 * (u[0] * v[1] - u[1] * v[0])};
  o[0] = (float)(v[0] + q[0] * t[0] + (u[1] * t[2] - u[2] * t[1]));
  o[1] = (float)(v[1] + q[0] * t[1] + (u[2] * t[0] - u[0] * t[2]));
  o[2] = (float)(v[2] + q[0] * t[2] + (u[0] * t[1] - u[1] * t[0]));
}

struct Pixels {
  std::vector<float> u;  // unit rays [npix][3]
  std::vector<float> e;  // pattern values [npix]
};

void pixels_of(const Tables& T, const std::vector<float>& pat, const double* t, Pixels& px) {
  px.u.clear();
  px.e.clear();
  for (int r = 0; r < T.h; ++r)
    for (int c = 0; c < T.w; ++c) {
      const float dr = (float)r - T.mask[0], dc = (float)c - T.mask[1];
      if (T.mask[2] > 0.f && dr * dr + dc * dc > T.mask[2]) continue;
      double v[3];
      for (int k = 0; k < 3; ++k) v[k] = T.c0[k] * (double)r + T.c1[k] * (double)c + t[k];
      const double nrm = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (int k = 0; k < 3; ++k) px.u.push_back((float)(v[k] / nrm));
      px.e.push_back(pat[r * T.w + c]);
    }
}

// the 19 sums → NCC, gradient and GN matrix (xx, xy, xz, yy, yz, zz)
double ncc_grad_hess(const Tables& T, const Pixels& px, const double* q, double* g, double* H) {
  double s[19] = {0};
  const size_t n = px.e.size();
  for (size_t i = 0; i < n; ++i) {
    float c[3], m[4];
    qapply(q, &px.u[i * 3], c);
    lookup(T.grad, 4, T.side, c, m);
    const float d[3] = {c[1] * m[2] - c[2] * m[1], c[2] * m[0] - c[0] * m[2], c[0] * m[1] - c[1] * m[0]};
    const float e = px.e[i];
    s[0] += 1.0; s[1] += m[3]; s[2] += (double)m[3] * m[3]; s[3] += (double)m[3] * e;
    for (int k = 0; k < 3; ++k) {
      s[4 + k] += d[k];
      s[7 + k] += (double)m[3] * d[k];
      s[10 + k] += (double)e * d[k];
      s[13 + k] += (double)d[k] * d[k];
    }
    s[16] += (double)d[0] * d[1]; s[17] += (double)d[0] * d[2]; s[18] += (double)d[1] * d[2];
  }
  const double nn = std::max(s[0], 1.0), mean = s[1] / nn, var_n = s[2] - nn * mean * mean;
  for (int k = 0; k < 3; ++k) g[k] = 0.0;
  for (int k = 0; k < 6; ++k) H[k] = 0.0;
  if (!(var_n > 1e-12)) return -2.0;
  const double inv = 1.0 / std::sqrt(var_n), ncc = s[3] * inv, iv = inv * inv;
  double au[3];
  for (int k = 0; k < 3; ++k) {
    au[k] = (s[7 + k] - mean * s[4 + k]) * inv;
    g[k] = (s[10 + k] - ncc * au[k]) * inv;
  }
  const double* sd = s + 4;
  H[0] = (s[13] - sd[0] * sd[0] / nn - au[0] * au[0]) * iv;
  H[1] = (s[16] - sd[0] * sd[1] / nn - au[0] * au[1]) * iv;
  H[2] = (s[17] - sd[0] * sd[2] / nn - au[0] * au[2]) * iv;
  H[3] = (s[14] - sd[1] * sd[1] / nn - au[1] * au[1]) * iv;
  H[4] = (s[18] - sd[1] * sd[2] / nn - au[1] * au[2]) * iv;
  H[5] = (s[15] - sd[2] * sd[2] / nn - au[2] * au[2]) * iv;
  return ncc;
}

void solve3(const double* h, const double* g, double* x) {
  const double a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5];
  const double det = a * (d * f - e * e) - b * (b * f - e * c) + c * (b * e - d * c);
  if (std::fabs(det) < 1e-30) {
    x[0] = x[1] = x[2] = 0.0;
    return;
  }
  x[0] = (g[0] * (d * f - e * e) - b * (g[1] * f - e * g[2]) + c * (g[1] * e - d * g[2])) / det;
  x[1] = (a * (g[1] * f - e * g[2]) - g[0] * (b * f - e * c) + c * (b * g[2] - g[1] * c)) / det;
  x[2] = (a * (d * g[2] - g[1] * e) - b * (b * g[2] - g[1] * c) + g[0] * (b * e - d * c)) / det;
}

void refine(const Tables& T, const Pixels& px, const float* q0, double* qb, double& best, double& last_good) {
  double qc[4] = {q0[0], q0[1], q0[2], q0[3]};
  for (int k = 0; k < 4; ++k) qb[k] = qc[k];
  best = -2.0;
  double mu = 1.0, gb[3] = {0, 0, 0}, hb[6] = {0, 0, 0, 0, 0, 0}, promised = 0.0, step_len = 0.0;
  int accepted = 0;
  last_good = 0.0;
  for (int it = 0; it <= T.iters; ++it) {
    double g[3], H[6];
    const double ncc = ncc_grad_hess(T, px, qc, g, H);
    if (ncc > best) {
      if (accepted > 0 && promised > 1e-6) {
        const double rho = (ncc - best) / promised;
        mu = std::min(std::max(mu * (2.0 - rho), mu / 3.0), mu * 3.0);
      }
      for (int k = 0; k < 4; ++k) qb[k] = qc[k];
      best = ncc;
      std::memcpy(gb, g, sizeof(gb));
      std::memcpy(hb, H, sizeof(hb));
      last_good = step_len;
      ++accepted;
    } else {
      mu *= 3.0;
    }
    mu = std::min(std::max(mu, 0.02), 1e4);
    if (it == T.iters) break;
    double hh[6];
    for (int k = 0; k < 6; ++k) hh[k] = hb[k] * mu;
    const double tr = std::max(hh[0] + hh[3] + hh[5], 1e-20);
    hh[0] += 1e-6 * tr; hh[3] += 1e-6 * tr; hh[5] += 1e-6 * tr;
    double st[3];
    solve3(hh, gb, st);
    double ln = std::sqrt(st[0] * st[0] + st[1] * st[1] + st[2] * st[2]);
    if (ln > T.max_step) for (double& v : st) v *= T.max_step / ln;
    const double quad = hh[0] * st[0] * st[0] + hh[3] * st[1] * st[1] + hh[5] * st[2] * st[2] +
                        2.0 * (hh[1] * st[0] * st[1] + hh[2] * st[0] * st[2] + hh[4] * st[1] * st[2]);
    promised = gb[0] * st[0] + gb[1] * st[1] + gb[2] * st[2] - 0.5 * quad;
    step_len = std::sqrt(st[0] * st[0] + st[1] * st[1] + st[2] * st[2]);
    const double th2 = step_len * step_len, th = step_len;
    const double kk = th < 1e-6 ? 0.5 - th2 / 48.0 : std::sin(0.5 * th) / th;
    const double e[4] = {std::cos(0.5 * th), kk * st[0], kk * st[1], kk * st[2]};
    double qn[4] = {e[0] * qb[0] - e[1] * qb[1] - e[2] * qb[2] - e[3] * qb[3],
                    e[0] * qb[1] + e[1] * qb[0] + e[2] * qb[3] - e[3] * qb[2],
                    e[0] * qb[2] - e[1] * qb[3] + e[2] * qb[0] + e[3] * qb[1],
                    e[0] * qb[3] + e[1] * qb[2] - e[2] * qb[1] + e[3] * qb[0]};
    const double nq = std::sqrt(qn[0] * qn[0] + qn[1] * qn[1] + qn[2] * qn[2] + qn[3] * qn[3]);
    for (int k = 0; k < 4; ++k) qc[k] = qn[k] / nq;
  }
}

double nmi(const Tables& T, const Pixels& px, const double* q) {
  const size_t n = px.e.size();
  const int nb = T.nmi_bins;
  std::vector<float> sim(n);
  float elo = 3.4e38f, ehi = -3.4e38f, slo = 3.4e38f, shi = -3.4e38f;
  for (size_t i = 0; i < n; ++i) {
    float c[3];
    qapply(q, &px.u[i * 3], c);
    lookup(T.sheets, 1, T.side, c, &sim[i]);
    elo = std::min(elo, px.e[i]); ehi = std::max(ehi, px.e[i]);
    slo = std::min(slo, sim[i]); shi = std::max(shi, sim[i]);
  }
  const double ke = nb / std::max((double)ehi - elo, 1e-20), ks = nb / std::max((double)shi - slo, 1e-20);
  std::vector<double> hist((size_t)nb * nb, 0.0);
  for (size_t i = 0; i < n; ++i) {
    const int be = std::min((int)((px.e[i] - elo) * ke), nb - 1), bs = std::min((int)((sim[i] - slo) * ks), nb - 1);
    hist[(size_t)be * nb + bs] += 1.0;
  }
  double tot = 0.0, hj = 0.0, hm = 0.0;
  for (double c : hist) {
    tot += c;
    if (c > 0) hj -= c * std::log(c);
  }
  for (int a = 0; a < nb; ++a) {
    double rs = 0.0, cs = 0.0;
    for (int b = 0; b < nb; ++b) {
      rs += hist[(size_t)a * nb + b];
      cs += hist[(size_t)b * nb + a];
    }
    if (rs > 0) hm -= rs * std::log(rs);
    if (cs > 0) hm -= cs * std::log(cs);
  }
  const double nn = std::max(tot, 1.0);
  const double h_joint = std::log(nn) + hj / nn;  // hj = −Σ c log c over the joint histogram
  const double h_marg = 2.0 * std::log(nn) + hm / nn;  // hm: the same over both marginals
  return h_marg > 1e-12 ? 2.0 * (h_marg - h_joint) / h_marg : 0.0;
}

}  // namespace

extern "C" {

// Index n stored patterns (u16 [n][h·w]) at detector positions ts ([n][3], pixels) on `threads`
// host threads (0: every hardware thread). out[i][8] = (q of the refined orientation, w x y z, not
// reduced to the zone; NCC; NMI; last improving step; the spherical peak's score). Returns 0.
int zcr_index(const Tables* T, int n, const uint16_t* raws, const double* ts, float* out, int threads) {
  const int nt = std::max(1, std::min(threads > 0 ? threads : (int)std::thread::hardware_concurrency(), n));
  std::atomic<int> next(0);
  auto work = [&]() {
    std::vector<float> pat;
    std::vector<cf> alm;
    std::vector<float> Are, Aim;
    Pixels px;
    const size_t hw = (size_t)T->h * T->w;
    for (int i = next++; i < n; i = next++) {
      prep(*T, raws + hw * i, pat);
      coefficients(*T, pat, ts + 3 * i, alm);
      const Peak pk = correlate(*T, alm, Are, Aim);
      pixels_of(*T, pat, ts + 3 * i, px);
      double qb[4], best, step;
      refine(*T, px, pk.q, qb, best, step);
      const double v = nmi(*T, px, qb);
      float* o = out + (size_t)i * 8;
      for (int k = 0; k < 4; ++k) o[k] = (float)qb[k];
      o[4] = (float)best; o[5] = (float)v; o[6] = (float)step; o[7] = pk.score;
    }
  };
  std::vector<std::thread> pool;
  for (int k = 1; k < nt; ++k) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  return 0;
}

int zcr_threads(void) { return std::max(1, (int)std::thread::hardware_concurrency()); }

}  // extern "C"
