// Non-local pattern averaging (NLPAR; Brewick, Wright and Rowenhorst, Ultramicroscopy 200 (2019)
// 50): each pattern replaced by a weighted mean of itself and its neighbours in the map, a
// neighbour weighing as much as it looks like the same pattern under other noise.
//
//   d²(i, j)  the mean squared difference of patterns i and j over their px pixels
//   σ²(i)     the noise of stored pattern i: half the least d² to one of its eight nearest
//             neighbours
//   e(i, j)   the d² noise alone gives: Σ_u (a_i[u] − a_j[u − o])² σ²(i + u) over the stored
//             patterns' shares a of each average (σ²(i) + σ²(j) for stored patterns)
//   w(i, j)   1 where d² ≤ e, else exp(−sqrt(px / 2) · (d²/e − 1) / λ²) (0 where e = 0); 1 for i
//   out(i)    Σ w(i, j) pattern(j) / Σ w(i, j) over the (2 radius + 1)² window
//
// in `passes` passes, each on the patterns the last one left. The patterns come as a list: the
// wanted cells first, then ring after ring of the map's cells around them; counts[d] cells lie
// within d rings of the wanted ones, so each pass works on a prefix. nbr[c · F + slot] is the
// list index of the cell at offset (dy, dx) of cell c, up to reach = radius · passes each way
// (F = (2 reach + 1)² slots, rows first), or ZEB_NLPAR_NONE. d² and weights have one slot per
// offset of the radius window (K = (2 radius + 1)²), the cell itself in the middle.
// (shaders/nlpar.wgsl distance, sigma, weights, average, shares; src/nlpar.zig:89-138.)
#include "abi_util.cuh"

namespace zeb {

constexpr uint32_t NL_NONE = 0xffffffffu;

struct NlArgs {
  const float* pin;
  float* pout;
  const uint32_t* nbr;
  float* d2;
  float* sig;
  float* wts;
  const float* share_in;
  float* share;
  int n, px, radius, reach, out0, spread;
  float inv_l2, sqn;  // 1 / λ², sqrt(px / 2)
};

__device__ __forceinline__ int nl_wide(const NlArgs& a, int dy, int dx) {
  return (dy + a.reach) * (2 * a.reach + 1) + dx + a.reach;
}
__device__ __forceinline__ int nl_F(const NlArgs& a) { return (2 * a.reach + 1) * (2 * a.reach + 1); }
__device__ __forceinline__ int2 nl_offset(const NlArgs& a, int q) {
  const int side = 2 * a.radius + 1;
  return make_int2(q / side - a.radius, q % side - a.radius);
}
__device__ __forceinline__ bool nl_within(int dy, int dx, int r) { return abs(dy) <= r && abs(dx) <= r; }

// one block per (cell, later offset of its window): d² of the pair, written from both cells
__global__ void __launch_bounds__(256) k_nl_distance(NlArgs a) {
  __shared__ float red[8];
  const int side = 2 * a.radius + 1, K = side * side, later = K / 2;
  const long long pair = blockIdx.x;
  const int c = (int)(pair / later);
  const int q = later + 1 + (int)(pair % later);
  const int2 o = nl_offset(a, q);
  const uint32_t j = a.nbr[(size_t)c * nl_F(a) + nl_wide(a, o.x, o.y)];
  if (j == NL_NONE) return;
  const float* pc = a.pin + (size_t)c * a.px;
  const float* pj = a.pin + (size_t)j * a.px;
  float acc = 0.f;
  for (int p = threadIdx.x; p < a.px; p += blockDim.x) {
    const float d = pc[p] - pj[p];
    acc = fmaf(d, d, acc);
  }
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    const float v = t / (float)a.px;
    a.d2[(size_t)c * K + q] = v;
    a.d2[(size_t)j * K + (K - 1 - q)] = v;
  }
}

__global__ void k_nl_sigma(NlArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  const int side = 2 * a.radius + 1;
  float least = -1.f;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      if ((dy == 0 && dx == 0) || a.nbr[(size_t)c * nl_F(a) + nl_wide(a, dy, dx)] == NL_NONE) continue;
      const float v = a.d2[(size_t)c * side * side + (dy + a.radius) * side + (dx + a.radius)];
      if (least < 0.f || v < least) least = v;
    }
  a.sig[c] = 0.5f * fmaxf(least, 0.f);  // no neighbours: no estimate, 0 (only itself averages)
}

// the noise in the difference of the averages of cell c and its neighbour j at offset o
__device__ float nl_expected(const NlArgs& a, int c, uint32_t j, int2 o) {
  if (a.spread == 0) return a.sig[c] + a.sig[j];
  const int F = nl_F(a), m = a.spread + a.radius;
  float e = 0.f;
  for (int uy = -m; uy <= m; ++uy)
    for (int ux = -m; ux <= m; ++ux) {
      const uint32_t at = a.nbr[(size_t)c * F + nl_wide(a, uy, ux)];
      if (at == NL_NONE) continue;
      const float mine = nl_within(uy, ux, a.spread) ? a.share_in[(size_t)c * F + nl_wide(a, uy, ux)] : 0.f;
      const int vy = uy - o.x, vx = ux - o.y;
      const float theirs = nl_within(vy, vx, a.spread) ? a.share_in[(size_t)j * F + nl_wide(a, vy, vx)] : 0.f;
      const float d = mine - theirs;
      e += d * d * a.sig[at];
    }
  return e;
}

__global__ void k_nl_weights(NlArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.n) return;
  const int side = 2 * a.radius + 1, K = side * side, own = K / 2;
  float total = 1.f;
  for (int q = 0; q < K; ++q) {
    if (q == own) continue;
    const int2 o = nl_offset(a, q);
    const uint32_t j = a.nbr[(size_t)c * nl_F(a) + nl_wide(a, o.x, o.y)];
    float w = 0.f;
    if (j != NL_NONE) {
      const float e = nl_expected(a, c, j, o);
      const float d = a.d2[(size_t)c * K + q];
      if (d <= e) w = 1.f;
      else if (e > 0.f) w = expf(-a.sqn * (d / e - 1.f) * a.inv_l2);
    }
    a.wts[(size_t)c * K + q] = w;
    total += w;
  }
  for (int q = 0; q < K; ++q) a.wts[(size_t)c * K + q] = q == own ? 1.f / total : a.wts[(size_t)c * K + q] / total;
}

__global__ void k_nl_average(NlArgs a) {
  const long long total = (long long)a.n * a.px;
  const int side = 2 * a.radius + 1, K = side * side;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / a.px), p = (int)(t - (long long)c * a.px);
    float acc = 0.f;
    for (int q = 0; q < K; ++q) {
      const float w = a.wts[(size_t)c * K + q];
      if (w == 0.f) continue;
      const int2 o = nl_offset(a, q);
      acc += w * a.pin[(size_t)a.nbr[(size_t)c * nl_F(a) + nl_wide(a, o.x, o.y)] * a.px + p];
    }
    a.pout[(size_t)(a.out0 + c) * a.px + p] = acc;
  }
}

// a'_c[u] = Σ_j w(c, j) a_j[u − o_j]: the average's share of the stored pattern at offset u
__global__ void k_nl_shares(NlArgs a) {
  const int F = nl_F(a), wn = 2 * a.reach + 1;
  const long long total = (long long)a.n * F;
  const int side = 2 * a.radius + 1, K = side * side;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / F), slot = (int)(t - (long long)c * F);
    const int uy = slot / wn - a.reach, ux = slot % wn - a.reach;
    float acc = 0.f;
    for (int q = 0; q < K; ++q) {
      const float w = a.wts[(size_t)c * K + q];
      if (w == 0.f) continue;
      const int2 o = nl_offset(a, q);
      const int vy = uy - o.x, vx = ux - o.y;
      if (a.spread == 0) {
        if (vy == 0 && vx == 0) acc += w;
      } else if (nl_within(vy, vx, a.spread)) {
        acc += w * a.share_in[(size_t)a.nbr[(size_t)c * F + nl_wide(a, o.x, o.y)] * F + nl_wide(a, vy, vx)];
      }
    }
    a.share[t] = acc;
  }
}

static unsigned nl_grid(long long count) {
  const long long b = (count + 255) / 256;
  return (unsigned)(b < 1 ? 1 : (b > 148LL * 64 ? 148LL * 64 : b));
}

struct NlScratch {
  float *b, *d2, *wts, *sig, *sa, *sb;
};

static size_t nl_layout(int n_win, int px, int radius, int passes, char* base, NlScratch* s) {
  const size_t K = (size_t)(2 * radius + 1) * (2 * radius + 1);
  const size_t reach = (size_t)radius * passes, F = (2 * reach + 1) * (2 * reach + 1);
  const size_t sizes[6] = {passes > 1 ? (size_t)n_win * px : 0, (size_t)n_win * K, (size_t)n_win * K, (size_t)n_win,
                           (size_t)n_win * F, (size_t)n_win * F};
  size_t off = 0;
  float** slots[6] = {&s->b, &s->d2, &s->wts, &s->sig, &s->sa, &s->sb};
  for (int i = 0; i < 6; ++i) {
    if (base) *slots[i] = (float*)(base + off);
    off += ((sizes[i] * sizeof(float) + 255) / 256) * 256;
  }
  return off;
}

}  // namespace zeb

using namespace zeb;

extern "C" size_t zeb_nlpar_scratch_bytes(int n_win, int px, int radius, int passes) {
  if (n_win <= 0 || px <= 0 || radius < 1 || passes < 1) return 0;
  NlScratch s{};
  return nl_layout(n_win, px, radius, passes, nullptr, &s);
}

extern "C" int zeb_nlpar(float* patterns, int px, const uint32_t* nbr, const int* counts, int radius, int passes,
                         float lambda, float* out, float* sig_out, float* shares_out, void* scratch, void* stream) {
  ZEB_REQUIRE(patterns && nbr && counts && out && scratch && px > 0 && radius >= 1 && passes >= 1 &&
                  radius * passes <= 8 && lambda > 0.f,
              ZEB_EARG, "nlpar: bad arguments");
  const int rings = radius * passes + 1;
  for (int d = 1; d <= rings; ++d)
    ZEB_REQUIRE(counts[d] >= counts[d - 1] && counts[0] >= 0, ZEB_EARG, "nlpar: counts must not decrease");
  const int n_win = counts[rings];
  if (counts[0] == 0) return ZEB_OK;
  NlScratch s{};
  nl_layout(n_win, px, radius, passes, (char*)scratch, &s);
  cudaStream_t st = (cudaStream_t)stream;
  const int K = (2 * radius + 1) * (2 * radius + 1);
  const int F = (2 * radius * passes + 1) * (2 * radius * passes + 1);
  NlArgs a{};
  a.nbr = nbr; a.d2 = s.d2; a.sig = s.sig; a.wts = s.wts;
  a.px = px; a.radius = radius; a.reach = radius * passes;
  a.inv_l2 = (float)(1.0 / ((double)lambda * lambda));
  a.sqn = (float)sqrt(0.5 * (double)px);
  float* src = patterns;
  float* dst = s.b;
  float* s_in = s.sa;
  float* s_out = s.sb;
  for (int t = 1; t <= passes; ++t) {
    const int d = (passes - t) * radius;
    a.spread = (t - 1) * radius;
    a.pin = src;
    a.share_in = s_in;
    a.share = s_out;
    // the differences of every pair a weight below reads (in the first pass, of every pair a
    // noise reads too: all of them)
    a.n = counts[t == 1 ? rings : d + radius];
    if (a.n > 0) k_nl_distance<<<(unsigned)((long long)a.n * (K / 2)), 256, 0, st>>>(a);
    if (t == 1) {
      a.n = counts[rings - 1];
      if (a.n > 0) k_nl_sigma<<<(a.n + 63) / 64, 64, 0, st>>>(a);
    }
    a.n = counts[d];
    if (a.n > 0) {
      k_nl_weights<<<(a.n + 63) / 64, 64, 0, st>>>(a);
      const bool last = t == passes;
      a.pout = last ? out : dst;
      a.out0 = 0;
      k_nl_average<<<nl_grid((long long)a.n * px), 256, 0, st>>>(a);
      k_nl_shares<<<nl_grid((long long)a.n * F), 256, 0, st>>>(a);
    }
    float* tmp = src; src = dst; dst = tmp;
    tmp = s_in; s_in = s_out; s_out = tmp;
  }
  // what the averaging did, when asked: the stored patterns' noise (the cells within rings − 1)
  // and the wanted averages' shares of the stored patterns
  if (sig_out && cudaMemcpyAsync(sig_out, s.sig, sizeof(float) * counts[rings - 1], cudaMemcpyDeviceToDevice, st) !=
                     cudaSuccess)
    return zeb_launch_check("nlpar noise");
  if (shares_out && cudaMemcpyAsync(shares_out, s_in, sizeof(float) * (size_t)counts[0] * F, cudaMemcpyDeviceToDevice,
                                    st) != cudaSuccess)
    return zeb_launch_check("nlpar shares");
  return zeb_launch_check("nlpar");
}
