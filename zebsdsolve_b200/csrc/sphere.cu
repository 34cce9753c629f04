// (a) Patterns onto the sphere and into spherical harmonics.
//
// k_sphere_rings: one thread block per item. The pattern sits in shared memory; every Gauss–
// Legendre direction's ray is intersected with the detector plane and the pattern sampled
// bilinearly there (zero off the detector and outside the mask).  A first pass takes the
// window's quadrature-weighted sums (its area and mean); the second takes each northern ring
// with its mirror as one complex line (ring real, mirror imaginary), window-mean centred,
// transforms it along φ in shared memory and keeps of the two spectra their orders m < L as
// sum and difference (sphere.wgsl:128-269).
// With ring spans (zeb_sphere_spans: per ring the cyclic run of φ samples that can meet the
// detector, with a margin), only those samples are taken; a ring whose span's end samples are
// themselves on the detector (the span did not cover this item) is taken whole, so the result
// equals the full sampling.  Ring pairs with no samples get zero spectra without a transform.
// k_legendre: contracts the ring spectra with the weighted Legendre table, a block per
// (order m, tile of items) with the table's rows for m staged in shared memory (sphere.wgsl:
// 271-288). k_sh_norm: unit harmonic norm and the item's stats (sphere.wgsl:290-324).
#include <algorithm>

#include "abi_util.cuh"

namespace zeb {

struct SphereArgs {
  const float* pats;
  const float4* items;
  int n_items, h, w;
  float c0[3], c1[3], c2[3], mask[3];
  int L, n_theta, n_phi, lg_phi, n_pairs;
  const float4* ring;
  const float2* phi_cs;
  const float* wplm;
  const float2* tw;
  unsigned flags;
  float4* spectra;  // [item][n_theta/2][L]
  float2* alm;      // [item][n_pairs]
  float* stats;     // [item][4]
  int lines_per_chunk;
  int pat_in_smem;
  const int2* spans;  // [n_theta] (first φ sample, count), cyclic; null: every sample
  int ring_major;     // spectra laid out [item][m][ring pair] (else [item][ring pair][m])
  int leg_items;      // items per k_legendre block (a multiple of 4)
  int cache_cap;      // k_sphere_rings_w: samples its shared cache holds (0: none)
};

struct Sampler {
  const float* pat;
  int h, w;
  float3 c0, c1, c2, t;
  float c2t;
  float mask[3];
  bool window;

  // (pattern value, window weight) of direction d (sphere.wgsl:128-163)
  __device__ __forceinline__ float2 sample(float3 d) const {
    float nd = dot3(c2, d);
    float val = 0.f, wv = 0.f;
    if (nd > 1e-4f) {
      float s = c2t / nd;
      float3 hh = make_float3(s * d.x - t.x, s * d.y - t.y, s * d.z - t.z);
      float row = dot3(c0, hh), col = dot3(c1, hh);
      float hmax = (float)(h - 1), wmax = (float)(w - 1);
      float dr = row - mask[0], dc = col - mask[1];
      if (row >= 0.f && row <= hmax && col >= 0.f && col <= wmax && zeb_in_circle(dr, dc, mask[2])) {
        wv = 1.f;
        val = 1.f;
        if (!window) {
          int r0 = min((int)row, h - 2), q0 = min((int)col, w - 2);
          float fr = row - (float)r0, fc = col - (float)q0;
          const float* p = pat + r0 * w + q0;
          float top = lerpf(p[0], p[1], fc), bot = lerpf(p[w], p[w + 1], fc);
          val = lerpf(top, bot, fr);
        }
      }
    }
    return make_float2(val, wv);
  }
};

// index of the last prefix entry <= e (prefix[0] = 0, non-decreasing, n + 1 entries)
__device__ __forceinline__ int span_of(const int* prefix, int n, int e) {
  int lo = 0, hi = n;  // prefix[lo] <= e < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

constexpr int SPH_MAX_THETA = 512;

__global__ void __launch_bounds__(256) k_sphere_rings(SphereArgs a) {
  extern __shared__ float4 smem4[];
  __shared__ float red[2 * 8];
  __shared__ int2 sp[SPH_MAX_THETA];        // this item's spans (whole rings where a span fell short)
  __shared__ int pre[SPH_MAX_THETA + 1];    // prefix sums of span counts
  __shared__ int act[SPH_MAX_THETA / 2];    // ring pairs with samples
  __shared__ int n_act;
  const int b = blockIdx.x;
  const int hw = a.h * a.w;
  float2* lines = (float2*)smem4;
  float* spat = (float*)(lines + (size_t)a.lines_per_chunk * a.n_phi);
  const float4 it = a.items[b];
  const bool window = (a.flags & ZEB_FLAG_WINDOW) != 0;
  Sampler s;
  s.pat = nullptr;
  if (!window) {
    const float* src = a.pats + (size_t)(int)it.w * hw;
    if (a.pat_in_smem) {
      for (int i = threadIdx.x; i < hw; i += blockDim.x) spat[i] = src[i];
      s.pat = spat;
    } else {
      s.pat = src;
    }
  }
  s.h = a.h; s.w = a.w;
  s.c0 = make_float3(a.c0[0], a.c0[1], a.c0[2]);
  s.c1 = make_float3(a.c1[0], a.c1[1], a.c1[2]);
  s.c2 = make_float3(a.c2[0], a.c2[1], a.c2[2]);
  s.t = make_float3(it.x, it.y, it.z);
  s.c2t = dot3(s.c2, s.t);
  s.mask[0] = a.mask[0]; s.mask[1] = a.mask[1]; s.mask[2] = a.mask[2];
  s.window = window;
  const int nphi = a.n_phi, nt = a.n_theta, lg = a.lg_phi, nh = nt / 2, L = a.L;
  const int pmask = nphi - 1;

  // spans: the table's, widened to the whole ring where an end sample is on the detector
  for (int y = threadIdx.x; y < nt; y += blockDim.x) {
    int2 v = a.spans ? a.spans[y] : make_int2(0, nphi);
    if (v.y > 0 && v.y < nphi) {
      const float4 rg = __ldg(a.ring + y);
      const float2 c0 = __ldg(a.phi_cs + (v.x & pmask)), c1 = __ldg(a.phi_cs + ((v.x + v.y - 1) & pmask));
      const float w0 = s.sample(make_float3(rg.y * c0.x, rg.y * c0.y, rg.x)).y;
      const float w1 = s.sample(make_float3(rg.y * c1.x, rg.y * c1.y, rg.x)).y;
      if (w0 > 0.f || w1 > 0.f) v = make_int2(0, nphi);
    }
    sp[y] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0, na = 0;
    for (int y = 0; y < nt; ++y) {
      pre[y] = acc;
      acc += sp[y].y;
    }
    pre[nt] = acc;
    for (int y = 0; y < nh; ++y)
      if (sp[y].y > 0 || sp[nt - 1 - y].y > 0) act[na++] = y;
    n_act = na;
  }
  __syncthreads();

  // the window's sums over the spans
  float acc[2] = {0.f, 0.f};
  const int total = pre[nt];
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int y = span_of(pre, nt, e);
    const int j = (sp[y].x + (e - pre[y])) & pmask;
    float4 rg = __ldg(a.ring + y);
    float2 cs = __ldg(a.phi_cs + j);
    float2 g = s.sample(make_float3(rg.y * cs.x, rg.y * cs.y, rg.x));
    acc[0] += g.x * g.y * rg.z;
    acc[1] += g.y * rg.z;
  }
  block_sums<2>(acc, red);
  const float mean = (a.flags & ZEB_FLAG_CENTER) ? acc[0] / fmaxf(acc[1], 1e-20f) : 0.f;
  if (threadIdx.x == 0) {
    a.stats[b * 4 + 0] = acc[1] * ZEB_TAU / (float)nphi;
    a.stats[b * 4 + 1] = mean;
  }

  // ring pairs without samples: zero spectra
  float4* outb = a.spectra + (size_t)b * nh * L;
  for (int e = threadIdx.x; e < nh * L; e += blockDim.x) {
    const int y = e / L;
    if (sp[y].y == 0 && sp[nt - 1 - y].y == 0) outb[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }

  // the others, a chunk of lines at a time: slot i holds pair act[c0 + i] (ring real, mirror
  // imaginary), zero where not sampled
  const int na = n_act;
  const int CH = a.lines_per_chunk;
  RowLines idx{lg};
  __shared__ int cpre[2 * 64 + 1];  // (slot, side) prefix of the chunk; lines_per_chunk <= 64
  for (int c0 = 0; c0 < na; c0 += CH) {
    const int cnt = min(CH, na - c0);
    for (int e = threadIdx.x; e < cnt * nphi; e += blockDim.x) lines[e] = make_float2(0.f, 0.f);
    if (threadIdx.x == 0) {
      int q = 0;
      for (int k = 0; k < 2 * cnt; ++k) {
        cpre[k] = q;
        const int y = act[c0 + (k >> 1)];
        q += sp[(k & 1) ? nt - 1 - y : y].y;
      }
      cpre[2 * cnt] = q;
    }
    __syncthreads();
    const int ctot = cpre[2 * cnt];
    for (int e = threadIdx.x; e < ctot; e += blockDim.x) {
      const int k = span_of(cpre, 2 * cnt, e);
      const int i = k >> 1, side = k & 1;
      const int y = side ? nt - 1 - act[c0 + i] : act[c0 + i];
      const int j = (sp[y].x + (e - cpre[k])) & pmask;
      const float4 rg = __ldg(a.ring + y);
      const float2 cs = __ldg(a.phi_cs + j);
      const float2 g = s.sample(make_float3(rg.y * cs.x, rg.y * cs.y, rg.x));
      ((float*)&lines[idx(i, bitrev(j, lg))])[side] = (g.x - mean) * g.y;
    }
    __syncthreads();
    fft_lines_smem(lines, cnt, lg, a.tw, idx);
    // the two apart: Z = N + iS for real N, S gives N_m = (Z_m + conj Z_{n−m})/2 and
    // S_m = (Z_m − conj Z_{n−m})/2i; keep (N+S, N−S) for m < L
    for (int e = threadIdx.x; e < cnt * L; e += blockDim.x) {
      int i = e / L, m = e - i * L;
      float2 z = lines[idx(i, m)];
      float2 zr = lines[idx(i, (nphi - m) & (nphi - 1))];
      float2 rn = make_float2(0.5f * (z.x + zr.x), 0.5f * (z.y - zr.y));
      float2 dd = make_float2(z.x - zr.x, z.y + zr.y);
      float2 rs = make_float2(0.5f * dd.y, -0.5f * dd.x);
      outb[(size_t)act[c0 + i] * L + m] = make_float4(rn.x + rs.x, rn.y + rs.y, rn.x - rs.x, rn.y - rs.y);
    }
    __syncthreads();
  }
}

// forward 8-point DFT in registers (radix-2, decimation in time, natural order in and out)
__device__ __forceinline__ void fft_reg8(float2 (&x)[8]) {
  const float r = 0.70710678118654752f;
  float2 t;
  t = x[1]; x[1] = x[4]; x[4] = t;
  t = x[3]; x[3] = x[6]; x[6] = t;
#pragma unroll
  for (int i = 0; i < 8; i += 2) {
    const float2 p = x[i], q = x[i + 1];
    x[i] = make_float2(p.x + q.x, p.y + q.y);
    x[i + 1] = make_float2(p.x - q.x, p.y - q.y);
  }
#pragma unroll
  for (int i = 0; i < 8; i += 4) {
    float2 p = x[i], q = x[i + 2];
    x[i] = make_float2(p.x + q.x, p.y + q.y);
    x[i + 2] = make_float2(p.x - q.x, p.y - q.y);
    p = x[i + 1];
    q = make_float2(x[i + 3].y, -x[i + 3].x);  // × e^{−iπ/2}
    x[i + 1] = make_float2(p.x + q.x, p.y + q.y);
    x[i + 3] = make_float2(p.x - q.x, p.y - q.y);
  }
  {
    float2 p = x[0], q = x[4];
    x[0] = make_float2(p.x + q.x, p.y + q.y);
    x[4] = make_float2(p.x - q.x, p.y - q.y);
    p = x[1];
    q = make_float2(r * (x[5].x + x[5].y), r * (x[5].y - x[5].x));  // × e^{−iπ/4}
    x[1] = make_float2(p.x + q.x, p.y + q.y);
    x[5] = make_float2(p.x - q.x, p.y - q.y);
    p = x[2];
    q = make_float2(x[6].y, -x[6].x);  // × e^{−iπ/2}
    x[2] = make_float2(p.x + q.x, p.y + q.y);
    x[6] = make_float2(p.x - q.x, p.y - q.y);
    p = x[3];
    q = make_float2(r * (x[7].y - x[7].x), -r * (x[7].x + x[7].y));  // × e^{−3iπ/4}
    x[3] = make_float2(p.x + q.x, p.y + q.y);
    x[7] = make_float2(p.x - q.x, p.y - q.y);
  }
}

// ── the rings of one item, a warp per ring pair, for n_φ = 256 ──
//
// The block holds the item's pattern and the φ cosines; the window sums (over the spans) sample
// every direction once and keep each sample in a shared cache (span order: ring y's samples from
// the prefix sum of the spans before it), the value where the window holds it and a marker where
// it does not; the transforms then read the cache, and their lines take the pattern's shared
// memory.  Where an item's spans hold more samples than the cache (a span that fell short makes
// its ring whole), the transforms sample again, from the pattern in global memory.
// Each warp takes one ring pair with samples at a time: it zeroes its 256-point line, fills the
// northern ring (real part) and its mirror (imaginary part) over their spans, and transforms the
// line with no block barrier, in three register steps with the line between them (8-point DFTs
// over the stride-32 points, 8-point DFTs of the 32-point transforms' quarters, their 4-point sums,
// only for the orders kept), and the lanes split N and S for m < L.  Spectra are written [item][m][ring pair].
constexpr int RW_WARPS = 8;
constexpr int RW_PAD = 256 + 32;  // line slots per warp: F + F/8
constexpr int RW_CACHE = 7168;    // cached samples (28 KB): the spans of a 60 × 60 or 80 × 80 frame
constexpr uint32_t RW_OUT = 0x7fc0dea1u;  // cache marker of a sample outside the window: a NaN no
                                          // arithmetic produces (computed NaNs are canonical)

__device__ __forceinline__ int rw_slot(int f) { return f + (f >> 3); }

__global__ void __launch_bounds__(RW_WARPS * 32) k_sphere_rings_w(SphereArgs a) {
  extern __shared__ float4 smem4[];
  __shared__ float red[2 * 8];
  __shared__ int2 sp[SPH_MAX_THETA];
  __shared__ int pre[SPH_MAX_THETA + 1];
  __shared__ int act[SPH_MAX_THETA / 2];
  __shared__ int n_act;
  __shared__ float2 pcs[256];
  const int b = blockIdx.x;
  const int hw = a.h * a.w;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // dynamic shared memory: [the pattern (sampling), then the lines (transforms)] [the cache]
  float2* lines = (float2*)smem4;  // [RW_WARPS][RW_PAD]
  float* spat = (float*)smem4;
  const int region = max(RW_WARPS * RW_PAD * 2, a.pat_in_smem ? hw : 0);  // floats
  float* cache = (float*)smem4 + region;
  const float4 it = a.items[b];
  const bool window = (a.flags & ZEB_FLAG_WINDOW) != 0;
  const float* src = window ? nullptr : a.pats + (size_t)(int)it.w * hw;
  Sampler s;
  s.pat = nullptr;
  if (!window) {
    if (a.pat_in_smem) {
      for (int i = threadIdx.x; i < hw; i += blockDim.x) spat[i] = src[i];
      s.pat = spat;
    } else {
      s.pat = src;
    }
  }
  s.h = a.h; s.w = a.w;
  s.c0 = make_float3(a.c0[0], a.c0[1], a.c0[2]);
  s.c1 = make_float3(a.c1[0], a.c1[1], a.c1[2]);
  s.c2 = make_float3(a.c2[0], a.c2[1], a.c2[2]);
  s.t = make_float3(it.x, it.y, it.z);
  s.c2t = dot3(s.c2, s.t);
  s.mask[0] = a.mask[0]; s.mask[1] = a.mask[1]; s.mask[2] = a.mask[2];
  s.window = window;
  constexpr int nphi = 256, pmask = 255;
  const int nt = a.n_theta, nh = nt / 2, L = a.L;
  for (int j = threadIdx.x; j < nphi; j += blockDim.x) pcs[j] = __ldg(a.phi_cs + j);
  __syncthreads();

  for (int y = threadIdx.x; y < nt; y += blockDim.x) {
    int2 v = a.spans ? a.spans[y] : make_int2(0, nphi);
    if (v.y > 0 && v.y < nphi) {
      const float4 rg = __ldg(a.ring + y);
      const float2 c0 = pcs[v.x & pmask], c1 = pcs[(v.x + v.y - 1) & pmask];
      const float w0 = s.sample(make_float3(rg.y * c0.x, rg.y * c0.y, rg.x)).y;
      const float w1 = s.sample(make_float3(rg.y * c1.x, rg.y * c1.y, rg.x)).y;
      if (w0 > 0.f || w1 > 0.f) v = make_int2(0, nphi);
    }
    sp[y] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0, na = 0;
    for (int y = 0; y < nt; ++y) {
      pre[y] = acc;
      acc += sp[y].y;
    }
    pre[nt] = acc;
    for (int y = 0; y < nh; ++y)
      if (sp[y].y > 0 || sp[nt - 1 - y].y > 0) act[na++] = y;
    n_act = na;
  }
  __syncthreads();

  // the window's sums over the spans, a warp per ring pair as below (no search for a flat
  // index's ring); each sample into the cache when the item's spans fit it
  const bool cached = pre[nt] <= a.cache_cap;
  float acc[2] = {0.f, 0.f};
  for (int ai = warp; ai < n_act; ai += RW_WARPS) {
    const int y2[2] = {act[ai], nt - 1 - act[ai]};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float4 rg = __ldg(a.ring + y2[h]);
      const int2 v = sp[y2[h]];
      float* cy = cache + pre[y2[h]];
      for (int e = lane; e < v.y; e += 32) {
        const float2 cs = pcs[(v.x + e) & pmask];
        const float2 g = s.sample(make_float3(rg.y * cs.x, rg.y * cs.y, rg.x));
        acc[0] += g.x * g.y * rg.z;
        acc[1] += g.y * rg.z;
        if (cached) cy[e] = g.y > 0.f ? g.x : __uint_as_float(RW_OUT);
      }
    }
  }
  block_sums<2>(acc, red);  // (its barriers also end every read of the pattern in shared memory)
  if (!cached && a.pat_in_smem) s.pat = src;  // the lines take the pattern's shared memory
  const float mean = (a.flags & ZEB_FLAG_CENTER) ? acc[0] / fmaxf(acc[1], 1e-20f) : 0.f;
  if (threadIdx.x == 0) {
    a.stats[b * 4 + 0] = acc[1] * ZEB_TAU / (float)nphi;
    a.stats[b * 4 + 1] = mean;
  }

  float4* outb = a.spectra + (size_t)b * L * nh;  // [m][ring pair]
  for (int e = threadIdx.x; e < nh * L; e += blockDim.x) {
    const int m = e / nh, y = e - m * nh;
    if (sp[y].y == 0 && sp[nt - 1 - y].y == 0) outb[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }

  // this lane's twiddles: e^{−2πi l k/256} (the 256-point step, l = lane) and e^{−2πi a c/32}
  // (the 32-point step, a = lane mod 4), k, c < 8
  float2 tw8[8], tw32[8];
  const int grp = lane >> 2, qa = lane & 3;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    tw8[k] = __ldg(a.tw + ((lane * k * 4) & (ZEB_TW_LEN - 1)));
    tw32[k] = __ldg(a.tw + ((qa * k * (ZEB_TW_LEN / 32)) & (ZEB_TW_LEN - 1)));
  }
  float2* buf = lines + warp * RW_PAD;
  const int na = n_act;
  for (int ai = warp; ai < na; ai += RW_WARPS) {
    const int y = act[ai], ys = nt - 1 - y;
#pragma unroll
    for (int k = 0; k < 8; ++k) buf[lane + 32 * k] = make_float2(0.f, 0.f);
    __syncwarp();
    if (cached) {
      const int2 vn = sp[y], vs = sp[ys];
      const float* cn = cache + pre[y];
      const float* cq = cache + pre[ys];
      for (int e = lane; e < vn.y; e += 32) {
        const float c = cn[e];
        buf[(vn.x + e) & pmask].x = __float_as_uint(c) == RW_OUT ? 0.f : c - mean;
      }
      for (int e = lane; e < vs.y; e += 32) {
        const float c = cq[e];
        buf[(vs.x + e) & pmask].y = __float_as_uint(c) == RW_OUT ? 0.f : c - mean;
      }
    } else {
      {
        const float4 rg = __ldg(a.ring + y);
        const int2 v = sp[y];
        for (int e = lane; e < v.y; e += 32) {
          const int j = (v.x + e) & pmask;
          const float2 cs = pcs[j];
          const float2 g = s.sample(make_float3(rg.y * cs.x, rg.y * cs.y, rg.x));
          buf[j].x = (g.x - mean) * g.y;
        }
      }
      {
        const float4 rg = __ldg(a.ring + ys);
        const int2 v = sp[ys];
        for (int e = lane; e < v.y; e += 32) {
          const int j = (v.x + e) & pmask;
          const float2 cs = pcs[j];
          const float2 g = s.sample(make_float3(rg.y * cs.x, rg.y * cs.y, rg.x));
          buf[j].y = (g.x - mean) * g.y;
        }
      }
    }
    __syncwarp();
    // X[m] = Σ_j x[j] W^{jm} (W = e^{−2πi/256}) with j = j1 + 32 j2, m = m2 + 8 m1:
    // (1) lane j1: the 8-point DFTs over j2, × W^{j1 m2} → Z[j1][m2] (to the line, 9 a row);
    // (2) lane (m2, a) of the 8 groups of 4: with j1 = a + 4b and m1 = c + 8d, the 8-point DFT over
    //     b of Z[a + 4b][m2], × e^{−2πi a c/32} → V[m2][a][c] (to the line);
    // (3) lane (m2, a) finishes c = 2a, 2a + 1: the 4-point sums over a for d = 0 and d = 3 only,
    //     m = m2 + 8c + 64d: the orders m < 64 and 256 − m the split below reads (n_φ = 256 means
    //     L ≤ 64), written at rw_slot(m)
    float2 x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = buf[lane + 32 * k];
    fft_reg8(x);
#pragma unroll
    for (int k = 1; k < 8; ++k) x[k] = cmulf(x[k], tw8[k]);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k) buf[lane * 9 + k] = x[k];
    __syncwarp();
#pragma unroll
    for (int b = 0; b < 8; ++b) x[b] = buf[(qa + 4 * b) * 9 + grp];
    fft_reg8(x);
#pragma unroll
    for (int c = 1; c < 8; ++c) x[c] = cmulf(x[c], tw32[c]);
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 8; ++c) buf[(grp * 4 + qa) * 9 + c] = x[c];
    __syncwarp();
    float2 o0[2], o3[2];
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int c = 2 * qa + hh;
      const float2 v0 = buf[(grp * 4 + 0) * 9 + c], v1 = buf[(grp * 4 + 1) * 9 + c];
      const float2 v2 = buf[(grp * 4 + 2) * 9 + c], v3 = buf[(grp * 4 + 3) * 9 + c];
      o0[hh] = make_float2(v0.x + v1.x + v2.x + v3.x, v0.y + v1.y + v2.y + v3.y);
      // d = 3: the weights e^{−2πi 3a/4} = 1, i, −1, −i
      o3[hh] = make_float2(v0.x - v1.y - v2.x + v3.y, v0.y + v1.x - v2.y - v3.x);
    }
    __syncwarp();
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int m = grp + 8 * (2 * qa + hh);
      buf[rw_slot(m)] = o0[hh];
      buf[rw_slot(m + 192)] = o3[hh];
    }
    __syncwarp();
    // the two apart: Z = N + iS for real N, S gives N_m = (Z_m + conj Z_{n−m})/2 and
    // S_m = (Z_m − conj Z_{n−m})/2i; keep (N+S, N−S) for m < L
    for (int m = lane; m < L; m += 32) {
      const float2 z = buf[rw_slot(m)];
      const float2 zr = buf[rw_slot((nphi - m) & pmask)];
      const float2 rn = make_float2(0.5f * (z.x + zr.x), 0.5f * (z.y - zr.y));
      const float2 dd = make_float2(z.x - zr.x, z.y + zr.y);
      const float2 rs = make_float2(0.5f * dd.y, -0.5f * dd.x);
      outb[(size_t)m * nh + y] = make_float4(rn.x + rs.x, rn.y + rs.y, rn.x - rs.x, rn.y - rs.y);
    }
    __syncwarp();
  }
}

// Spans of the sphere's rings for a set of detector positions: per ring, the shortest cyclic run
// of φ samples holding every sample that meets the masked detector for any of the n_t positions,
// widened by `margin` samples on each side ((0, 0): none; (0, n_φ): the whole ring).
__global__ void k_sphere_spans(SphereArgs a, const float4* __restrict__ ts, int n_t, int margin, int2* spans) {
  __shared__ unsigned char hit[ZEB_TW_LEN];
  const int y = blockIdx.x, nphi = a.n_phi;
  const float4 rg = __ldg(a.ring + y);
  Sampler s;
  s.pat = nullptr;
  s.h = a.h; s.w = a.w;
  s.c0 = make_float3(a.c0[0], a.c0[1], a.c0[2]);
  s.c1 = make_float3(a.c1[0], a.c1[1], a.c1[2]);
  s.c2 = make_float3(a.c2[0], a.c2[1], a.c2[2]);
  s.mask[0] = a.mask[0]; s.mask[1] = a.mask[1]; s.mask[2] = a.mask[2];
  s.window = true;
  for (int j = threadIdx.x; j < nphi; j += blockDim.x) {
    const float2 cs = __ldg(a.phi_cs + j);
    const float3 d = make_float3(rg.y * cs.x, rg.y * cs.y, rg.x);
    unsigned char h = 0;
    for (int k = 0; k < n_t; ++k) {
      s.t = make_float3(ts[k].x, ts[k].y, ts[k].z);
      s.c2t = dot3(s.c2, s.t);
      if (s.sample(d).y > 0.f) h = 1;
    }
    hit[j] = h;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // the longest cyclic run of misses; the span is its complement
    int first = -1;
    for (int j = 0; j < nphi; ++j)
      if (hit[j]) { first = j; break; }
    int2 out = make_int2(0, 0);
    if (first >= 0) {
      int best = 0, best_end = first, run = 0;
      for (int k = 1; k <= nphi; ++k) {
        const int j = (first + k) % nphi;
        if (hit[j]) {
          if (run > best) { best = run; best_end = j; }
          run = 0;
        } else {
          ++run;
        }
      }
      // hits lie in [best_end, best_end + nphi − best): start after the longest gap
      int start = best_end, count = nphi - best;
      start -= margin;
      count += 2 * margin;
      if (count >= nphi) out = make_int2(0, nphi);
      else out = make_int2(((start % nphi) + nphi) % nphi, count);
    }
    spans[y] = out;
  }
}

// a_lm = Σ_y wplm[y, pair] · (N+S or N−S by the parity of l+m): block (m, tile of 16 items).
// A block per (order m, group of leg_items items): the group's ring spectra of order m and the
// table column wplm[y][pair(m, l)] go to shared memory; a thread then takes a tile of 4 items ×
// 4 degrees l and walks the ring pairs y: per y, four 16-byte spectrum loads (shared by the
// lanes of an item group) and one 16-byte load of four table entries feed 32 FMAs.  The tile's
// first degree has l + m even, so its 2nd and 4th degrees take the odd ring combination
// (N − S) and the others the even one (N + S).  Each coefficient sums over y in increasing order
// (fmaf), as a thread per coefficient would.
constexpr int LEG_THREADS = 128;

// asynchronous global → shared copies of 16 or 4 bytes; `bytes` of them read, the rest zero-filled
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__host__ __device__ inline int leg_nlp(int nl) { return (nl + 3) & ~3; }

__global__ void __launch_bounds__(LEG_THREADS) k_legendre(SphereArgs a) {
  extern __shared__ float4 smem4[];
  const int m = blockIdx.x;
  const int G = a.leg_items;
  const int b0 = blockIdx.y * G;
  const int L = a.L, nh = a.n_theta / 2, np = a.n_pairs;
  const int nl = L - m, nlp = leg_nlp(nl);
  const int p0 = m * L - (m * (m - 1)) / 2;
  float4* spec = smem4;                   // [G][nh]
  float* wp = (float*)(spec + G * nh);    // [nh][nlp]
  const int nb = min(G, a.n_items - b0);
  // both through asynchronous copies (cp.async: no round trip through registers, every copy of
  // the thread in flight at once); entries past the items or the degrees are zero-filled
  for (int e = threadIdx.x; e < G * nh; e += blockDim.x) {
    int i = e / nh, y = e - i * nh;
    const float4* src = a.spectra;
    if (i < nb)
      src += a.ring_major ? ((size_t)(b0 + i) * L + m) * nh + y : ((size_t)(b0 + i) * nh + y) * L + m;
    cp_async16(spec + e, src, i < nb ? 16 : 0);
  }
  for (int e = threadIdx.x; e < nh * nlp; e += blockDim.x) {
    int y = e / nlp, l = e - y * nlp;
    cp_async4(wp + e, a.wplm + (l < nl ? (size_t)y * np + p0 + l : 0), l < nl ? 4 : 0);
  }
  cp_async_wait_all();
  __syncthreads();
  const int nlg = nlp / 4, tiles = (G / 4) * nlg;
  for (int t = threadIdx.x; t < tiles; t += blockDim.x) {
    const int lg = t % nlg, ig = t / nlg;
    float re[4][4], im[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int j = 0; j < 4; ++j) re[k][j] = im[k][j] = 0.f;
    const float4* sp = spec + (size_t)ig * 4 * nh;
    const float* wq = wp + lg * 4;
#pragma unroll 2
    for (int y = 0; y < nh; ++y) {
      const float4 w4 = *(const float4*)(wq + (size_t)y * nlp);
      const float wj[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 r = sp[k * nh + y];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          re[k][j] = fmaf(wj[j], (j & 1) ? r.z : r.x, re[k][j]);
          im[k][j] = fmaf(wj[j], (j & 1) ? r.w : r.y, im[k][j]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = ig * 4 + k;
      if (i >= nb) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int l = lg * 4 + j;
        if (l < nl) a.alm[(size_t)(b0 + i) * np + p0 + l] = make_float2(re[k][j], im[k][j]);
      }
    }
  }
}

// unit harmonic norm (Σ over signed orders: m > 0 twice) and the stats
__global__ void __launch_bounds__(256) k_sh_norm(SphereArgs a) {
  __shared__ float red[8];
  const int b = blockIdx.x;
  const int L = a.L, np = a.n_pairs;
  float2* al = a.alm + (size_t)b * np;
  float e[1] = {0.f};
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    float2 v = al[p];
    float k = p < L ? 1.f : 2.f;  // pairs 0 … L−1 are m = 0
    e[0] += k * (v.x * v.x + v.y * v.y);
  }
  block_sums<1>(e, red);
  const float nrm = sqrtf(fmaxf(e[0], 1e-30f));
  if (a.flags & ZEB_FLAG_NORM) {
    const float inv = 1.f / nrm;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
      float2 v = al[p];
      al[p] = make_float2(v.x * inv, v.y * inv);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a.stats[b * 4 + 2] = nrm;
    a.stats[b * 4 + 3] = al[0].x;
  }
}

static int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

}  // namespace zeb

using namespace zeb;

extern "C" size_t zeb_sphere_scratch_bytes(const zeb_sphere_tables_t* tb, int n_items) {
  if (!tb || n_items <= 0) return 0;
  return (size_t)n_items * (tb->n_theta / 2) * tb->L * sizeof(float4);
}

static bool sphere_fill(SphereArgs& a, const zeb_frame_t* fr, const zeb_sphere_tables_t* tb) {
  const int L = tb->L, nphi = tb->n_phi, nt = tb->n_theta;
  if (!(L >= 2 && L <= 256 && nt >= 2 * L - 1 && nt <= SPH_MAX_THETA && (nphi & (nphi - 1)) == 0 && nphi >= 32 &&
        nphi <= ZEB_TW_LEN && nt % 2 == 0 && tb->n_pairs == L * (L + 1) / 2 && fr->h >= 2 && fr->w >= 2 &&
        L <= nphi / 2))
    return false;
  a.h = fr->h; a.w = fr->w;
  for (int k = 0; k < 3; ++k) {
    a.c0[k] = fr->c0[k]; a.c1[k] = fr->c1[k]; a.c2[k] = fr->c2[k]; a.mask[k] = fr->mask[k];
  }
  a.L = L; a.n_theta = nt; a.n_phi = nphi; a.lg_phi = ilog2(nphi); a.n_pairs = tb->n_pairs;
  a.ring = (const float4*)tb->ring; a.phi_cs = (const float2*)tb->phi_cs; a.wplm = tb->wplm;
  a.tw = (const float2*)tb->tw;
  return true;
}

extern "C" int zeb_sphere_spans(const zeb_frame_t* fr, const zeb_sphere_tables_t* tb, const float* ts, int n_t,
                                int margin, int* spans, void* stream) {
  ZEB_REQUIRE(fr && tb && ts && spans && n_t >= 1 && n_t <= 64 && margin >= 0, ZEB_EARG, "sphere_spans: bad arguments");
  ZEB_REQUIRE(tb->ring && tb->phi_cs, ZEB_EARG, "sphere_spans: table missing");
  SphereArgs a{};
  ZEB_REQUIRE(sphere_fill(a, fr, tb), ZEB_EARG, "sphere_spans: bad tables");
  k_sphere_spans<<<tb->n_theta, 256, 0, (cudaStream_t)stream>>>(a, (const float4*)ts, n_t, margin, (int2*)spans);
  return zeb_launch_check("sphere_spans");
}

extern "C" int zeb_sphere_coefficients(const float* pats, const float* items, int n_items, const zeb_frame_t* fr,
                                       const zeb_sphere_tables_t* tb, unsigned flags, float* alm, float* stats,
                                       void* scratch, void* stream) {
  return zeb_sphere_coefficients_spans(pats, items, n_items, fr, tb, nullptr, flags, alm, stats, scratch, stream);
}

extern "C" int zeb_sphere_coefficients_spans(const float* pats, const float* items, int n_items, const zeb_frame_t* fr,
                                             const zeb_sphere_tables_t* tb, const int* spans, unsigned flags,
                                             float* alm, float* stats, void* scratch, void* stream) {
  ZEB_REQUIRE(items && fr && tb && alm && stats && scratch, ZEB_EARG, "sphere_coefficients: null argument");
  ZEB_REQUIRE((flags & ZEB_FLAG_WINDOW) || pats, ZEB_EARG, "sphere_coefficients: patterns missing");
  ZEB_REQUIRE(tb->ring && tb->phi_cs && tb->wplm && tb->tw, ZEB_EARG, "sphere_coefficients: table missing");
  const int L = tb->L, nphi = tb->n_phi, nt = tb->n_theta;
  SphereArgs a{};
  ZEB_REQUIRE(sphere_fill(a, fr, tb), ZEB_EARG, "sphere_coefficients: bad tables L=%d nt=%d nphi=%d", L, nt, nphi);
  if (n_items == 0) return ZEB_OK;
  a.pats = pats; a.items = (const float4*)items; a.n_items = n_items;
  a.flags = flags;
  a.spans = (const int2*)spans;
  a.spectra = (float4*)scratch; a.alm = (float2*)alm; a.stats = stats;
  // a chunk of lines of 32 KB, whole lines
  a.lines_per_chunk = max(1, min(min(nt / 2, 64), 4096 / nphi));
  size_t hw = (size_t)fr->h * fr->w;
  size_t lines_bytes = (size_t)a.lines_per_chunk * nphi * sizeof(float2);
  a.pat_in_smem = (!(flags & ZEB_FLAG_WINDOW) && hw * 4 + lines_bytes <= 200 * 1024) ? 1 : 0;
  size_t smem = lines_bytes + (a.pat_in_smem ? hw * 4 : 0);
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (nphi == 256) {
    // the warp-per-ring-pair kernel; a pattern above 48 KB is read from global memory (through
    // L1) rather than held in shared memory, which would leave one block an SM
    a.ring_major = 1;
    if (hw * 4 > 48 * 1024) a.pat_in_smem = 0;
    a.cache_cap = RW_CACHE;
    const size_t wsm = std::max((size_t)RW_WARPS * RW_PAD * sizeof(float2), a.pat_in_smem ? hw * 4 : (size_t)0) +
                       (size_t)RW_CACHE * sizeof(float);
    cudaFuncSetAttribute(k_sphere_rings_w, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
    k_sphere_rings_w<<<n_items, RW_WARPS * 32, wsm, st>>>(a);
    rc = zeb_launch_check("sphere_rings (warps)");
  } else {
    cudaFuncSetAttribute(k_sphere_rings, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_sphere_rings<<<n_items, 256, smem, st>>>(a);
    rc = zeb_launch_check("sphere_rings");
  }
  if (rc) return rc;
  const int nh = nt / 2;
  // items per block: 32, or fewer where the spectra and the table column would not fit
  int G = 32;
  auto lsm_of = [&](int g) { return (size_t)g * nh * sizeof(float4) + (size_t)nh * leg_nlp(L) * sizeof(float); };
  while (G > 4 && lsm_of(G) > 96 * 1024) G /= 2;
  const size_t lsm = lsm_of(G);
  ZEB_REQUIRE(lsm <= 220 * 1024, ZEB_ESIZE, "sphere_coefficients: L=%d needs %zu bytes of shared memory", L, lsm);
  a.leg_items = G;
  cudaFuncSetAttribute(k_legendre, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsm);
  dim3 g(L, (n_items + G - 1) / G);
  k_legendre<<<g, LEG_THREADS, lsm, st>>>(a);
  rc = zeb_launch_check("legendre");
  if (rc) return rc;
  k_sh_norm<<<n_items, 256, 0, st>>>(a);
  return zeb_launch_check("sh_norm");
}
