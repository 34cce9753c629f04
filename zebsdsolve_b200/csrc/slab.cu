// (b, second stage) The correlation volume's transform along a, and the peak.
//
// The slab U[b][j][m' < L][c < nc] arrives already transformed along b and c (both folded into
// the master's table); the real transform along a, C(a) = V[0] + 2 Re Σ_{m'>0} V[m'] e^{−i m' a}
// at the n grid values of a, comes out of one complex FFT of length h = n/2 per column c: its
// input is Z_q = (X_q + X_{q+h}) + i e^{−2πiq/n}(X_q − X_{q+h}) with X_{q+h} = conj X_{h−q}, and
// its output z_p = C(a_{2p}) + i C(a_{2p+1}) (so3.wgsl:279-315, 396-593).  Each column's values
// are scaled by the reciprocal denominator volume and the largest kept with its volume index
// (j·nc + c)·n + ia; each slab keeps its best (first index of equal values).
// k_peak_finish then takes each item's best slab, re-evaluates the six neighbours of the peak by
// direct sums over m' and fits the parabolic vertex along a, c and b (so3.wgsl:665-796).
#include <cuda.h>
#include <cuda_fp16.h>

#include <mutex>

#include "abi_util.cuh"
#include "twiddles.cuh"

namespace zeb {

struct SlabArgs {
  const float2* U;
  int n_items;
  zeb_so3_dims_t d;
  int lgc, lgh;
  const float2* tw;
  const float* rden;
  int rden_div;
  float2* cand;  // [item][nb]: (value, bits of index)
  float* vol;    // volume mode: [item][nb][nc][n]
};

template <bool VOLUME>
__global__ void __launch_bounds__(256) k_slab(SlabArgs a) {
  extern __shared__ float2 sm2[];
  __shared__ float redv[8];
  __shared__ uint32_t redi[8];
  const zeb_so3_dims_t& d = a.d;
  const int L = d.L, nc = d.nc, n = d.n, nb = d.nb;
  const int h = n >> 1;
  const int slab = blockIdx.x;  // b·nb + j
  const int b = slab / nb, j = slab - b * nb;
  const int lgc = a.lgc, lgh = a.lgh;
  float2* V = sm2;            // [L][nc]
  float2* Z = sm2 + L * nc;   // [h][nc]
  RowLines rows{lgc};
  ColLines cols{lgc};
  const float2* src = a.U + (size_t)slab * L * nc;
  for (int e = threadIdx.x; e < L * nc; e += blockDim.x) {
    int r = e >> lgc, c = e & (nc - 1);
    V[rows(r, c)] = src[e];
  }
  __syncthreads();
  // Z down each column, bit-reversed along a
  const int tws = ZEB_TW_LEN / (2 * h);
  for (int e = threadIdx.x; e < h * nc; e += blockDim.x) {
    int q = e >> lgc, c = e & (nc - 1);
    float2 x = make_float2(0.f, 0.f), y = make_float2(0.f, 0.f);
    if (q < L) x = V[rows(q, c)];
    if (q == 0) {
      x.y = 0.f;
    } else if (h - q < L) {
      float2 v = V[rows(h - q, c)];
      y = make_float2(v.x, -v.y);
    }
    float2 w = __ldg(a.tw + q * tws);
    float2 dd = make_float2(x.x - y.x, x.y - y.y);
    float2 z = make_float2(x.x + y.x - (w.x * dd.y + w.y * dd.x), x.y + y.y + (w.x * dd.x - w.y * dd.y));
    Z[cols(c, bitrev(q, lgh))] = z;
  }
  __syncthreads();
  fft_lines_smem_lf(Z, nc, lgh, a.tw, cols);

  if (VOLUME) {
    float* out = a.vol + (size_t)slab * nc * n;
    for (int e = threadIdx.x; e < nc * h; e += blockDim.x) {
      int c = e / h, p = e - c * h;
      float2 z = Z[cols(c, p)];
      out[c * n + 2 * p] = z.x;
      out[c * n + 2 * p + 1] = z.y;
    }
    return;
  }
  // the best of the slab: value × rden, first index of equal values
  const float* rd = a.rden + ((size_t)(b / a.rden_div) * nb + j) * nc * n;
  float bv = -3.4e38f;
  uint32_t bi = 0xffffffffu;
  for (int e = threadIdx.x; e < nc * h; e += blockDim.x) {
    int c = e / h, p = e - c * h;
    float2 z = Z[cols(c, p)];
    const float* r = rd + (size_t)c * n + 2 * p;
    float ev = z.x * __ldg(r), od = z.y * __ldg(r + 1);
    uint32_t ie = ((uint32_t)(j * nc + c)) * n + 2 * p;
    if (ev > bv || (ev == bv && ie < bi)) { bv = ev; bi = ie; }
    if (od > bv || (od == bv && ie + 1 < bi)) { bv = od; bi = ie + 1; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { redv[wid] = bv; redi[wid] = bi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      if (redv[w] > bv || (redv[w] == bv && redi[w] < bi)) { bv = redv[w]; bi = redi[w]; }
    }
    a.cand[slab] = make_float2(bv, __uint_as_float(bi));
  }
}

// ── the slab a warp at a time, its transform in registers ──
//
// A warp takes NC/32 columns per lane (or, for nc < 32, 32/nc slabs at once, one column per
// lane): the lane loads its column of the slab straight into registers (the lanes of a row read
// consecutive addresses; every load of the column is independent, so they are all in flight at
// once), forms the half-length real-transform input Z_q from V[q] and V[h−q] in place,
// transforms it along a in registers (radix-2, compile-time twiddles), scales by its rden row and
// keeps the largest value.  Within a lane the indices only grow, so the first of equal values is
// kept by a strict comparison; lanes then reduce by (value, lowest index).
template <int N>
__device__ __forceinline__ float2 tw_of(int t);
template <> __device__ __forceinline__ float2 tw_of<16>(int t) { return make_float2(kTwRe16[t], kTwIm16[t]); }
template <> __device__ __forceinline__ float2 tw_of<32>(int t) { return make_float2(kTwRe32[t], kTwIm32[t]); }
template <> __device__ __forceinline__ float2 tw_of<64>(int t) { return make_float2(kTwRe64[t], kTwIm64[t]); }
template <> __device__ __forceinline__ float2 tw_of<128>(int t) { return make_float2(kTwRe128[t], kTwIm128[t]); }

__host__ __device__ constexpr int brev_bits(int i, int bits) {
  int r = 0;
  for (int k = 0; k < bits; ++k) r |= ((i >> k) & 1) << (bits - 1 - k);
  return r;
}

__host__ __device__ constexpr int log2_const(int n) { return n <= 1 ? 0 : 1 + log2_const(n >> 1); }

// forward DFT of N points in registers (radix-2, decimation in time, natural order in and out)
template <int N>
__device__ __forceinline__ void fft_reg(float2 (&x)[N]) {
  constexpr int LG = log2_const(N);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = brev_bits(i, LG);
    if (j > i) {
      float2 t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
#pragma unroll
  for (int s = 1; s <= LG; ++s) {
    // every butterfly of the stage, by a flat index: constant trip counts unroll fully
#pragma unroll
    for (int e = 0; e < N / 2; ++e) {
      const int h = 1 << (s - 1);
      const int j = e & (h - 1);
      const int i0 = ((e >> (s - 1)) << s) + j;
      float2 b = x[i0 + h];
      float2 t;
      if (j == 0) {
        t = b;
      } else if (2 * j == h) {
        t = make_float2(b.y, -b.x);  // × e^{−iπ/2}
      } else {
        t = cmulf(b, tw_of<N>(j * (N >> s)));
      }
      float2 a = x[i0];
      x[i0] = make_float2(a.x + t.x, a.y + t.y);
      x[i0 + h] = make_float2(a.x - t.x, a.y - t.y);
    }
  }
}

// rden rows of one j staged per warp (rows padded by 4 floats: the lanes' 16-byte reads of
// their own rows fall in distinct banks)
template <int NC, int H>
struct ColsRden {
  static constexpr int RLD = 2 * H + 4;
  static constexpr int ROWS = NC < 32 ? 32 : NC;  // every slab of a warp: 32 rows, or NC
  static constexpr size_t BYTES = (size_t)ROWS * RLD * sizeof(float);
};

// SHARED: every item shares one rden volume; the warps then walk the slabs j-major in contiguous
// chunks, so a warp's j changes rarely, and keep the rows of their j in shared memory (the global
// rows of each lane otherwise come one dependent 16-byte load after another).
template <int NC, int H, int WARPS, int PER_SM, bool SHARED>
__global__ void __launch_bounds__(WARPS * 32, PER_SM) k_slab_cols(SlabArgs a) {
  constexpr int n = 2 * H;
  constexpr int SEG = NC < 32 ? NC : 32;  // lanes per slab
  constexpr int SPW = 32 / SEG;           // slabs per warp
  extern __shared__ __align__(16) float rtile_all[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / SEG, cl = lane - sub * SEG;
  const int L = a.d.L, nb = a.d.nb, ni = a.n_items;
  const long long total = (long long)ni * nb;
  const long long steps = (total + SPW - 1) / SPW;
  float* rtile = rtile_all + (size_t)warp * ColsRden<NC, H>::ROWS * ColsRden<NC, H>::RLD;
  int tile_j[SPW];
#pragma unroll
  for (int k = 0; k < SPW; ++k) tile_j[k] = -1;
  long long t0, t1, tstep;
  if (SHARED) {
    const long long wid = (long long)blockIdx.x * WARPS + warp, nw = (long long)gridDim.x * WARPS;
    const long long chunk = (steps + nw - 1) / nw;
    t0 = wid * chunk;
    t1 = t0 + chunk < steps ? t0 + chunk : steps;
    tstep = 1;
  } else {
    t0 = (long long)blockIdx.x * WARPS + warp;
    t1 = steps;
    tstep = (long long)gridDim.x * WARPS;
  }
  for (long long t = t0; t < t1; t += tstep) {
    const long long s0 = t * SPW;
    const long long slab = s0 + sub;
    const bool live = slab < total;
    const long long sl = live ? slab : s0;
    int b, j;
    if (SHARED) {  // work order j-major: (j, b) ↔ U slab b·nb + j
      j = (int)(sl / ni);
      b = (int)(sl - (long long)j * ni);
    } else {
      b = (int)(sl / nb);
      j = (int)(sl - (long long)b * nb);
    }
    const long long uslab = (long long)b * nb + j;
    const float2* src = a.U + uslab * L * NC;
    const float* rslab;
    int rstride;
    if (SHARED) {
      // (re)stage the rows of each sub-slab's j when it changed (warp-uniform: every lane sees all)
#pragma unroll
      for (int k = 0; k < SPW; ++k) {
        long long sk = s0 + k;
        if (sk >= total) sk = s0;
        const int jk = (int)(sk / ni);
        if (jk != tile_j[k]) {
          __syncwarp();
          const float4* g = (const float4*)(a.rden + (size_t)jk * NC * n);
          float* dst = rtile + (size_t)k * NC * ColsRden<NC, H>::RLD;
          for (int e = lane; e < NC * n / 4; e += 32) {
            const int c = e / (n / 4), p4 = e - c * (n / 4);
            *(float4*)(dst + c * ColsRden<NC, H>::RLD + 4 * p4) = __ldg(g + e);
          }
          tile_j[k] = jk;
          __syncwarp();
        }
      }
      rslab = rtile + (size_t)sub * NC * ColsRden<NC, H>::RLD;
      rstride = ColsRden<NC, H>::RLD;
    } else {
      rslab = a.rden + ((size_t)(b / a.rden_div) * nb + j) * NC * n;
      rstride = n;
    }
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
#pragma unroll 1
    for (int c = cl; c < NC; c += SEG) {
      float2 z[H];
#pragma unroll
      for (int q = 0; q < H; ++q) z[q] = q < L ? __ldcs(src + q * NC + c) : make_float2(0.f, 0.f);
      // Z_q = (X_q + X_{q+h}) + i w_q (X_q − X_{q+h}), X_{q+h} = conj X_{h−q}, w_q = e^{−2πi q/n},
      // computed for q and h − q together from the same two points (in place)
#pragma unroll
      for (int q = 0; q <= H / 2; ++q) {
        const int qm = (H - q) & (H - 1);
        float2 xq = z[q], xm = z[qm];
        float2 zq;
        {
          float2 x = xq, y = make_float2(0.f, 0.f);
          if (q == 0) x.y = 0.f;
          else y = make_float2(xm.x, -xm.y);
          const float2 w = tw_of<2 * H>(q);
          const float2 dd = make_float2(x.x - y.x, x.y - y.y);
          zq = make_float2(x.x + y.x - (w.x * dd.y + w.y * dd.x), x.y + y.y + (w.x * dd.x - w.y * dd.y));
        }
        if (q != 0 && qm != q) {
          float2 x = xm, y = make_float2(xq.x, -xq.y);
          const float2 w = tw_of<2 * H>(qm);
          const float2 dd = make_float2(x.x - y.x, x.y - y.y);
          z[qm] = make_float2(x.x + y.x - (w.x * dd.y + w.y * dd.x), x.y + y.y + (w.x * dd.x - w.y * dd.y));
        }
        z[q] = zq;
      }
      fft_reg<H>(z);
      const float4* rd = (const float4*)(rslab + (size_t)c * rstride);
      const uint32_t base = ((uint32_t)(j * NC + c)) * n;
#pragma unroll
      for (int p = 0; p < H; p += 2) {
        const float4 r = rd[p / 2];
        const float v0 = z[p].x * r.x, v1 = z[p].y * r.y, v2 = z[p + 1].x * r.z, v3 = z[p + 1].y * r.w;
        const uint32_t i0 = base + 2 * p;
        if (v0 > bv) { bv = v0; bi = i0; }
        if (v1 > bv) { bv = v1; bi = i0 + 1; }
        if (v2 > bv) { bv = v2; bi = i0 + 2; }
        if (v3 > bv) { bv = v3; bi = i0 + 3; }
      }
    }
    // the slab's best over its SEG lanes (xor offsets below SEG stay inside the segment)
#pragma unroll
    for (int o = SEG / 2; o > 0; o >>= 1) {
      float ov = __shfl_xor_sync(0xffffffffu, bv, o);
      uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (cl == 0 && live) a.cand[uslab] = make_float2(bv, __uint_as_float(bi));
  }
}

// V[j; m', c] of item b: U is already transformed along c (so3.wgsl:667-674)
struct UReader32 {  // FP32, [item][j][m'][c]
  const float2* U;
  __device__ __forceinline__ float2 operator()(int b, int j, int mp, int c, const zeb_so3_dims_t& d) const {
    return __ldg(U + (((size_t)b * d.nb + j) * d.L + mp) * d.nc + c);
  }
};
struct UReader16 {  // s·U in FP16, [item tile][(j, c)][m'][re|im][128 items]
  const __half* U;
  size_t ptiles;
  float inv;  // 1/s
  __device__ __forceinline__ float2 operator()(int b, int j, int mp, int c, const zeb_so3_dims_t& d) const {
    const size_t o = (((((size_t)(b >> 7) * d.nb + j) * d.nc + c) * d.L + mp) * 2) * 128 + (b & 127);
    return make_float2(__half2float(U[o]) * inv, __half2float(U[o + 128]) * inv);
  }
};

// Re(V e^{−i m a}) at grid point ia (so3.wgsl:766-769)
__device__ __forceinline__ float a_term(float2 v, int m, int ia, int n) {
  float ang = ZEB_TAU * (float)((m * ia) & (n - 1)) / (float)n;
  float sa, ca;
  sincosf(ang, &sa, &ca);
  return v.x * ca + v.y * sa;
}

__device__ __forceinline__ float vertex(float lo, float mid, float hi) {
  float den = lo - 2.f * mid + hi;
  if (den >= -1e-12f) return 0.f;
  return fminf(fmaxf(0.5f * (lo - hi) / den, -0.5f), 0.5f);
}

// CENTER: the peak's own value comes again from the direct sum (with exact twiddles) rather than
// from the candidate, so that the vertex fit sees seven values of the same arithmetic (the FP16
// spectrum's transform along a runs with FP16 twiddles)
template <class R, bool CENTER>
__global__ void __launch_bounds__(64) k_peak_finish(SlabArgs a, R v_at, float* __restrict__ peaks) {
  __shared__ float pf[7][64];
  __shared__ float2 best;
  const zeb_so3_dims_t& d = a.d;
  const int b = blockIdx.x;
  const int n = d.n, nc = d.nc, nb = d.nb, L = d.L;
  if (threadIdx.x < 32) {
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
    for (int j = threadIdx.x; j < nb; j += 32) {
      float2 c = a.cand[(size_t)b * nb + j];
      uint32_t ci = __float_as_uint(c.y);
      if (c.x > bv || (c.x == bv && ci < bi)) { bv = c.x; bi = ci; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float ov = __shfl_xor_sync(0xffffffffu, bv, o);
      uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (threadIdx.x == 0) best = make_float2(bv, __uint_as_float(bi));
  }
  __syncthreads();
  const float vbest = best.x;
  uint32_t idx = __float_as_uint(best.y);
  // no candidate, or one a transform that gave up on a wait never wrote (its status word reports
  // it): the volume's first cell, so that every read below stays inside U and rden
  if (idx >= (uint32_t)nb * (uint32_t)nc * (uint32_t)n) idx = 0;
  const int ia = idx & (n - 1);
  const int iq = (idx / n) & (nc - 1);
  const int j = idx / (n * nc);
  const bool inner = j > 0 && j < n / 2;
  const int iqm = (iq + nc - 1) & (nc - 1), iqp = (iq + 1) & (nc - 1);
  const int iam = (ia + n - 1) & (n - 1), iap = (ia + 1) & (n - 1);
  float s[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int m = threadIdx.x; m < L; m += 64) {
    float f = m == 0 ? 1.f : 2.f;
    float2 vc = v_at(b, j, m, iq, d);
    float2 vm = v_at(b, j, m, iqm, d);
    float2 vp = v_at(b, j, m, iqp, d);
    s[0] += f * a_term(vc, m, iam, n);
    s[1] += f * a_term(vc, m, iap, n);
    s[2] += f * a_term(vm, m, ia, n);
    s[3] += f * a_term(vp, m, ia, n);
    if (inner) {
      s[4] += f * a_term(v_at(b, j - 1, m, iq, d), m, ia, n);
      s[5] += f * a_term(v_at(b, j + 1, m, iq, d), m, ia, n);
    }
    if (CENTER) s[6] += f * a_term(vc, m, ia, n);
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) pf[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int off = 32; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off)
#pragma unroll
      for (int k = 0; k < 7; ++k) pf[k][threadIdx.x] += pf[k][threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const float* rd = a.rden + (size_t)(b / a.rden_div) * nb * nc * n;
  auto rat = [&](int jj, int qq, int aa) { return __ldg(rd + ((size_t)jj * nc + qq) * n + aa); };
  const float v0 = CENTER ? pf[6][0] * rat(j, iq, ia) : vbest;
  float da = vertex(pf[0][0] * rat(j, iq, iam), v0, pf[1][0] * rat(j, iq, iap));
  float dc = vertex(pf[2][0] * rat(j, iqm, ia), v0, pf[3][0] * rat(j, iqp, ia));
  float dj = 0.f;
  if (inner) dj = vertex(pf[4][0] * rat(j - 1, iq, ia), v0, pf[5][0] * rat(j + 1, iq, ia));
  // S = Rz(a) Ry(b) Rz(c); the orientation is its inverse, w ≥ 0 (so3.wgsl:776-796)
  const float step = ZEB_TAU / (float)n;
  float aa = ((float)ia + da) * step, bb = ((float)j + dj) * step, cc = ((float)iq + dc) * step;
  float4 qa = make_float4(cosf(0.5f * aa), 0.f, 0.f, sinf(0.5f * aa));
  float4 qb = make_float4(cosf(0.5f * bb), 0.f, sinf(0.5f * bb), 0.f);
  float4 qc = make_float4(cosf(0.5f * cc), 0.f, 0.f, sinf(0.5f * cc));
  float4 q = qmul(qa, qmul(qb, qc));
  q = make_float4(q.x, -q.y, -q.z, -q.w);
  if (q.x < 0.f) q = make_float4(-q.x, -q.y, -q.z, -q.w);
  float* o = peaks + (size_t)b * 8;
  o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
  o[4] = v0; o[5] = aa; o[6] = bb; o[7] = cc;
}

__global__ void k_rden_build(const float* __restrict__ vf, const float* __restrict__ vf2, const float* __restrict__ stats,
                             long long per_item, long long total, float* __restrict__ rden) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  float ar = fmaxf(stats[(t / per_item) * 4], 1e-12f);
  float m = vf[t];
  float v = vf2[t] - m * m / ar;
  rden[t] = v > 1e-6f * ar ? rsqrtf(v) : 0.f;
}

static int ilog2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

static bool dims_ok(const zeb_so3_dims_t* d) {
  return d && d->L >= 2 && d->L <= 256 && d->n >= 2 * d->L - 1 && (d->n & (d->n - 1)) == 0 && d->nb == d->n / 2 + 1 &&
         d->fold >= 1 && d->nc == d->n / d->fold && (d->nc & (d->nc - 1)) == 0 && d->L <= d->n / 2 &&
         d->n <= ZEB_TW_LEN;
}

static size_t slab_smem(const zeb_so3_dims_t* d) {
  return ((size_t)d->L * d->nc + (size_t)(d->n / 2) * d->nc) * sizeof(float2);
}

}  // namespace zeb

using namespace zeb;

extern "C" size_t zeb_peaks_scratch_bytes(const zeb_so3_dims_t* d, int n_items) {
  if (!dims_ok(d) || n_items <= 0) return 0;
  return (size_t)n_items * d->nb * sizeof(float2);
}

static int slab_launch(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw, SlabArgs& a, bool vol,
                       cudaStream_t st) {
  a.U = (const float2*)U;
  a.n_items = n_items;
  a.d = *d;
  a.lgc = ilog2i(d->nc);
  a.lgh = ilog2i(d->n / 2);
  a.tw = (const float2*)tw;
  size_t smem = slab_smem(d);
  ZEB_REQUIRE(smem <= 220 * 1024, ZEB_ESIZE, "correlate: slab of L=%d, nc=%d needs %zu bytes of shared memory", d->L,
              d->nc, smem);
  long long blocks = (long long)n_items * d->nb;
  ZEB_REQUIRE(blocks < (1LL << 31), ZEB_ESIZE, "correlate: too many slabs");
  if (!vol && d->L <= d->n / 2) {
    // the warp-per-slab kernels, where a lane's column fits in registers
    const int H = d->n / 2, NC = d->nc;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
#define ZEB_SLAB_COLS(nc_, h_, w_, per_sm_)                                                                    \
  if (NC == nc_ && H == h_) {                                                                                \
    constexpr int spw = (nc_) < 32 ? 32 / (nc_) : 1;                                                        \
    long long want = (blocks + (long long)(w_)*spw - 1) / ((long long)(w_)*spw);                             \
    if (a.rden_div >= n_items) {                                                                              \
      const size_t sm = (size_t)(w_) * ColsRden<nc_, h_>::BYTES;                                             \
      cudaFuncSetAttribute(k_slab_cols<nc_, h_, w_, per_sm_, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                           (int)sm);                                                                          \
      const long long fit = (long long)((220u * 1024u) / sm) < (per_sm_) ? (long long)((220u * 1024u) / sm)     \
                                                                           : (long long)(per_sm_);           \
      long long grid = want < (long long)sms * fit ? want : (long long)sms * fit;                              \
      k_slab_cols<nc_, h_, w_, per_sm_, true><<<(unsigned)grid, (w_)*32, sm, st>>>(a);                        \
    } else {                                                                                                  \
      long long grid = want < (long long)sms * (per_sm_)*8 ? want : (long long)sms * (per_sm_)*8;             \
      k_slab_cols<nc_, h_, w_, per_sm_, false><<<(unsigned)grid, (w_)*32, 0, st>>>(a);                        \
    }                                                                                                         \
    return zeb_launch_check("correlate slab (columns)");                                                    \
  }
    ZEB_SLAB_COLS(8, 16, 4, 6)
    ZEB_SLAB_COLS(16, 16, 4, 6)
    ZEB_SLAB_COLS(16, 32, 4, 4)
    ZEB_SLAB_COLS(32, 32, 4, 4)
    ZEB_SLAB_COLS(64, 32, 4, 4)
    ZEB_SLAB_COLS(32, 64, 4, 3)
    ZEB_SLAB_COLS(64, 64, 4, 3)
#undef ZEB_SLAB_COLS
  }
  if (vol) {
    cudaFuncSetAttribute(k_slab<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_slab<true><<<(unsigned)blocks, 256, smem, st>>>(a);
  } else {
    cudaFuncSetAttribute(k_slab<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_slab<false><<<(unsigned)blocks, 256, smem, st>>>(a);
  }
  return zeb_launch_check("correlate slab");
}

extern "C" int zeb_correlate_peaks(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw,
                                   const float* rden, int rden_div, float* peaks, void* scratch, void* stream) {
  ZEB_REQUIRE(U && tw && rden && peaks && scratch, ZEB_EARG, "correlate_peaks: null argument");
  ZEB_REQUIRE(dims_ok(d), ZEB_EARG, "correlate_peaks: inconsistent dims");
  ZEB_REQUIRE(rden_div >= 1, ZEB_EARG, "correlate_peaks: rden_div=%d", rden_div);
  if (n_items <= 0) return ZEB_OK;
  SlabArgs a{};
  a.rden = rden;
  a.rden_div = rden_div;
  a.cand = (float2*)scratch;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = slab_launch(U, n_items, d, tw, a, false, st);
  if (rc) return rc;
  k_peak_finish<UReader32, false><<<n_items, 64, 0, st>>>(a, UReader32{(const float2*)U}, peaks);
  return zeb_launch_check("peak_finish");
}

// the candidates of the tensor-core transform (slab_tc.cu) reduced, and the vertex fitted from
// the FP16 spectrum: zeb_correlate_peaks_h's last step
extern "C" int zeb_peak_finish_h(const void* U16, int n_items, const zeb_so3_dims_t* d, float scale, const float* rden,
                                 const float2* cand, float* peaks, void* stream) {
  SlabArgs a{};
  a.n_items = n_items;
  a.d = *d;
  a.rden = rden;
  a.rden_div = 1 << 30;
  a.cand = const_cast<float2*>(cand);
  UReader16 r{(const __half*)U16, (size_t)((n_items + 127) / 128), 1.f / scale};
  k_peak_finish<UReader16, true><<<n_items, 64, 0, (cudaStream_t)stream>>>(a, r, peaks);
  return zeb_launch_check("peak_finish (FP16 spectrum)");
}

extern "C" int zeb_correlate_volume(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw, float* vol,
                                    void* stream) {
  ZEB_REQUIRE(U && tw && vol, ZEB_EARG, "correlate_volume: null argument");
  ZEB_REQUIRE(dims_ok(d), ZEB_EARG, "correlate_volume: inconsistent dims");
  if (n_items <= 0) return ZEB_OK;
  SlabArgs a{};
  a.vol = vol;
  return slab_launch(U, n_items, d, tw, a, true, (cudaStream_t)stream);
}

extern "C" int zeb_rden_build(const float* vol_f, const float* vol_f2, const float* stats, int n, long long cells,
                              float* rden, void* stream) {
  ZEB_REQUIRE(vol_f && vol_f2 && stats && rden && n >= 0 && cells > 0, ZEB_EARG, "rden_build: bad arguments");
  long long total = (long long)n * cells;
  if (total == 0) return ZEB_OK;
  k_rden_build<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(vol_f, vol_f2, stats, cells, total,
                                                                                  rden);
  return zeb_launch_check("rden_build");
}

// ── the same peaks with their scratch in a static device array (no allocation anywhere) ──
//
// The candidates of zeb_correlate_peaks (one (value, index) per (item, j) slab) live here instead
// of in caller memory: ZEB_PEAKS_STATIC_SLABS of them, 4 MiB, held by every device that loads the
// library until the process exits. Host code may not hand g_peaks_scratch to a kernel (in host
// code the name stands for a host-side shadow, not a device address): the address is looked up
// with cudaGetSymbolAddress, with the device current, and passed to the kernels.
//
// Each CUDA context has its own copy of the array (a context loads the module for itself), so the
// address is cached per context, keyed by the context's unique ID (cuCtxGetId: an ID is never
// reused, unlike a context handle or a device ordinal). After a cudaDeviceReset, or under another
// context made current on the same device, the next call meets a new ID and looks the address up
// again with that context current.
static __device__ __align__(256) float2 g_peaks_scratch[ZEB_PEAKS_STATIC_SLABS];

namespace {
std::mutex g_static_mu;
struct StaticAddr {
  unsigned long long ctx_id;
  float2* addr;
};
StaticAddr g_static_addr[64];  // the most recent contexts, oldest replaced first
int g_static_next = 0;

typedef CUresult (*ctx_current_fn)(CUcontext*);
typedef CUresult (*ctx_id_fn)(CUcontext, unsigned long long*);

// the current context's unique ID through the runtime's driver entry points (no link against libcuda)
bool current_ctx_id(unsigned long long* id) {
  static ctx_current_fn get_current = nullptr;
  static ctx_id_fn get_id = nullptr;
  if (!get_current || !get_id) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return false;
    get_current = (ctx_current_fn)p;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return false;
    get_id = (ctx_id_fn)p;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return get_id(ctx, id) == CUDA_SUCCESS;
}
}  // namespace

extern "C" int zeb_correlate_peaks_static(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw,
                                          const float* rden, int rden_div, float* peaks, void* stream) {
  ZEB_REQUIRE(U && tw && rden && peaks, ZEB_EARG, "correlate_peaks_static: null argument");
  ZEB_REQUIRE(dims_ok(d), ZEB_EARG, "correlate_peaks_static: inconsistent dims");
  ZEB_REQUIRE(rden_div >= 1, ZEB_EARG, "correlate_peaks_static: rden_div=%d", rden_div);
  if (n_items <= 0) return ZEB_OK;
  ZEB_REQUIRE((long long)n_items * d->nb <= (long long)ZEB_PEAKS_STATIC_SLABS, ZEB_ESIZE,
              "correlate_peaks_static: %d items need %lld slabs of scratch; the static scratch holds %d "
              "(at most %d items at this bandwidth)",
              n_items, (long long)n_items * d->nb, ZEB_PEAKS_STATIC_SLABS, ZEB_PEAKS_STATIC_SLABS / d->nb);
  unsigned long long id = 0;
  cudaError_t e = cudaSuccess;
  if (!current_ctx_id(&id)) {
    // no context is current on this thread yet: cudaSetDevice makes the device's primary one so
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaSetDevice(dev);
    ZEB_REQUIRE(e == cudaSuccess && current_ctx_id(&id), ZEB_ECUDA, "correlate_peaks_static: no CUDA context: %s",
                cudaGetErrorString(e));
  }
  float2* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_static_mu);
    for (const StaticAddr& a : g_static_addr)
      if (a.addr && a.ctx_id == id) scratch = a.addr;
    if (!scratch) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_peaks_scratch);
      ZEB_REQUIRE(e == cudaSuccess && p, ZEB_ECUDA, "correlate_peaks_static: cudaGetSymbolAddress: %s",
                  cudaGetErrorString(e));
      scratch = (float2*)p;
      g_static_addr[g_static_next] = StaticAddr{id, scratch};
      g_static_next = (g_static_next + 1) % 64;
    }
  }
  // every slab writes its candidate before k_peak_finish reads it: nothing needs clearing
  SlabArgs a{};
  a.rden = rden;
  a.rden_div = rden_div;
  a.cand = scratch;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = slab_launch(U, n_items, d, tw, a, false, st);
  if (rc) return rc;
  k_peak_finish<UReader32, false><<<n_items, 64, 0, st>>>(a, UReader32{(const float2*)U}, peaks);
  return zeb_launch_check("peak_finish");
}
