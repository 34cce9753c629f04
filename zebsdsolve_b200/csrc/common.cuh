// Shared device helpers for the sm_100a kernels of the spherical indexing path.
//
// Conventions (the reference's, zebsdsolve 0.2.8 shaders/common.wgsl:1-62): a quaternion is
// (w, x, y, z) held in a float4 as (.x, .y, .z, .w) and rotates v as q v q*; an orientation maps
// sample directions to crystal directions.  A master pattern is two side × side equal-area
// Lambert sheets [north | south].
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define ZEB_PI 3.14159265358979f
#define ZEB_TAU 6.28318530717959f
// length of the twiddle table: tw[t] = e^{−2πi t / ZEB_TW_LEN}
#define ZEB_TW_LEN 1024

namespace zeb {

__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
  return make_float4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
                     a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
                     a.x * b.z - a.y * b.w + a.z * b.x + a.w * b.y,
                     a.x * b.w + a.y * b.z - a.z * b.y + a.w * b.x);
}

__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// The circular mask's test dr² + dc² ≤ r² (r² ≤ 0: no mask) with every product and the sum rounded
// on its own (no fused multiply-add), on the device as on the host, so that both count the same
// pixels (a boundary pixel must not be in one list and not the other).
__host__ __device__ __forceinline__ bool zeb_in_circle(float dr, float dc, float r2) {
#ifdef __CUDA_ARCH__
  return r2 <= 0.f || __fadd_rn(__fmul_rn(dr, dr), __fmul_rn(dc, dc)) <= r2;
#else
  const volatile float a = dr * dr, b = dc * dc;
  return r2 <= 0.f || (float)(a + b) <= r2;
#endif
}

// q v q*
__device__ __forceinline__ float3 qrot(float4 q, float3 v) {
  float3 u = make_float3(q.y, q.z, q.w);
  float3 t = cross3(u, v);
  t.x *= 2.f; t.y *= 2.f; t.z *= 2.f;
  float3 ut = cross3(u, t);
  return make_float3(v.x + q.x * t.x + ut.x, v.y + q.x * t.y + ut.y, v.z + q.x * t.z + ut.z);
}

__device__ __forceinline__ float3 normalize3(float3 v) {
  float inv = rsqrtf(dot3(v, v));
  return make_float3(v.x * inv, v.y * inv, v.z * inv);
}

// exp of a rotation vector
__device__ __forceinline__ float4 qexp(float3 phi) {
  float th2 = dot3(phi, phi);
  float th = sqrtf(th2);
  float k = 0.5f - th2 / 48.f;
  if (th > 1e-3f) k = sinf(0.5f * th) / th;
  return make_float4(cosf(0.5f * th), k * phi.x, k * phi.y, k * phi.z);
}

// Unit vector → equal-area square coordinates in [−1, 1]² of its own hemisphere; 1 − |z| taken
// as (x² + y²)/(1 + |z|) (common.wgsl:44-57).
__device__ __forceinline__ float2 sphere_to_square(float3 v) {
  float ax = fabsf(v.x), ay = fabsf(v.y);
  float xn = sqrtf(fmaxf(ZEB_PI * 0.5f * (ax * ax + ay * ay) / (1.f + fabsf(v.z)), 0.f));
  float u = xn, w = xn;
  if (ax >= ay) {
    w = (4.f * xn / ZEB_PI) * atan2f(ay, fmaxf(ax, 1e-30f));
  } else {
    u = (4.f * xn / ZEB_PI) * atan2f(ax, fmaxf(ay, 1e-30f));
  }
  const float sc = 0.79788456080286536f;  // 1 / sqrt(π / 2)
  return make_float2(u * sc * (v.x < 0.f ? -1.f : 1.f), w * sc * (v.y < 0.f ? -1.f : 1.f));
}

// atan(t) for t in [0, 1]: t·P(t²), P an 8-term polynomial fitted here (least squares over 4000
// Chebyshev nodes of [0, 1], reweighted toward the largest errors until equi-ripple); evaluated
// by Horner in FP32 its error is below 1.5e-7 absolute (2.5 ulp of π/4) over the interval.
__device__ __forceinline__ float atan01(float t) {
  const float t2 = t * t;
  float p = -4.054563120e-03f;
  p = fmaf(p, t2, 2.186294459e-02f);
  p = fmaf(p, t2, -5.591231585e-02f);
  p = fmaf(p, t2, 9.642197192e-02f);
  p = fmaf(p, t2, -1.390862912e-01f);
  p = fmaf(p, t2, 1.994656622e-01f);
  p = fmaf(p, t2, -3.332985938e-01f);
  p = fmaf(p, t2, 9.999993443e-01f);
  return t * p;
}

// sphere_to_square with approximate arithmetic (the fast square root, atan01): within a few ulp
// of the exact map, for the per-pixel loops of the detector kernels. square_map keeps the
// intermediates the derivative of the lookup reuses (sheet_jacobian_of): ρ² = x² + y²,
// 1/(1 + |z|), q = (π/2) ρ²/(1 + |z|), 1/√q, xn = √q and the fitted arctangent.
struct SquareMap {
  float2 uv;
  float rho2, rden, rq, xn, at;
};

__device__ __forceinline__ SquareMap square_map(float3 v) {
  SquareMap m;
  const float ax = fabsf(v.x), ay = fabsf(v.y);
  m.rho2 = ax * ax + ay * ay;
  m.rden = __frcp_rn(1.f + fabsf(v.z));
  const float q = ZEB_PI * 0.5f * m.rho2 * m.rden;
  m.rq = rsqrtf(q);
  m.xn = q > 0.f ? q * m.rq : 0.f;
  const float lo = fminf(ax, ay), hi = fmaxf(fmaxf(ax, ay), 1e-30f);
  m.at = atan01(__fdividef(lo, hi));
  const float ang = (4.f / ZEB_PI) * m.xn * m.at;
  const float u = ax >= ay ? m.xn : ang, w = ax >= ay ? ang : m.xn;
  const float sc = 0.79788456080286536f;  // 1 / sqrt(π / 2)
  m.uv = make_float2(copysignf(u * sc, v.x < 0.f ? -1.f : 1.f), copysignf(w * sc, v.y < 0.f ? -1.f : 1.f));
  return m;
}

__device__ __forceinline__ float2 sphere_to_square_fast(float3 v) { return square_map(v).uv; }

// Square coordinates → unit vector on the northern or southern hemisphere (mastersph.wgsl:40-62).
__device__ __forceinline__ float3 square_to_sphere(float px, float py, bool south) {
  const float sc = 1.2533141373155003f;  // sqrt(π / 2)
  float xa = fabsf(px) * sc, ya = fabsf(py) * sc;
  bool swap = xa >= ya;
  float xn = fmaxf(xa, ya), yn = fminf(xa, ya);
  float3 v = make_float3(0.f, 0.f, 1.f);
  if (xn > 0.f) {
    float r = (2.f * xn / ZEB_PI) * sqrtf(fmaxf(ZEB_PI - xn * xn, 0.f));
    float ang = ZEB_PI * yn / (4.f * xn);
    float hx = r * cosf(ang), hy = r * sinf(ang);
    if (!swap) { float t = hx; hx = hy; hy = t; }
    v = normalize3(make_float3(hx * (px < 0.f ? -1.f : 1.f), hy * (py < 0.f ? -1.f : 1.f), 1.f - 2.f * xn * xn / ZEB_PI));
  }
  if (south) v.z = -v.z;
  return v;
}

// Bilinear placement of direction v on its hemisphere's sheet: the base texel offset and the two
// fractions (detector.wgsl:102-115).
struct SheetPos {
  uint32_t o;
  float tj, ti;
};

// FAST: sphere_to_square_fast (the detector kernels' per-pixel loops); else the exact map
template <bool FAST = true>
__device__ __forceinline__ SheetPos sheet_pos(float3 v, int side) {
  float2 uv = FAST ? sphere_to_square_fast(v) : sphere_to_square(v);
  float last = (float)(side - 1);
  float fj = fminf(fmaxf((uv.x + 1.f) * 0.5f * last, 0.f), last);
  float fi = fminf(fmaxf((uv.y + 1.f) * 0.5f * last, 0.f), last);
  uint32_t c0 = min((uint32_t)fj, (uint32_t)(side - 2));
  uint32_t r0 = min((uint32_t)fi, (uint32_t)(side - 2));
  SheetPos p;
  p.o = r0 * side + c0;
  if (v.z < 0.f) p.o += side * side;
  p.tj = fj - (float)c0;
  p.ti = fi - (float)r0;
  return p;
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + (b - a) * t; }

template <bool FAST = true>
__device__ __forceinline__ float master_at(const float* __restrict__ m, float3 v, int side) {
  SheetPos p = sheet_pos<FAST>(v, side);
  float top = lerpf(__ldg(m + p.o), __ldg(m + p.o + 1), p.tj);
  float bot = lerpf(__ldg(m + p.o + side), __ldg(m + p.o + side + 1), p.tj);
  return lerpf(top, bot, p.ti);
}

__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
  return make_float4(lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t), lerpf(a.w, b.w, t));
}

// The master's tangent gradient (.xyz) and value (.w) at v, bilinear in the float4 table.
__device__ __forceinline__ float4 grad_at(const float4* __restrict__ g, float3 v, int side) {
  SheetPos p = sheet_pos(v, side);
  float4 a = __ldg(g + p.o), b = __ldg(g + p.o + 1), c = __ldg(g + p.o + side), d = __ldg(g + p.o + side + 1);
  return lerp4(lerp4(a, b, p.tj), lerp4(c, d, p.tj), p.ti);
}

// The same lookups from the pair tables (zeb_master_pairs): one 32-byte (gradient) or 8-byte
// (value) record per row of the 2 × 2 neighbourhood, the same arithmetic.
__device__ __forceinline__ void ldg_v8(const float* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

__device__ __forceinline__ float4 grad_at_pair(const float* __restrict__ gp, float3 v, int side) {
  SheetPos p = sheet_pos(v, side);
  float4 a, b, c, d;
  ldg_v8(gp + 8 * (size_t)p.o, a, b);
  ldg_v8(gp + 8 * ((size_t)p.o + side), c, d);
  return lerp4(lerp4(a, b, p.tj), lerp4(c, d, p.tj), p.ti);
}

// two floats rounded to FP16 in one word (the first in the low half), and back
__device__ __forceinline__ uint32_t zeb_half2(float lo, float hi) {
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float2 zeb_unhalf2(uint32_t w) {
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}

// The same lookup from the FP16 neighbourhood records (zeb_master_quads): one 32-byte record a
// pixel, each texel's (gx, gy) and (gz, value) as two half2; the bilinear interpolation in packed
// FP16 arithmetic (two channels an instruction, the weights rounded to FP16), its result widened
// to FP32 for the sums.
__device__ __forceinline__ float4 grad_at_quad(const float* __restrict__ gq, float3 v, int side) {
  SheetPos p = sheet_pos(v, side);
  uint32_t h[8];
  asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(h[0]), "=r"(h[1]), "=r"(h[2]), "=r"(h[3]), "=r"(h[4]), "=r"(h[5]), "=r"(h[6]), "=r"(h[7])
      : "l"(gq + 8 * (size_t)p.o));
  const __half2 tj = __float2half2_rn(p.tj), ti = __float2half2_rn(p.ti);
  const __half2* t = reinterpret_cast<const __half2*>(h);
  // texels 0 (right 1) above, 2 (right 3) below: top = t0 + (t1 − t0)·tj, bot likewise, then ti
  const __half2 top_xy = __hfma2(__hsub2(t[2], t[0]), tj, t[0]);
  const __half2 top_zm = __hfma2(__hsub2(t[3], t[1]), tj, t[1]);
  const __half2 bot_xy = __hfma2(__hsub2(t[6], t[4]), tj, t[4]);
  const __half2 bot_zm = __hfma2(__hsub2(t[7], t[5]), tj, t[5]);
  const float2 xy = __half22float2(__hfma2(__hsub2(bot_xy, top_xy), ti, top_xy));
  const float2 zm = __half22float2(__hfma2(__hsub2(bot_zm, top_zm), ti, top_zm));
  return make_float4(xy.x, xy.y, zm.x, zm.y);
}

__device__ __forceinline__ float master_at_pair(const float2* __restrict__ vp, float3 v, int side) {
  SheetPos p = sheet_pos(v, side);
  const float2 t = __ldg(vp + p.o), u = __ldg(vp + p.o + side);
  return lerpf(lerpf(t.x, t.y, p.tj), lerpf(u.x, u.y, p.tj), p.ti);
}

// ── block reductions ──

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of `count` per-thread values across the block; every thread gets the totals. `red` holds
// count × (blockDim/32) floats.
template <int COUNT>
__device__ __forceinline__ void block_sums(float (&v)[COUNT], float* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < COUNT; ++k) {
    float s = warp_sum(v[k]);
    if (lane == 0) red[k * nw + wid] = s;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < COUNT; ++k) {
    float s = 0.f;
    for (int w = 0; w < nw; ++w) s += red[k * nw + w];
    v[k] = s;
  }
  __syncthreads();
}

// ── in-shared-memory radix-2 FFT over several lines ──
//
// `count` lines of length 2^lg, point p of line i at data[idx(i, p)] (idx: a layout functor),
// loaded in bit-reversed order. Forward transform (e^{−i…}) with twiddles
// tw[t] = e^{−2πi t/ZEB_TW_LEN}. Every thread of the block takes part; the caller synchronizes
// before, and the function synchronizes after each stage.
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <typename Index>
__device__ void fft_lines_smem(float2* data, int count, int lg, const float2* __restrict__ tw, Index idx) {
  const int len = 1 << lg;
  const int half_total = count * (len >> 1);
  for (int st = 0; st < lg; ++st) {
    const int half = 1 << st;
    const int tstep = ZEB_TW_LEN >> (st + 1);
    for (int e = threadIdx.x; e < half_total; e += blockDim.x) {
      const int line = e >> (lg - 1);
      const int r = e & ((len >> 1) - 1);
      const int j = r & (half - 1);
      const int p0 = ((r >> st) << (st + 1)) + j;
      const int i0 = idx(line, p0), i1 = idx(line, p0 + half);
      float2 w = __ldg(tw + j * tstep);
      float2 b = cmulf(data[i1], w);
      float2 a = data[i0];
      data[i0] = make_float2(a.x + b.x, a.y + b.y);
      data[i1] = make_float2(a.x - b.x, a.y - b.y);
    }
    __syncthreads();
  }
}

// The same stages with the line index varying fastest across threads (for lines that are the
// columns of a row-major slab: neighbouring threads then touch neighbouring words).
template <typename Index>
__device__ void fft_lines_smem_lf(float2* data, int count, int lg, const float2* __restrict__ tw, Index idx) {
  const int len = 1 << lg;
  const int half_total = count * (len >> 1);
  for (int st = 0; st < lg; ++st) {
    const int half = 1 << st;
    const int tstep = ZEB_TW_LEN >> (st + 1);
    for (int e = threadIdx.x; e < half_total; e += blockDim.x) {
      const int line = e % count;
      const int r = e / count;
      const int j = r & (half - 1);
      const int p0 = ((r >> st) << (st + 1)) + j;
      const int i0 = idx(line, p0), i1 = idx(line, p0 + half);
      float2 w = __ldg(tw + j * tstep);
      float2 b = cmulf(data[i1], w);
      float2 a = data[i0];
      data[i0] = make_float2(a.x + b.x, a.y + b.y);
      data[i1] = make_float2(a.x - b.x, a.y - b.y);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int bitrev(int x, int lg) { return (int)(__brev((unsigned)x) >> (32 - lg)); }

// Shared-memory index of point i of a set of lines lying back to back: the low four bits crossed
// with the four above them, so that bit-reversed loads and the first butterfly stages spread
// over the banks (a bijection on every aligned block of 256).
__device__ __forceinline__ int fsw(int i) { return i ^ ((i >> 4) & 15); }

// Line-major layout: point p of line `line` (lines of 2^lg points).
struct RowLines {
  int lg;
  __device__ __forceinline__ int operator()(int line, int p) const { return fsw((line << lg) + p); }
};

// Column layout of a row-major 2-D slab of 2^lgc columns: line = column, point = row.
struct ColLines {
  int lgc;
  __device__ __forceinline__ int operator()(int line, int p) const { return fsw((p << lgc) + line); }
};

}  // namespace zeb
