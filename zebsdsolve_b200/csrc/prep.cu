// Pattern preprocessing: one thread block per pattern does the whole chain (unpack, static
// background, dynamic background, mask and normalization) with the image held in shared memory
// when it fits, so a pattern is read from HBM once and written once.
//
// The arithmetic follows shaders/prep.wgsl: the direct Gaussian (taps to ceil(3σ), renormalized
// over the taps inside the image) below σ = 12 pixels, the box-sum construction above it
// (box sums of s = ⌊σ/6⌋ pixels, a coarse Gaussian over them with a margin of cpad = 3 cells,
// and a spread of deviation s back over the pixels).
#include "abi_util.cuh"

namespace zeb {

struct PrepArgs {
  const void* raw;
  int pixel, n, h, w;
  int sh, sw;      // the stored pattern's size (h, w when nothing is reduced)
  double factor;   // reduction factor (1: none)
  int kwhole;      // the factor as a whole number, 0 when it is not one
  const float* static_bg;
  int dynamic;  // 0 none, 1 subtract, 2 divide, 3 the blur itself
  float sigma;
  float mask[3];
  int normalize;
  float* out;
  float* scratch;  // per pattern: scratch_per floats
  long long scratch_per;
  int use_smem;
  // direct blur
  int radius;
  float k0;
  // wide blur
  int bin, cpad, wradius;
  float kx, kz;
};

// the image against its blurred self: 1 subtract, 2 divide (the dynamic background), 3 the
// blurred image itself (a band pass's Gaussians)
__device__ __forceinline__ float with_background(int dynamic, float v, float bg) {
  return dynamic == 1 ? v - bg : (dynamic == 2 ? v / fmaxf(bg, 1e-6f) : bg);
}

__device__ __forceinline__ float2 wide_cell(int jr, int n, int s) {
  int lo = jr * s;
  int hi = lo + s;
  if (jr >= 0 && lo < n) hi = min(hi, n);
  return make_float2(0.5f * (float)(lo + hi - 1), (float)(hi - lo));
}

// zero mean and unit norm under the mask (prep.wgsl:405-443), or the plain copy out
__device__ void prep_finish(const PrepArgs& a, float* img, float* out, float* red) {
  const int h = a.h, w = a.w, hw = h * w;
  if (!a.normalize) {
    if (a.use_smem)
      for (int i = threadIdx.x; i < hw; i += blockDim.x) out[i] = img[i];
    return;
  }
  float v2[2] = {0.f, 0.f};
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    int r = i / w, c = i - r * w;
    float dr = (float)r - a.mask[0], dc = (float)c - a.mask[1];
    if (zeb_in_circle(dr, dc, a.mask[2])) {
      v2[0] += img[i];
      v2[1] += 1.f;
    }
  }
  block_sums<2>(v2, red);
  const float mean = v2[0] / fmaxf(v2[1], 1.f);
  float ss[1] = {0.f};
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    int r = i / w, c = i - r * w;
    float dr = (float)r - a.mask[0], dc = (float)c - a.mask[1];
    float v = 0.f;
    if (zeb_in_circle(dr, dc, a.mask[2])) v = img[i] - mean;
    img[i] = v;
    ss[0] += v * v;
  }
  block_sums<1>(ss, red);
  const float inv = rsqrtf(fmaxf(ss[0], 1e-30f));
  for (int i = threadIdx.x; i < hw; i += blockDim.x) out[i] = img[i] * inv;
}

__device__ __forceinline__ float stored_px(const PrepArgs& a, size_t i) {
  if (a.pixel == 0) return (float)((const uint8_t*)a.raw)[i];
  if (a.pixel == 1) return (float)((const uint16_t*)a.raw)[i];
  return ((const float*)a.raw)[i];
}

// Output pixel (r, c) of stored pattern b reduced by a.factor (reduce.zig:44-131): for a whole
// factor k the k × k block's mean (integer pixels summed exactly, f32 ones row by row); otherwise
// the source area the output pixel covers, each source row's part summed in FP64 then shared
// between the one or two output rows it lies in, in the order of the source rows (products and
// sums rounded one at a time, as the host reduction does).
__device__ float reduced_px(const PrepArgs& a, int b, int r, int c) {
  const size_t base = (size_t)b * a.sh * a.sw;
  if (a.kwhole > 0) {
    const int k = a.kwhole;
    const float inv = 1.f / (float)(k * k);
    if (a.pixel != 2) {
      uint32_t acc = 0;
      for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) acc += (uint32_t)stored_px(a, base + (size_t)(r * k + i) * a.sw + c * k + j);
      return __fmul_rn((float)acc, inv);
    }
    float out = 0.f;
    for (int i = 0; i < k; ++i) {
      float acc = 0.f;
      for (int j = 0; j < k; ++j) acc = __fadd_rn(acc, stored_px(a, base + (size_t)(r * k + i) * a.sw + c * k + j));
      out = __fadd_rn(out, acc);
    }
    return __fmul_rn(out, inv);
  }
  const double f = a.factor;
  const int rows = (int)ceil((double)a.h * f - 1e-9);
  const double x0 = (double)c * f, x1 = x0 + f;
  const int j0 = (int)floor(x0);
  float out = 0.f;
  const int lo = max(0, (int)floor(((double)r - 1.0) * f) - 1), hi = min(rows - 1, (int)ceil(((double)r + 1.0) * f) + 1);
  for (int rs = lo; rs <= hi; ++rs) {
    const double y0 = (double)rs;
    const int top = (int)floor(y0 / f + 1e-12);
    const double edge = (double)(top + 1) * f;
    const float w0 = (float)(fmin(y0 + 1.0, edge) - y0);
    float wt;
    if (top == r) wt = w0;
    else if (top + 1 == r && w0 < 1.f) wt = __fsub_rn(1.f, w0);
    else continue;
    double acc = 0.0;
    for (int j = j0; (double)j < x1 - 1e-12; ++j) {
      const double aa = fmax(x0, (double)j), bb = fmin(x1, (double)(j + 1));
      acc = __dadd_rn(acc, __dmul_rn(bb - aa, (double)stored_px(a, base + (size_t)rs * a.sw + j)));
    }
    out = __fadd_rn(out, __fmul_rn(wt, (float)acc));
  }
  return __fmul_rn(out, (float)(1.0 / (f * f)));
}

// one pixel of pattern b as the chain starts from it: stored (or reduced), static background off
__device__ __forceinline__ float prep_pixel(const PrepArgs& a, int b, int i) {
  float v;
  if (a.factor == 1.0) {
    v = stored_px(a, (size_t)b * a.h * a.w + i);
  } else {
    const int r = i / a.w;
    v = reduced_px(a, b, r, i - r * a.w);
  }
  if (a.static_bg) v -= __ldg(a.static_bg + i);
  return v;
}

__global__ void __launch_bounds__(256) k_prep(PrepArgs a) {
  extern __shared__ float sm[];
  __shared__ float taps[64];
  __shared__ float red[2 * 8];
  const int b = blockIdx.x;
  const int h = a.h, w = a.w, hw = h * w;
  float* img = a.use_smem ? sm : a.out + (size_t)b * hw;
  float* tmp = a.use_smem ? sm + hw : a.scratch + (size_t)b * a.scratch_per;

  // unpack
  const size_t base = (size_t)b * hw;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) img[i] = prep_pixel(a, b, i);
  __syncthreads();

  if (a.dynamic != 0 && a.sigma > 0.f) {
    float* bg;  // the blurred image, one value per pixel
    if (a.bin < 2) {
      for (int d = threadIdx.x; d <= min(a.radius, 63); d += blockDim.x) taps[d] = expf(-(float)(d * d) * a.k0);
      __syncthreads();
      const int R = a.radius;
      // along the rows into tmp
      for (int i = threadIdx.x; i < hw; i += blockDim.x) {
        int r = i / w, c = i - r * w;
        float s = 0.f, g = 0.f;
        for (int x = max(c - R, 0); x <= min(c + R, w - 1); ++x) {
          int dd = abs(x - c);
          float t = dd <= R ? taps[min(dd, 63)] : 0.f;
          s += t * img[r * w + x];
          g += t;
        }
        tmp[i] = s / g;
      }
      __syncthreads();
      // along the columns: the background, combined with the image in place
      for (int i = threadIdx.x; i < hw; i += blockDim.x) {
        int r = i / w, c = i - r * w;
        float s = 0.f, g = 0.f;
        for (int y = max(r - R, 0); y <= min(r + R, h - 1); ++y) {
          int dd = abs(y - r);
          float t = dd <= R ? taps[min(dd, 63)] : 0.f;
          s += t * tmp[y * w + c];
          g += t;
        }
        float bgv = s / g;
        img[i] = with_background(a.dynamic, img[i], bgv);
      }
      __syncthreads();
      bg = nullptr;
    } else {
      const int s = a.bin, cp = a.cpad;
      const int hs = (h + s - 1) / s, ws = (w + s - 1) / s, wp = ws + 2 * cp, hp = hs + 2 * cp;
      float2* box = (float2*)(a.scratch + (size_t)b * a.scratch_per + (a.use_smem ? 0 : hw));
      float2* rows = box + hs * ws;
      float2* cols = rows + hs * wp;
      float2* spread = cols + hp * wp;
      for (int t = threadIdx.x; t < hs * ws; t += blockDim.x) {
        int i = t / ws, j = t - i * ws;
        int r1 = min((i + 1) * s, h), c1 = min((j + 1) * s, w);
        float acc = 0.f;
        for (int r = i * s; r < r1; ++r)
          for (int c = j * s; c < c1; ++c) acc += img[r * w + c];
        box[t] = make_float2(acc, (float)((r1 - i * s) * (c1 - j * s)));
      }
      __syncthreads();
      const float reach = (float)a.wradius;
      for (int t = threadIdx.x; t < hs * wp; t += blockDim.x) {
        int line = t / wp, tc = t - line * wp;
        float c = wide_cell(tc - cp, w, s).x;
        int j0 = max((int)floorf((c - reach) / (float)s), 0);
        int j1 = min((int)floorf((c + reach) / (float)s), ws - 1);
        float2 acc = make_float2(0.f, 0.f);
        for (int j = j0; j <= j1; ++j) {
          float d = wide_cell(j, w, s).x - c;
          float e = expf(-d * d * a.kx);
          float2 v = box[line * ws + j];
          acc.x += e * v.x; acc.y += e * v.y;
        }
        rows[t] = acc;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < hp * wp; t += blockDim.x) {
        int tr = t / wp, col = t - tr * wp;
        float c = wide_cell(tr - cp, h, s).x;
        int i0 = max((int)floorf((c - reach) / (float)s), 0);
        int i1 = min((int)floorf((c + reach) / (float)s), hs - 1);
        float2 acc = make_float2(0.f, 0.f);
        for (int i = i0; i <= i1; ++i) {
          float d = wide_cell(i, h, s).x - c;
          float e = expf(-d * d * a.kx);
          float2 v = rows[i * wp + col];
          acc.x += e * v.x; acc.y += e * v.y;
        }
        cols[t] = acc;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < hp * w; t += blockDim.x) {
        int tr = t / w, x = t - tr * w;
        int own = x / s;
        float2 acc = make_float2(0.f, 0.f);
        for (int q = 0; q <= 2 * cp; ++q) {
          float2 cw = wide_cell(own + q - cp, w, s);
          float d = (float)x - cw.x;
          float e = cw.y * expf(-d * d * a.kz);
          float2 v = cols[tr * wp + own + q];
          acc.x += e * v.x; acc.y += e * v.y;
        }
        spread[t] = acc;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < hw; i += blockDim.x) {
        int y = i / w, x = i - y * w;
        int own = y / s;
        float2 acc = make_float2(0.f, 0.f);
        for (int q = 0; q <= 2 * cp; ++q) {
          float2 cw = wide_cell(own + q - cp, h, s);
          float d = (float)y - cw.x;
          float e = cw.y * expf(-d * d * a.kz);
          float2 v = spread[(own + q) * w + x];
          acc.x += e * v.x; acc.y += e * v.y;
        }
        float bgv = acc.x / acc.y;
        img[i] = with_background(a.dynamic, img[i], bgv);
      }
      __syncthreads();
      bg = nullptr;
    }
    (void)bg;
  }

  prep_finish(a, img, a.out + base, red);
}


// The direct blur in shared memory: the image inside its zero-padded rows P[h][pw] (R zeros on
// the left, at least R + 14 on the right, pw odd so that rows at stride pw fall in different
// banks) and the zero-padded row-blurred image Q[R + h + R + 16][w].  A thread takes eight
// consecutive outputs along the blur's direction and walks the taps eight at a time: eight taps
// (two 16-byte loads) and the 23 inputs they reach go into registers, then 128 FMAs, so a shared
// load serves several FMAs (the taps beyond 2R are zeros, adding exact zeros).  Each output sums
// its taps in increasing order with fmaf, the order of k_prep, so the results are the same bits;
// the taps inside the image are summed once per column and per row for the edge renormalization.
constexpr int PD_OUT = 16;  // outputs a thread takes along the blur
constexpr int PD_TB = 8;    // taps a step

__host__ __device__ inline int pd_pw(int w, int R) { return ((w + 2 * R + 2 * PD_OUT) | 1); }
__host__ __device__ inline int pd_qrows(int h, int R) { return h + 2 * R + 2 * PD_OUT; }
__host__ __device__ inline size_t pd_smem(int h, int w, int R) {
  return 4 * ((size_t)h * pd_pw(w, R) + (size_t)pd_qrows(h, R) * w);
}

__global__ void __launch_bounds__(256) k_prep_direct(PrepArgs a) {
  extern __shared__ float sm[];
  __shared__ __align__(16) float taps[128 + PD_TB];
  __shared__ float gsum[2][512];  // Σ taps inside the image, per column and per row
  __shared__ float red[2 * 8];
  const int b = blockIdx.x;
  const int h = a.h, w = a.w, hw = h * w, R = a.radius;
  const int pw = pd_pw(w, R), qr = pd_qrows(h, R);
  const int ntap = 2 * R + 1, nblk = (ntap + PD_TB - 1) / PD_TB;
  float* P = sm;           // [h][pw], the image at columns R … R + w − 1
  float* Q = P + h * pw;   // [qr][w], the row-blurred image at rows R … R + h − 1
  const size_t base = (size_t)b * hw;
  for (int d = threadIdx.x; d < nblk * PD_TB; d += blockDim.x) {
    const int dd = abs(d - R);
    taps[d] = d < ntap ? expf(-(float)(dd * dd) * a.k0) : 0.f;
  }
  for (int i = threadIdx.x; i < h * pw; i += blockDim.x) P[i] = 0.f;
  for (int i = threadIdx.x; i < R * w; i += blockDim.x) Q[i] = 0.f;
  for (int i = threadIdx.x; i < (qr - R - h) * w; i += blockDim.x) Q[(R + h) * w + i] = 0.f;
  __syncthreads();
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    const int r = i / w, c = i - r * w;
    P[r * pw + R + c] = prep_pixel(a, b, i);
  }
  for (int k = threadIdx.x; k < w + h; k += blockDim.x) {
    const int n = k < w ? w : h, c = k < w ? k : k - w;
    float g = 0.f;
    for (int x = max(c - R, 0); x <= min(c + R, n - 1); ++x) g += taps[x - c + R];
    gsum[k < w ? 0 : 1][c] = g;
  }
  __syncthreads();
  // along the rows: Q[R + r][c] = Σ_d taps[d] P[r][c + d] / gsum_col[c]; a thread takes row r,
  // columns c0 … c0 + 7 (threads of a warp: consecutive rows)
  const int cg = (w + PD_OUT - 1) / PD_OUT;
  for (int t = threadIdx.x; t < cg * h; t += blockDim.x) {
    const int r = t % h, c0 = (t / h) * PD_OUT;
    const float* src = P + r * pw + c0;
    float acc[PD_OUT];
#pragma unroll
    for (int k = 0; k < PD_OUT; ++k) acc[k] = 0.f;
    for (int d0 = 0; d0 < nblk * PD_TB; d0 += PD_TB) {
      float x[PD_OUT + PD_TB - 1];
      const float4 ta = *reinterpret_cast<const float4*>(taps + d0);
      const float4 tb = *reinterpret_cast<const float4*>(taps + d0 + 4);
      const float tv[PD_TB] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
      for (int k = 0; k < PD_OUT + PD_TB - 1; ++k) x[k] = src[d0 + k];
#pragma unroll
      for (int dd = 0; dd < PD_TB; ++dd)
#pragma unroll
        for (int k = 0; k < PD_OUT; ++k) acc[k] = fmaf(tv[dd], x[k + dd], acc[k]);
    }
#pragma unroll
    for (int k = 0; k < PD_OUT; ++k)
      if (c0 + k < w) Q[(R + r) * w + c0 + k] = acc[k] / gsum[0][c0 + k];
  }
  __syncthreads();
  // along the columns: the background, combined with the image in place (P's interior); a thread
  // takes column c, rows r0 … r0 + 7 (threads of a warp: consecutive columns)
  const int rg = (h + PD_OUT - 1) / PD_OUT;
  for (int t = threadIdx.x; t < rg * w; t += blockDim.x) {
    const int c = t % w, r0 = (t / w) * PD_OUT;
    const float* src = Q + r0 * w + c;
    float acc[PD_OUT];
#pragma unroll
    for (int k = 0; k < PD_OUT; ++k) acc[k] = 0.f;
    for (int d0 = 0; d0 < nblk * PD_TB; d0 += PD_TB) {
      float x[PD_OUT + PD_TB - 1];
      const float4 ta = *reinterpret_cast<const float4*>(taps + d0);
      const float4 tb = *reinterpret_cast<const float4*>(taps + d0 + 4);
      const float tv[PD_TB] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
      for (int k = 0; k < PD_OUT + PD_TB - 1; ++k) x[k] = src[(d0 + k) * w];
#pragma unroll
      for (int dd = 0; dd < PD_TB; ++dd)
#pragma unroll
        for (int k = 0; k < PD_OUT; ++k) acc[k] = fmaf(tv[dd], x[k + dd], acc[k]);
    }
#pragma unroll
    for (int k = 0; k < PD_OUT; ++k) {
      if (r0 + k < h) {
        float* px = P + (r0 + k) * pw + R + c;
        const float bgv = acc[k] / gsum[1][r0 + k];
        *px = with_background(a.dynamic, *px, bgv);
      }
    }
  }
  __syncthreads();
  // the combined image, contiguous, where Q was
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    const int r = i / w, c = i - r * w;
    Q[i] = P[r * pw + R + c];
  }
  __syncthreads();
  prep_finish(a, Q, a.out + base, red);
}

struct WideDims {
  int bin, hs, ws, hp, wp;
};

static WideDims wide_dims(int h, int w, float sigma) {
  WideDims d{};
  d.bin = (int)floorf(sigma / 6.f);
  if (d.bin < 2) return d;
  d.hs = (h + d.bin - 1) / d.bin;
  d.ws = (w + d.bin - 1) / d.bin;
  d.hp = d.hs + 6;
  d.wp = d.ws + 6;
  return d;
}

static long long scratch_floats(int h, int w, float sigma, int dynamic, bool smem) {
  long long per = 0;
  if (!smem) per += (long long)h * w;  // the row-blurred image
  if (dynamic && sigma > 0.f) {
    WideDims d = wide_dims(h, w, sigma);
    if (d.bin >= 2) per += 2LL * (d.hs * d.ws + d.hs * d.wp + d.hp * d.wp + (long long)d.hp * w);
  }
  return per;
}

static bool prep_smem(int h, int w) { return 2LL * h * w * 4 <= 160 * 1024; }

}  // namespace zeb

using namespace zeb;

extern "C" size_t zeb_prep_scratch_bytes(int n, int h, int w, float sigma) {
  if (n <= 0 || h <= 0 || w <= 0) return 0;
  long long per = scratch_floats(h, w, sigma, 1, prep_smem(h, w));
  if (!prep_smem(h, w) && per == 0) per = (long long)h * w;
  return (size_t)per * 4 * (size_t)n;
}

static int prep_launch(const void* raw, int pixel, int n, int src_h, int src_w, double factor, const float* static_bg,
                       int dynamic, float sigma, const float mask[3], int normalize, float* out, void* scratch,
                       void* stream) {
  ZEB_REQUIRE(raw && out && mask, ZEB_EARG, "prep: null pointer");
  ZEB_REQUIRE(factor >= 1.0 && factor <= 64.0, ZEB_EARG, "prep: reduction factor %g", factor);
  const int h = (int)floor((double)src_h / factor + 1e-9), w = (int)floor((double)src_w / factor + 1e-9);
  ZEB_REQUIRE(pixel >= 0 && pixel <= 2 && n >= 0 && h >= 4 && w >= 4 && dynamic >= 0 && dynamic <= 3, ZEB_EARG,
              "prep: bad arguments pixel=%d n=%d h=%d w=%d dynamic=%d", pixel, n, h, w, dynamic);
  if (n == 0) return ZEB_OK;
  PrepArgs a{};
  a.raw = raw; a.pixel = pixel; a.n = n; a.h = h; a.w = w; a.static_bg = static_bg;
  a.sh = src_h; a.sw = src_w; a.factor = factor;
  a.kwhole = fabs(factor - round(factor)) < 1e-9 && factor > 1.0 ? (int)round(factor) : 0;
  if (a.kwhole == 1) { a.kwhole = 0; a.factor = 1.0; }
  a.dynamic = (sigma > 0.f) ? dynamic : 0; a.sigma = sigma;
  a.mask[0] = mask[0]; a.mask[1] = mask[1]; a.mask[2] = mask[2];
  a.normalize = normalize; a.out = out;
  a.use_smem = prep_smem(h, w) ? 1 : 0;
  a.scratch_per = scratch_floats(h, w, sigma, a.dynamic, a.use_smem);
  a.scratch = (float*)scratch;
  ZEB_REQUIRE(a.scratch_per == 0 || scratch, ZEB_EARG, "prep: scratch needed (%lld floats per pattern)",
              a.scratch_per);
  if (a.dynamic) {
    WideDims d = wide_dims(h, w, sigma);
    a.bin = d.bin;
    if (d.bin < 2) {
      a.radius = (int)fmaxf(1.f, ceilf(3.f * sigma));
      ZEB_REQUIRE(a.radius <= 63, ZEB_ESIZE, "prep: blur radius %d", a.radius);
      a.k0 = (float)(1.0 / (2.0 * (double)sigma * sigma));
    } else {
      double sf = d.bin;
      double cs = sqrt((double)sigma * sigma - sf * sf - (sf * sf - 1.0) / 12.0);
      a.cpad = 3;
      a.wradius = (int)ceil(4.0 * cs);
      a.kx = (float)(1.0 / (2.0 * cs * cs));
      a.kz = (float)(1.0 / (2.0 * sf * sf));
    }
  }
  if (a.dynamic && a.bin < 2 && a.use_smem && h <= 512 && w <= 512 && 2 * a.radius + 1 <= 128) {
    const size_t dsm = pd_smem(h, w, a.radius);
    if (dsm <= 200 * 1024) {
      cudaFuncSetAttribute(k_prep_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
      k_prep_direct<<<n, 256, dsm, (cudaStream_t)stream>>>(a);
      return zeb_launch_check("prep (direct blur)");
    }
  }
  size_t smem = a.use_smem ? 2 * (size_t)h * w * 4 : 0;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_prep<<<n, 256, smem, (cudaStream_t)stream>>>(a);
  return zeb_launch_check("prep");
}

extern "C" int zeb_prep_ex(const void* raw, int pixel, int n, int h, int w, const float* static_bg, int dynamic,
                           float sigma, const float mask[3], int normalize, float* out, void* scratch,
                           void* stream) {
  return prep_launch(raw, pixel, n, h, w, 1.0, static_bg, dynamic, sigma, mask, normalize, out, scratch, stream);
}

extern "C" int zeb_prep_reduced(const void* raw, int pixel, int n, int src_h, int src_w, double factor,
                                const float* static_bg, int dynamic, float sigma, const float mask[3], int normalize,
                                float* out, void* scratch, void* stream) {
  return prep_launch(raw, pixel, n, src_h, src_w, factor, static_bg, dynamic, sigma, mask, normalize, out, scratch,
                     stream);
}

extern "C" int zeb_prep(const void* raw, int pixel, int n, int h, int w, const float* static_bg, int dynamic,
                        float sigma, const float mask[3], int normalize, float* out, void* stream) {
  ZEB_REQUIRE(zeb_prep_scratch_bytes(n, h, w, dynamic ? sigma : 0.f) == 0, ZEB_EARG,
              "prep: this size needs scratch (zeb_prep_ex)");
  return zeb_prep_ex(raw, pixel, n, h, w, static_bg, dynamic, sigma, mask, normalize, out, nullptr, stream);
}
