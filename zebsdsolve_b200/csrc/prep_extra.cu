// The preprocessing filters that follow the backgrounds: contrast-limited adaptive histogram
// equalization (CLAHE) and the band pass's difference of Gaussians, on a batch of f32 images in
// place; and the mean of a master over its point group after a filter that does not commute with
// it (CLAHE on the sheets).
//
// CLAHE (shaders/prep.wgsl stretch, clahe_hist, clahe_cdf, clahe_apply): each image stretched to
// [0, 1] between its extremes; padded by reflection at its top and left to a whole number of
// tiles; each tile's histogram of `bins` levels clipped at clip × the mean count per level, what
// was cut spread evenly over the levels (the remainder one count each to the first levels), and
// cumulated; a pixel takes its value from the four nearest tiles' tables, each read between its
// two nearest levels. The table arithmetic is float32 with every product and sum rounded on its
// own, in the order of the levels.
#include <algorithm>

#include "abi_util.cuh"

namespace zeb {

__global__ void __launch_bounds__(256) k_stretch(float* __restrict__ img, int hw) {
  __shared__ float red[2 * 8];
  float* p = img + (size_t)blockIdx.x * hw;
  float lo = 3.4e38f, hi = -3.4e38f;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    const float v = p[i];
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    red[wid] = lo;
    red[8 + wid] = hi;
  }
  __syncthreads();
  lo = red[0];
  hi = red[8];
  for (int k = 1; k < nw; ++k) {
    lo = fminf(lo, red[k]);
    hi = fmaxf(hi, red[8 + k]);
  }
  const float k = __frcp_rn(fmaxf(__fsub_rn(hi, lo), 1e-20f));
  for (int i = threadIdx.x; i < hw; i += blockDim.x) p[i] = __fmul_rn(__fsub_rn(p[i], lo), k);
}

struct ClaheArgs {
  float* img;
  int n, h, w, tiles, bins, pad_h, pad_w, tile_h, tile_w;
  float clip;
  unsigned* hist;  // [n][tiles²][bins]
  float* cdf;      // [n][tiles²][bins]
};

__device__ __forceinline__ int clahe_reflect(int i, int n, int pad) {
  if (n <= 1) return 0;
  int x = i - pad;
  if (x < 0) x = -x;
  if (x >= n) x = 2 * n - 2 - x;
  return min(max(x, 0), n - 1);
}

__global__ void k_clahe_hist(ClaheArgs a) {
  const int hp = a.h + a.pad_h, wp = a.w + a.pad_w;
  const long long total = (long long)a.n * hp * wp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / ((long long)hp * wp));
    const int r = (int)(t % ((long long)hp * wp));
    const int py = r / wp, px = r - py * wp;
    const int oy = clahe_reflect(py, a.h, a.pad_h), ox = clahe_reflect(px, a.w, a.pad_w);
    const float v = fminf(fmaxf(a.img[(size_t)b * a.h * a.w + oy * a.w + ox], 0.f), 1.f);
    const float top = (float)(a.bins - 1);
    const int bin = (int)fminf(fmaxf(__fmul_rn(v, top), 0.f), top);
    const int tile = (py / a.tile_h) * a.tiles + px / a.tile_w;
    atomicAdd(a.hist + ((size_t)b * a.tiles * a.tiles + tile) * a.bins + bin, 1u);
  }
}

__global__ void k_clahe_cdf(ClaheArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n * a.tiles * a.tiles) return;
  const size_t base = (size_t)t * a.bins;
  const float voxels = (float)max(a.tile_h * a.tile_w, 1);
  const float nb = (float)a.bins;
  const float limit = fmaxf(__fdiv_rn(__fmul_rn(a.clip, voxels), nb), 1.f);
  float sumc = 0.f;
  for (int i = 0; i < a.bins; ++i) sumc = __fadd_rn(sumc, fminf((float)a.hist[base + i], limit));
  const float clipped = __fsub_rn(voxels, sumc);
  const int residual = (int)__fsub_rn(clipped, __fmul_rn(nb, floorf(__fdiv_rn(clipped, nb))));
  const float redist = __fdiv_rn(__fsub_rn(clipped, (float)residual), nb);
  float acc = 0.f;
  for (int i = 0; i < a.bins; ++i) {
    float c = __fadd_rn(fminf((float)a.hist[base + i], limit), redist);
    if (i < residual) c = __fadd_rn(c, 1.f);
    acc = __fadd_rn(acc, c);
    a.cdf[base + i] = fminf(fmaxf(__fdiv_rn(acc, voxels), 0.f), 1.f);
  }
}

// WGSL's mix: a·(1 − t) + b·t, each operation rounded on its own
__device__ __forceinline__ float mix_rn(float x, float y, float t) {
  return __fadd_rn(__fmul_rn(x, __fsub_rn(1.f, t)), __fmul_rn(y, t));
}

__global__ void k_clahe_apply(ClaheArgs a) {
  const int hw = a.h * a.w;
  const long long total = (long long)a.n * hw;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / hw);
    const int pix = (int)(t % hw);
    const int row = pix / a.w, col = pix - row * a.w;
    const float v = fminf(fmaxf(a.img[t], 0.f), 1.f);
    const float tl = (float)(a.tiles - 1);
    const float gy = __fmul_rn(__fdiv_rn(__fadd_rn((float)row, 0.5f), (float)a.h), tl);
    const float gx = __fmul_rn(__fdiv_rn(__fadd_rn((float)col, 0.5f), (float)a.w), tl);
    const int y0 = (int)floorf(gy), x0 = (int)floorf(gx);
    const int y1 = min(y0 + 1, a.tiles - 1), x1 = min(x0 + 1, a.tiles - 1);
    const float fy = __fsub_rn(gy, (float)y0), fx = __fsub_rn(gx, (float)x0);
    const float bf = __fmul_rn(v, (float)(a.bins - 1));
    const int b0 = (int)fminf(fmaxf(floorf(bf), 0.f), (float)(a.bins - 2));
    const float fb = __fsub_rn(bf, (float)b0);
    const int b1 = b0 + 1;
    const size_t tb = (size_t)b * a.tiles * a.tiles;
    const float* c00 = a.cdf + (tb + y0 * a.tiles + x0) * a.bins;
    const float* c10 = a.cdf + (tb + y0 * a.tiles + x1) * a.bins;
    const float* c01 = a.cdf + (tb + y1 * a.tiles + x0) * a.bins;
    const float* c11 = a.cdf + (tb + y1 * a.tiles + x1) * a.bins;
    const float v00 = mix_rn(c00[b0], c00[b1], fb), v10 = mix_rn(c10[b0], c10[b1], fb);
    const float v01 = mix_rn(c01[b0], c01[b1], fb), v11 = mix_rn(c11[b0], c11[b1], fb);
    a.img[t] = mix_rn(mix_rn(v00, v10, fx), mix_rn(v01, v11, fx), fy);
  }
}

// prep.wgsl combine: a − b (op 0) or a / max(b, 1e-6) (op 1)
__global__ void k_combine(const float* __restrict__ x, const float* __restrict__ y, float* __restrict__ out,
                          long long count, int op) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += (long long)gridDim.x * blockDim.x)
    out[t] = op == 0 ? __fsub_rn(x[t], y[t]) : __fdiv_rn(x[t], fmaxf(y[t], 1e-6f));
}

// mastersph.wgsl symmetrize: each sheet pixel's direction d, the master (bilinear) at g·d for
// every operator g of the point group, averaged
__global__ void k_master_symmetrize(const float* __restrict__ src, float* __restrict__ dst, int side,
                                    const float* __restrict__ ops, int n_ops) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 2 * side * side) return;
  const int plane = side * side, pix = tid % plane;
  const float last = (float)(side - 1);
  const float3 d = square_to_sphere(2.f * (float)(pix % side) / last - 1.f, 2.f * (float)(pix / side) / last - 1.f,
                                    tid >= plane);
  float acc = 0.f;
  for (int g = 0; g < n_ops; ++g) {
    const float* m = ops + 9 * g;
    const float3 v = make_float3(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[3] * d.x + m[4] * d.y + m[5] * d.z,
                                 m[6] * d.x + m[7] * d.y + m[8] * d.z);
    acc += master_at<false>(src, normalize3(v), side);
  }
  dst[tid] = acc / (float)max(n_ops, 1);
}

static unsigned grid_for(long long count) {
  const long long blocks = (count + 255) / 256;
  return (unsigned)std::min<long long>(std::max<long long>(blocks, 1), 148LL * 64);
}

}  // namespace zeb

using namespace zeb;

extern "C" size_t zeb_clahe_scratch_bytes(int n, int tiles, int bins) {
  if (n <= 0 || tiles < 1 || bins < 2) return 0;
  return (size_t)n * tiles * tiles * bins * (sizeof(unsigned) + sizeof(float));
}

extern "C" int zeb_clahe(float* img, int n, int h, int w, int tiles, int bins, float clip, void* scratch, void* stream) {
  ZEB_REQUIRE(img && scratch && n >= 0 && h >= 1 && w >= 1 && tiles >= 1 && tiles <= 64 && bins >= 2 && bins <= 256 &&
                  clip > 0.f,
              ZEB_EARG, "clahe: bad arguments");
  if (n == 0) return ZEB_OK;
  ClaheArgs a{};
  a.img = img; a.n = n; a.h = h; a.w = w; a.tiles = tiles; a.bins = bins; a.clip = clip;
  a.pad_h = (tiles - h % tiles) % tiles;
  a.pad_w = (tiles - w % tiles) % tiles;
  a.tile_h = std::max(1, (h + a.pad_h) / tiles);
  a.tile_w = std::max(1, (w + a.pad_w) / tiles);
  const size_t cells = (size_t)n * tiles * tiles * bins;
  a.hist = (unsigned*)scratch;
  a.cdf = (float*)(a.hist + cells);
  cudaStream_t st = (cudaStream_t)stream;
  k_stretch<<<n, 256, 0, st>>>(img, h * w);
  if (cudaMemsetAsync(a.hist, 0, cells * sizeof(unsigned), st) != cudaSuccess) return zeb_launch_check("clahe memset");
  k_clahe_hist<<<grid_for((long long)n * (h + a.pad_h) * (w + a.pad_w)), 256, 0, st>>>(a);
  k_clahe_cdf<<<(n * tiles * tiles + 63) / 64, 64, 0, st>>>(a);
  k_clahe_apply<<<grid_for((long long)n * h * w), 256, 0, st>>>(a);
  return zeb_launch_check("clahe");
}

extern "C" int zeb_combine(const float* a, const float* b, float* out, long long count, int op, void* stream) {
  ZEB_REQUIRE(a && b && out && count >= 0 && (op == 0 || op == 1), ZEB_EARG, "combine: bad arguments");
  if (count == 0) return ZEB_OK;
  k_combine<<<grid_for(count), 256, 0, (cudaStream_t)stream>>>(a, b, out, count, op);
  return zeb_launch_check("combine");
}

extern "C" int zeb_master_symmetrize(const float* src, float* dst, int side, const float* ops, int n_ops,
                                     void* stream) {
  ZEB_REQUIRE(src && dst && ops && src != dst && side >= 3 && n_ops >= 1, ZEB_EARG, "master_symmetrize: bad arguments");
  const int total = 2 * side * side;
  k_master_symmetrize<<<(total + 255) / 256, 256, 0, (cudaStream_t)stream>>>(src, dst, side, ops, n_ops);
  return zeb_launch_check("master_symmetrize");
}
