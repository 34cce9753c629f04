// The master pattern as a function on the sphere: Gaussian smoothing in directions (not on the
// sheets, whose map is not conformal), the tangent-gradient table refinement reads, and the
// FP64 sampling of the master on a Gauss–Legendre grid for its harmonics.
#include "abi_util.cuh"

namespace zeb {

__device__ __forceinline__ float3 pixel_dir(int tid, int side) {
  const int plane = side * side;
  const int pix = tid % plane;
  const float last = (float)(side - 1);
  return square_to_sphere(2.f * (float)(pix % side) / last - 1.f, 2.f * (float)(pix / side) / last - 1.f, tid >= plane);
}

__device__ __forceinline__ void tangent_frame(float3 c, float3& e1, float3& e2) {
  float3 ref = fabsf(c.x) > 0.8f ? make_float3(0.f, 1.f, 0.f) : make_float3(1.f, 0.f, 0.f);
  e1 = normalize3(cross3(c, ref));
  e2 = cross3(c, e1);
}

// mastersph.wgsl:87-109 — each pixel direction averaged over a square lattice in its tangent plane.
__global__ void k_master_blur(const float* __restrict__ src, float* __restrict__ dst, int side, float step, float k,
                              int radius) {
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 2 * side * side) return;
  float3 d = pixel_dir(tid, side), e1, e2;
  tangent_frame(d, e1, e2);
  float acc = 0.f, wsum = 0.f;
  for (int i = -radius; i <= radius; ++i) {
    for (int j = -radius; j <= radius; ++j) {
      float a = (float)i * step, b = (float)j * step;
      float wgt = expf(-(a * a + b * b) * k);
      float3 v = normalize3(make_float3(d.x + a * e1.x + b * e2.x, d.y + a * e1.y + b * e2.y, d.z + a * e1.z + b * e2.z));
      acc += wgt * master_at<false>(src, v, side);
      wsum += wgt;
    }
  }
  dst[tid] = acc / wsum;
}

// mastersph.wgsl:124-138 — central differences a sheet pixel apart along two tangent directions.
__global__ void k_master_gradient(const float* __restrict__ src, float4* __restrict__ grad, int side) {
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 2 * side * side) return;
  float3 c = pixel_dir(tid, side), e1, e2;
  tangent_frame(c, e1, e2);
  const float h = 2.5066282746310002f / (float)side;  // sqrt(2π) / side
  float3 p1 = normalize3(make_float3(c.x + h * e1.x, c.y + h * e1.y, c.z + h * e1.z));
  float3 m1 = normalize3(make_float3(c.x - h * e1.x, c.y - h * e1.y, c.z - h * e1.z));
  float3 p2 = normalize3(make_float3(c.x + h * e2.x, c.y + h * e2.y, c.z + h * e2.z));
  float3 m2 = normalize3(make_float3(c.x - h * e2.x, c.y - h * e2.y, c.z - h * e2.z));
  float g1 = (master_at<false>(src, p1, side) - master_at<false>(src, m1, side)) / (2.f * h);
  float g2 = (master_at<false>(src, p2, side) - master_at<false>(src, m2, side)) / (2.f * h);
  grad[tid] = make_float4(g1 * e1.x + g2 * e2.x, g1 * e1.y + g2 * e2.y, g1 * e1.z + g2 * e2.z, src[tid]);
}

// lambert.zig:28-64 in FP64: the square coordinates of v and the bilinear sample of its sheet.
__device__ double master_at_f64(const float* __restrict__ sheets, int side, double vx, double vy, double vz) {
  const double pi = 3.14159265358979323846;
  double kz = fabs(vz);
  double u = 0.0, w = 0.0;
  if (kz < 1.0 - 1e-14) {
    double xn = sqrt(fmax(pi * (1.0 - kz) / 2.0, 0.0));
    double ax = fabs(vx), ay = fabs(vy);
    double sc = sqrt(pi / 2.0);
    if (ax >= ay) {
      u = xn;
      w = (4.0 * xn / pi) * atan2(ay, fmax(ax, 1e-300));
    } else {
      u = (4.0 * xn / pi) * atan2(ax, fmax(ay, 1e-300));
      w = xn;
    }
    u = (u / sc) * (vx < 0 ? -1.0 : 1.0);
    w = (w / sc) * (vy < 0 ? -1.0 : 1.0);
  }
  const float* sheet = sheets + (vz >= 0 ? 0 : (size_t)side * side);
  double last = (double)(side - 1);
  double fj = fmin(fmax((u + 1.0) * 0.5 * last, 0.0), last);
  double fi = fmin(fmax((w + 1.0) * 0.5 * last, 0.0), last);
  int c0 = (int)floor(fj), r0 = (int)floor(fi);
  int c1 = min(c0 + 1, side - 1), r1 = min(r0 + 1, side - 1);
  double tj = fj - c0, ti = fi - r0;
  double a = sheet[r0 * side + c0], b = sheet[r0 * side + c1], c = sheet[r1 * side + c0], d = sheet[r1 * side + c1];
  return (a * (1 - tj) + b * tj) * (1 - ti) + (c * (1 - tj) + d * tj) * ti;
}

// master.zig:680-688 — the master at every grid direction (sh.zig:138-143).
__global__ void k_master_sample_grid(const float* __restrict__ sheets, int side, const double* __restrict__ x,
                                     int n_theta, int n_phi, double* __restrict__ out) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n_theta * n_phi) return;
  int y = (int)(t / n_phi), j = (int)(t % n_phi);
  double ct = x[y];
  double st = sqrt(fmax(0.0, 1.0 - ct * ct));
  double phi = 2.0 * 3.14159265358979323846 * (double)j / (double)n_phi;
  out[t] = master_at_f64(sheets, side, st * cos(phi), st * sin(phi), ct);
}

}  // namespace zeb

using namespace zeb;

extern "C" int zeb_master_blur_pass(const float* src, float* dst, int side, float step, float k, int radius,
                                    void* stream) {
  ZEB_REQUIRE(src && dst && src != dst && side >= 3 && radius >= 0 && radius <= 16, ZEB_EARG,
              "master_blur_pass: bad arguments side=%d radius=%d", side, radius);
  int total = 2 * side * side;
  k_master_blur<<<(total + 255) / 256, 256, 0, (cudaStream_t)stream>>>(src, dst, side, step, k, radius);
  return zeb_launch_check("master_blur_pass");
}

extern "C" int zeb_master_gradient(const float* sheets, float* grad4, int side, void* stream) {
  ZEB_REQUIRE(sheets && grad4 && side >= 3, ZEB_EARG, "master_gradient: bad arguments side=%d", side);
  int total = 2 * side * side;
  k_master_gradient<<<(total + 255) / 256, 256, 0, (cudaStream_t)stream>>>(sheets, (float4*)grad4, side);
  return zeb_launch_check("master_gradient");
}

// Each sheet pixel with its right-hand neighbour side by side: vpair[i] = (M[i], M[i+1]),
// gpair[i] = (grad4[i], grad4[i+1]) (the last column repeats itself; bilinear lookups never read
// it), so a lookup reads one 8- or 32-byte record per row instead of two scattered texels.
__global__ void k_master_pairs(const float* __restrict__ sheets, const float4* __restrict__ grad4, int side,
                               float2* __restrict__ vpair, float4* __restrict__ gpair) {
  const long long total = 2LL * side * side;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int c = (int)(i % side);
  const long long k = c + 1 < side ? i + 1 : i;
  vpair[i] = make_float2(sheets[i], sheets[k]);
  gpair[2 * i] = grad4[i];
  gpair[2 * i + 1] = grad4[k];
}

extern "C" int zeb_master_pairs(const float* sheets, const float* grad4, int side, float* vpair, float* gpair,
                                void* stream) {
  ZEB_REQUIRE(sheets && grad4 && vpair && gpair && side >= 3, ZEB_EARG, "master_pairs: bad arguments side=%d", side);
  const long long total = 2LL * side * side;
  k_master_pairs<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(sheets, (const float4*)grad4, side,
                                                                                  (float2*)vpair, (float4*)gpair);
  return zeb_launch_check("master_pairs");
}

// The 2 × 2 neighbourhood of every texel in one 32-byte record of FP16 values: the master at the
// texel, its right-hand neighbour, the one below and the one below right, then their tangent
// gradients (xyz each) in the same order. A texel on the last row or column repeats itself where a
// neighbour would fall off the sheet (the lookups never start there).
__global__ void k_master_quads(const float4* __restrict__ grad4, int side, uint4* __restrict__ quads) {
  const long long total = 2LL * side * side;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int c = (int)(i % side), r = (int)((i / side) % side);
  const long long right = c + 1 < side ? 1 : 0, down = r + 1 < side ? side : 0;
  const float4 g[4] = {grad4[i], grad4[i + right], grad4[i + down], grad4[i + down + right]};
  uint32_t h[8];  // per texel (gx, gy) then (gz, value): the pairs the packed bilinear takes
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    h[2 * k] = zeb_half2(g[k].x, g[k].y);
    h[2 * k + 1] = zeb_half2(g[k].z, g[k].w);
  }
  quads[2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
  quads[2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

extern "C" int zeb_master_quads(const float* grad4, int side, void* quads, void* stream) {
  ZEB_REQUIRE(grad4 && quads && side >= 3, ZEB_EARG, "master_quads: bad arguments side=%d", side);
  ZEB_REQUIRE(((uintptr_t)quads & 31) == 0, ZEB_EARG, "master_quads: quads must be 32-byte aligned");
  const long long total = 2LL * side * side;
  k_master_quads<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>((const float4*)grad4, side,
                                                                                  (uint4*)quads);
  return zeb_launch_check("master_quads");
}

extern "C" int zeb_master_sample_grid(const float* sheets, int side, const double* x, int n_theta, int n_phi,
                                      double* out, void* stream) {
  ZEB_REQUIRE(sheets && x && out && side >= 2 && n_theta >= 1 && n_phi >= 1, ZEB_EARG,
              "master_sample_grid: bad arguments");
  long long total = (long long)n_theta * n_phi;
  k_master_sample_grid<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(sheets, side, x, n_theta,
                                                                                         n_phi, out);
  return zeb_launch_check("master_sample_grid");
}
