// (c) The detector side: refinement of each item's orientation on the detector, its NMI, chance
// decoys and simulated patterns.
//
// k_refine is one thread block per item for the whole refinement: the preprocessed pattern sits
// in shared memory across the iters + 1 passes; each pass sums the 19 rotation-only
// Gauss–Newton sums over the masked pixels (detector.wgsl:329-363), one thread takes the step
// (refine_item, detector.wgsl:561-640: NCC, gradient, J'J, accept/reject with the curvature
// scale μ adapted by the gain ratio, the 3×3 solve, the step clipped to max_step), and the block
// goes on from the new orientation.  The NMI of the best orientation follows in the same block
// (detector.wgsl:744-832), then the record (collect, detector.wgsl:545-558).
#include "abi_util.cuh"

namespace zeb {

struct DetArgs {
  const float* pats;
  const float4* items;
  const float* seeds;
  int seed_stride;
  int n, h, w;
  float3 c0, c1, c2;
  float mask[3];
  const float* master;   // plain sheets (zeb_project)
  const float2* vpair;   // value pairs (zeb_master_pairs)
  const float* gpair;    // gradient pairs (zeb_master_pairs)
  int side;
  zeb_refine_opts_t o;
  float* records;
  int pat_smem, sim_smem;
  int draws;
  float* chance;
};

__device__ __forceinline__ bool in_mask(const DetArgs& a, int row, int col) {
  float dr = (float)row - a.mask[0], dc = (float)col - a.mask[1];
  return zeb_in_circle(dr, dc, a.mask[2]);
}

__device__ __forceinline__ float3 ray_dir(const DetArgs& a, float3 t, int row, int col) {
  return normalize3(make_float3(a.c0.x * row + a.c1.x * col + t.x, a.c0.y * row + a.c1.y * col + t.y,
                                a.c0.z * row + a.c1.z * col + t.z));
}

// symmetric 3×3 (xx, xy, xz, yy, yz, zz) by Cramer's rule (detector.wgsl:519-527)
__device__ float3 solve3(const float* hm, float3 g) {
  float m00 = hm[0], m01 = hm[1], m02 = hm[2], m11 = hm[3], m12 = hm[4], m22 = hm[5];
  float det = m00 * (m11 * m22 - m12 * m12) - m01 * (m01 * m22 - m12 * m02) + m02 * (m01 * m12 - m11 * m02);
  if (fabsf(det) < 1e-30f) return make_float3(0.f, 0.f, 0.f);
  // columns of m: c0 = (m00, m01, m02), c1 = (m01, m11, m12), c2 = (m02, m12, m22)
  float x = g.x * (m11 * m22 - m12 * m12) - m01 * (g.y * m22 - m12 * g.z) + m02 * (g.y * m12 - m11 * g.z);
  float y = m00 * (g.y * m22 - g.z * m12) - g.x * (m01 * m22 - m12 * m02) + m02 * (m01 * g.z - g.y * m02);
  float z = m00 * (m11 * g.z - m12 * g.y) - m01 * (m01 * g.z - g.y * m02) + g.x * (m01 * m12 - m11 * m02);
  return make_float3(x / det, y / det, z / det);
}

// NMI of the pattern in `pat` against the master at orientation q (detector.wgsl:744-832).
// `sims` (shared, h·w floats) caches the simulation between the passes when given.
__device__ float nmi_block(const DetArgs& a, const float* pat, float* sims, float3 t, float4 q, int nbins,
                           uint32_t* hist, float* red) {
  const int hw = a.h * a.w;
  float ext[4] = {3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f};
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    int row = i / a.w, col = i - row * a.w;
    if (!in_mask(a, row, col)) continue;
    float e = pat[i];
    float s = master_at_pair(a.vpair, qrot(q, ray_dir(a, t, row, col)), a.side);
    if (sims) sims[i] = s;
    ext[0] = fminf(ext[0], e); ext[1] = fmaxf(ext[1], e);
    ext[2] = fminf(ext[2], s); ext[3] = fmaxf(ext[3], s);
  }
  for (int i = threadIdx.x; i < nbins * nbins; i += blockDim.x) hist[i] = 0u;
  // min / max across the block
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ext[0] = fminf(ext[0], __shfl_xor_sync(0xffffffffu, ext[0], o));
    ext[1] = fmaxf(ext[1], __shfl_xor_sync(0xffffffffu, ext[1], o));
    ext[2] = fminf(ext[2], __shfl_xor_sync(0xffffffffu, ext[2], o));
    ext[3] = fmaxf(ext[3], __shfl_xor_sync(0xffffffffu, ext[3], o));
  }
  if (lane == 0)
    for (int k = 0; k < 4; ++k) red[k * nw + wid] = ext[k];
  __syncthreads();
  float r[4] = {3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f};
  for (int w = 0; w < nw; ++w) {
    r[0] = fminf(r[0], red[0 * nw + w]); r[1] = fmaxf(r[1], red[1 * nw + w]);
    r[2] = fminf(r[2], red[2 * nw + w]); r[3] = fmaxf(r[3], red[3 * nw + w]);
  }
  __syncthreads();
  const float ke = (float)nbins / fmaxf(r[1] - r[0], 1e-20f);
  const float ks = (float)nbins / fmaxf(r[3] - r[2], 1e-20f);
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    int row = i / a.w, col = i - row * a.w;
    if (!in_mask(a, row, col)) continue;
    float e = pat[i];
    float s = sims ? sims[i] : master_at_pair(a.vpair, qrot(q, ray_dir(a, t, row, col)), a.side);
    uint32_t be = min((uint32_t)((e - r[0]) * ke), (uint32_t)(nbins - 1));
    uint32_t bs = min((uint32_t)((s - r[2]) * ks), (uint32_t)(nbins - 1));
    atomicAdd(&hist[be * nbins + bs], 1u);
  }
  __syncthreads();
  float acc[3] = {0.f, 0.f, 0.f};  // −Σ c log c (joint), −Σ (marginals), N
  for (int i = threadIdx.x; i < nbins * nbins; i += blockDim.x) {
    float c = (float)hist[i];
    acc[2] += c;
    if (c > 0.f) acc[0] -= c * logf(c);
  }
  if ((int)threadIdx.x < nbins) {
    float rs = 0.f, cs = 0.f;
    for (int k = 0; k < nbins; ++k) {
      rs += (float)hist[threadIdx.x * nbins + k];
      cs += (float)hist[k * nbins + threadIdx.x];
    }
    if (rs > 0.f) acc[1] -= rs * logf(rs);
    if (cs > 0.f) acc[1] -= cs * logf(cs);
  }
  block_sums<3>(acc, red);
  const float nn = fmaxf(acc[2], 1.f);
  const float h_joint = logf(nn) + acc[0] / nn;
  const float h_marg = 2.f * logf(nn) + acc[1] / nn;
  return h_marg > 1e-12f ? 2.f * (h_marg - h_joint) / h_marg : 0.f;
}

// One step of refine_item (detector.wgsl:561-640) from the 19 sums s of the orientation q just
// evaluated: NCC, gradient and J'J; accept (tracking the best) or reject, the curvature scale μ
// adapted by the gain ratio; then the damped 3×3 solve, clipped to max_step, from the best
// orientation.  q_next: the next orientation to evaluate (the best after the last pass).
__device__ void refine_step(const zeb_refine_opts_t& o, int iter, float4 q, const float* s, float& best, float& mu,
                            float* g_best, float* h_best, float& last_good, float& promised, float& step_len,
                            float& accepted, float4& q_best, float4& q_next) {
  const float n = fmaxf(s[0], 1.f);
  const float mean = s[1] / n;
  const float var_n = s[2] - n * mean * mean;
  float ncc = -2.f, g[3] = {0.f, 0.f, 0.f}, hs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (var_n > 1e-12f) {
    const float inv = rsqrtf(var_n);
    ncc = s[3] * inv;
    const float sd[3] = {s[4], s[5], s[6]};
    float au[3];
    for (int k = 0; k < 3; ++k) au[k] = (s[7 + k] - mean * sd[k]) * inv;
    for (int k = 0; k < 3; ++k) g[k] = (s[10 + k] - ncc * au[k]) * inv;
    const float iv = inv * inv;
    hs[0] = (s[13] - sd[0] * sd[0] / n - au[0] * au[0]) * iv;
    hs[1] = (s[16] - sd[0] * sd[1] / n - au[0] * au[1]) * iv;
    hs[2] = (s[17] - sd[0] * sd[2] / n - au[0] * au[2]) * iv;
    hs[3] = (s[14] - sd[1] * sd[1] / n - au[1] * au[1]) * iv;
    hs[4] = (s[18] - sd[1] * sd[2] / n - au[1] * au[2]) * iv;
    hs[5] = (s[15] - sd[2] * sd[2] / n - au[2] * au[2]) * iv;
  }
  if (ncc > best) {
    if (accepted > 0.5f && promised > 1e-6f) {
      float rho = (ncc - best) / promised;
      mu = fminf(fmaxf(mu * (2.f - rho), mu / 3.f), mu * 3.f);
    }
    q_best = q;
    best = ncc;
    for (int k = 0; k < 3; ++k) g_best[k] = g[k];
    for (int k = 0; k < 6; ++k) h_best[k] = hs[k];
    last_good = step_len;
    accepted += 1.f;
  } else {
    mu = mu * 3.f;
  }
  mu = fminf(fmaxf(mu, o.scale_min), o.scale_max);
  if (iter < o.iters) {
    float hh[6];
    for (int k = 0; k < 6; ++k) hh[k] = h_best[k] * mu;
    float tr = fmaxf(hh[0] + hh[3] + hh[5], 1e-20f);
    hh[0] += 1e-6f * tr; hh[3] += 1e-6f * tr; hh[5] += 1e-6f * tr;
    float3 gg = make_float3(g_best[0], g_best[1], g_best[2]);
    float3 stp = solve3(hh, gg);
    float len = sqrtf(dot3(stp, stp));
    if (len > o.max_step) {
      float k = o.max_step / len;
      stp = make_float3(stp.x * k, stp.y * k, stp.z * k);
    }
    float quad = hh[0] * stp.x * stp.x + hh[3] * stp.y * stp.y + hh[5] * stp.z * stp.z +
                 2.f * (hh[1] * stp.x * stp.y + hh[2] * stp.x * stp.z + hh[4] * stp.y * stp.z);
    promised = dot3(gg, stp) - 0.5f * quad;
    step_len = sqrtf(dot3(stp, stp));
    float4 qn = qmul(qexp(stp), q_best);
    float nq = sqrtf(qn.x * qn.x + qn.y * qn.y + qn.z * qn.z + qn.w * qn.w);
    q_next = nq > 0.f ? make_float4(qn.x / nq, qn.y / nq, qn.z / nq, qn.w / nq) : make_float4(1.f, 0.f, 0.f, 0.f);
  } else {
    q_next = q_best;
  }
}

__global__ void __launch_bounds__(256) k_refine_direct(DetArgs a) {
  extern __shared__ float smf[];
  __shared__ float red[24 * 8];
  __shared__ uint32_t hist[32 * 32];
  __shared__ float4 sh_q;
  const int b = blockIdx.x;
  const int hw = a.h * a.w;
  const float4 it = a.items[b];
  const float3 t = make_float3(it.x, it.y, it.z);
  const float* gpat = a.pats + (size_t)(int)it.w * hw;
  float* pat = smf;
  float* sims = a.sim_smem ? smf + hw : nullptr;
  if (a.pat_smem) {
    for (int i = threadIdx.x; i < hw; i += blockDim.x) pat[i] = gpat[i];
  } else {
    pat = (float*)gpat;
  }
  // refinement state (thread 0's registers): detector.wgsl:73-77
  const float* sd0 = a.seeds + (size_t)b * a.seed_stride;
  float4 q_best = make_float4(sd0[0], sd0[1], sd0[2], sd0[3]);
  float best = -2.f, mu = a.o.scale0, g_best[3] = {0.f, 0.f, 0.f}, h_best[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float last_good = 0.f, promised = 0.f, step_len = 0.f, accepted = 0.f;
  if (threadIdx.x == 0) sh_q = q_best;
  __syncthreads();

  for (int iter = 0; iter <= a.o.iters; ++iter) {
    const float4 q = sh_q;
    float s[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) s[k] = 0.f;
    for (int i = threadIdx.x; i < hw; i += blockDim.x) {
      int row = i / a.w, col = i - row * a.w;
      if (!in_mask(a, row, col)) continue;
      float3 c = qrot(q, ray_dir(a, t, row, col));
      float4 m = grad_at_pair(a.gpair, c, a.side);
      float3 d = cross3(c, make_float3(m.x, m.y, m.z));
      float e = pat[i];
      s[0] += 1.f; s[1] += m.w; s[2] += m.w * m.w; s[3] += m.w * e;
      s[4] += d.x; s[5] += d.y; s[6] += d.z;
      s[7] += m.w * d.x; s[8] += m.w * d.y; s[9] += m.w * d.z;
      s[10] += e * d.x; s[11] += e * d.y; s[12] += e * d.z;
      s[13] += d.x * d.x; s[14] += d.y * d.y; s[15] += d.z * d.z;
      s[16] += d.x * d.y; s[17] += d.x * d.z; s[18] += d.y * d.z;
    }
    block_sums<19>(s, red);
    if (threadIdx.x == 0) {
      float4 qn = q_best;
      refine_step(a.o, iter, q, s, best, mu, g_best, h_best, last_good, promised, step_len, accepted, q_best, qn);
      sh_q = qn;
    }
    __syncthreads();
  }
  const float4 qf = sh_q;
  float v = nmi_block(a, pat, sims, t, qf, a.o.nmi_bins, hist, red);
  if (threadIdx.x == 0) {
    float* r = a.records + (size_t)b * 8;
    r[0] = qf.x; r[1] = qf.y; r[2] = qf.z; r[3] = qf.w;
    r[4] = best; r[5] = v; r[6] = last_good; r[7] = a.o.stamp;
  }
}

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
  uint32_t v = x * 747796405u + 2891336453u;
  uint32_t w = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (w >> 22u) ^ w;
}

__device__ __forceinline__ float unit_rand(uint32_t x) { return (float)(hash_u32(x) >> 8u) / 16777216.f; }

// detector.wgsl:296-308 — Shoemake's uniform rotation, per item and draw
__device__ __forceinline__ float4 decoy_q(uint32_t b, uint32_t draw) {
  uint32_t s = hash_u32(b + 1u) ^ (draw * 0x9e3779b9u);
  float u1 = unit_rand(s);
  float a2 = unit_rand(s + 1u) * ZEB_TAU;
  float a3 = unit_rand(s + 2u) * ZEB_TAU;
  float ra = sqrtf(1.f - u1), rb = sqrtf(u1);
  return make_float4(ra * sinf(a2), ra * cosf(a2), rb * sinf(a3), rb * cosf(a3));
}

__global__ void __launch_bounds__(256) k_chance_direct(DetArgs a) {
  extern __shared__ float smf[];
  __shared__ float red[24 * 8];
  __shared__ uint32_t hist[32 * 32];
  const int b = blockIdx.x, draw = blockIdx.y;
  const int hw = a.h * a.w;
  const float4 it = a.items[b];
  const float3 t = make_float3(it.x, it.y, it.z);
  const float* gpat = a.pats + (size_t)(int)it.w * hw;
  float* pat = smf;
  float* sims = a.sim_smem ? smf + hw : nullptr;
  if (a.pat_smem) {
    for (int i = threadIdx.x; i < hw; i += blockDim.x) pat[i] = gpat[i];
  } else {
    pat = (float*)gpat;
  }
  __syncthreads();
  float4 q = decoy_q((uint32_t)b, (uint32_t)draw);
  float v = nmi_block(a, pat, sims, t, q, a.o.nmi_bins, hist, red);
  if (threadIdx.x == 0) a.chance[(size_t)draw * a.n + b] = v;
}

__global__ void k_project(DetArgs a, const float* __restrict__ poses, float* __restrict__ sims) {
  const int hw = a.h * a.w;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)a.n * hw) return;
  int b = (int)(t / hw), pix = (int)(t % hw);
  const float* p = poses + (size_t)b * 8;
  float3 tt = make_float3(p[0], p[1], p[2]);
  float4 q = make_float4(p[4], p[5], p[6], p[7]);
  int row = pix / a.w, col = pix - row * a.w;
  sims[t] = master_at(a.master, qrot(q, ray_dir(a, tt, row, col)), a.side);
}

// ── the same with the masked pixels compacted once per block ──
//
// The block first lists its item's masked pixels in raster order, each as (detector ray in the
// sample frame, pattern value) in shared memory; every pass then runs over that list alone: no
// mask test, no index arithmetic and no ray normalization per pixel and pass, and the sphere →
// square map with fast arithmetic.  For detectors whose list fits in shared memory.

// px[0..npix) ← (ray, value) of the masked pixels of the pattern at gpat; returns npix
__device__ int compact_pixels(const DetArgs& a, const float* gpat, float3 t, float4* px, int* wcnt) {
  const int hw = a.h * a.w;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int out = 0;
  for (int base = 0; base < hw; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int row = i / a.w, col = i - row * a.w;
    const bool m = i < hw && in_mask(a, row, col);
    const unsigned bal = __ballot_sync(0xffffffffu, m);
    if (lane == 0) wcnt[wid] = __popc(bal);
    __syncthreads();
    int off = out, tot = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < wid) off += wcnt[w];
      tot += wcnt[w];
    }
    if (m) {
      const float3 d = ray_dir(a, t, row, col);
      px[off + __popc(bal & ((1u << lane) - 1u))] = make_float4(d.x, d.y, d.z, __ldg(gpat + i));
    }
    out += tot;
    __syncthreads();
  }
  return out;
}

// NMI over the compacted pixels (detector.wgsl:744-832)
__device__ float nmi_compact(const DetArgs& a, const float4* px, int npix, float4 q, int nbins, uint32_t* hist,
                             float* red) {
  float ext[4] = {3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f};
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const float4 p = px[k];
    const float sv = master_at_pair(a.vpair, qrot(q, make_float3(p.x, p.y, p.z)), a.side);
    ext[0] = fminf(ext[0], p.w); ext[1] = fmaxf(ext[1], p.w);
    ext[2] = fminf(ext[2], sv); ext[3] = fmaxf(ext[3], sv);
  }
  for (int i = threadIdx.x; i < nbins * nbins; i += blockDim.x) hist[i] = 0u;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ext[0] = fminf(ext[0], __shfl_xor_sync(0xffffffffu, ext[0], o));
    ext[1] = fmaxf(ext[1], __shfl_xor_sync(0xffffffffu, ext[1], o));
    ext[2] = fminf(ext[2], __shfl_xor_sync(0xffffffffu, ext[2], o));
    ext[3] = fmaxf(ext[3], __shfl_xor_sync(0xffffffffu, ext[3], o));
  }
  if (lane == 0)
    for (int k = 0; k < 4; ++k) red[k * nw + wid] = ext[k];
  __syncthreads();
  float r[4] = {3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f};
  for (int w = 0; w < nw; ++w) {
    r[0] = fminf(r[0], red[0 * nw + w]); r[1] = fmaxf(r[1], red[1 * nw + w]);
    r[2] = fminf(r[2], red[2 * nw + w]); r[3] = fmaxf(r[3], red[3 * nw + w]);
  }
  __syncthreads();
  const float ke = (float)nbins / fmaxf(r[1] - r[0], 1e-20f);
  const float ks = (float)nbins / fmaxf(r[3] - r[2], 1e-20f);
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const float4 p = px[k];
    const float sv = master_at_pair(a.vpair, qrot(q, make_float3(p.x, p.y, p.z)), a.side);
    const uint32_t be = min((uint32_t)((p.w - r[0]) * ke), (uint32_t)(nbins - 1));
    const uint32_t bs = min((uint32_t)((sv - r[2]) * ks), (uint32_t)(nbins - 1));
    atomicAdd(&hist[be * nbins + bs], 1u);
  }
  __syncthreads();
  float acc[3] = {0.f, 0.f, 0.f};  // −Σ c log c (joint), −Σ (marginals), N
  for (int i = threadIdx.x; i < nbins * nbins; i += blockDim.x) {
    float c = (float)hist[i];
    acc[2] += c;
    if (c > 0.f) acc[0] -= c * logf(c);
  }
  if ((int)threadIdx.x < nbins) {
    float rs = 0.f, cs = 0.f;
    for (int k = 0; k < nbins; ++k) {
      rs += (float)hist[threadIdx.x * nbins + k];
      cs += (float)hist[k * nbins + threadIdx.x];
    }
    if (rs > 0.f) acc[1] -= rs * logf(rs);
    if (cs > 0.f) acc[1] -= cs * logf(cs);
  }
  block_sums<3>(acc, red);
  const float nn = fmaxf(acc[2], 1.f);
  const float h_joint = logf(nn) + acc[0] / nn;
  const float h_marg = 2.f * logf(nn) + acc[1] / nn;
  return h_marg > 1e-12f ? 2.f * (h_marg - h_joint) / h_marg : 0.f;
}

__global__ void __launch_bounds__(256, 3) k_refine(DetArgs a) {
  extern __shared__ float4 px[];
  __shared__ float red[24 * 8];
  __shared__ uint32_t hist[32 * 32];
  __shared__ int wcnt[8];
  __shared__ float4 sh_q;
  const int b = blockIdx.x;
  const int hw = a.h * a.w;
  const float4 it = a.items[b];
  const float3 t = make_float3(it.x, it.y, it.z);
  const int npix = compact_pixels(a, a.pats + (size_t)(int)it.w * hw, t, px, wcnt);
  // refinement state (thread 0's registers): detector.wgsl:73-77
  const float* sd0 = a.seeds + (size_t)b * a.seed_stride;
  float4 q_best = make_float4(sd0[0], sd0[1], sd0[2], sd0[3]);
  float best = -2.f, mu = a.o.scale0, g_best[3] = {0.f, 0.f, 0.f}, h_best[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float last_good = 0.f, promised = 0.f, step_len = 0.f, accepted = 0.f;
  if (threadIdx.x == 0) sh_q = q_best;
  __syncthreads();

  for (int iter = 0; iter <= a.o.iters; ++iter) {
    const float4 q = sh_q;
    float s[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) s[k] = 0.f;
    for (int k = threadIdx.x; k < npix; k += blockDim.x) {
      const float4 p = px[k];
      const float3 c = qrot(q, make_float3(p.x, p.y, p.z));
      const float4 m = grad_at_pair(a.gpair, c, a.side);
      const float3 d = cross3(c, make_float3(m.x, m.y, m.z));
      const float e = p.w;
      s[1] += m.w; s[2] += m.w * m.w; s[3] += m.w * e;
      s[4] += d.x; s[5] += d.y; s[6] += d.z;
      s[7] += m.w * d.x; s[8] += m.w * d.y; s[9] += m.w * d.z;
      s[10] += e * d.x; s[11] += e * d.y; s[12] += e * d.z;
      s[13] += d.x * d.x; s[14] += d.y * d.y; s[15] += d.z * d.z;
      s[16] += d.x * d.y; s[17] += d.x * d.z; s[18] += d.y * d.z;
    }
    block_sums<19>(s, red);
    s[0] = (float)npix;
    if (threadIdx.x == 0) {
      float4 qn = q_best;
      refine_step(a.o, iter, q, s, best, mu, g_best, h_best, last_good, promised, step_len, accepted, q_best, qn);
      sh_q = qn;
    }
    __syncthreads();
  }
  const float4 qf = sh_q;
  float v = nmi_compact(a, px, npix, qf, a.o.nmi_bins, hist, red);
  if (threadIdx.x == 0) {
    float* r = a.records + (size_t)b * 8;
    r[0] = qf.x; r[1] = qf.y; r[2] = qf.z; r[3] = qf.w;
    r[4] = best; r[5] = v; r[6] = last_good; r[7] = a.o.stamp;
  }
}

__global__ void __launch_bounds__(256, 3) k_chance(DetArgs a) {
  extern __shared__ float4 px[];
  __shared__ float red[24 * 8];
  __shared__ uint32_t hist[32 * 32];
  __shared__ int wcnt[8];
  const int b = blockIdx.x, draw = blockIdx.y;
  const int hw = a.h * a.w;
  const float4 it = a.items[b];
  const int npix = compact_pixels(a, a.pats + (size_t)(int)it.w * hw, make_float3(it.x, it.y, it.z), px, wcnt);
  const float4 q = decoy_q((uint32_t)b, (uint32_t)draw);
  const float v = nmi_compact(a, px, npix, q, a.o.nmi_bins, hist, red);
  if (threadIdx.x == 0) a.chance[(size_t)draw * a.n + b] = v;
}

// The records' orientations reduced to the fundamental zone of a group (the landing's
// reduction, sym.zig:120-131): the symmetry-equivalent g·q of largest w (unit norm, w >= 0), ties
// within 1e-12 keeping the first; FP64 with every product and sum rounded on its own (no fused
// multiply-add), in the order of the host's reduction.
__device__ __forceinline__ double4 qstd_d(double4 q) {
  double s = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q.x, q.x), __dmul_rn(q.y, q.y)), __dmul_rn(q.z, q.z)),
                       __dmul_rn(q.w, q.w));
  double nrm = sqrt(s);
  if (nrm == 0.0) nrm = 1.0;
  const double sg = q.x < 0.0 ? -1.0 : 1.0;
  return make_double4(__dmul_rn(__ddiv_rn(q.x, nrm), sg), __dmul_rn(__ddiv_rn(q.y, nrm), sg),
                      __dmul_rn(__ddiv_rn(q.z, nrm), sg), __dmul_rn(__ddiv_rn(q.w, nrm), sg));
}

__device__ __forceinline__ double4 qmul_d(double4 a, double4 b) {
  // (w, x, y, z) in (.x, .y, .z, .w)
  const double w = __dsub_rn(__dsub_rn(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z)),
                             __dmul_rn(a.w, b.w));
  const double x = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)), __dmul_rn(a.z, b.w)),
                             __dmul_rn(a.w, b.z));
  const double y = __dadd_rn(__dadd_rn(__dsub_rn(__dmul_rn(a.x, b.z), __dmul_rn(a.y, b.w)), __dmul_rn(a.z, b.x)),
                             __dmul_rn(a.w, b.y));
  const double z = __dadd_rn(__dsub_rn(__dadd_rn(__dmul_rn(a.x, b.w), __dmul_rn(a.y, b.z)), __dmul_rn(a.z, b.y)),
                             __dmul_rn(a.w, b.x));
  return make_double4(w, x, y, z);
}

// Bunge angles (φ1, Φ, φ2), radians in [0, 2π) × [0, π] × [0, 2π), of a quaternion (rot.zig:151-173):
// standardized, then the host's formulas in FP64 with every product, sum and quotient rounded
// on its own in the host's order; atan2 is CUDA's (within 2 ulp of FP64), so after rounding to
// FP32 the angles are the host's but where an FP64 value lies within those ulps of an FP32
// rounding boundary.
__device__ void bunge_d(double4 q, float* e) {
  q = qstd_d(q);
  const double w = q.x, x = q.y, y = q.z, z = q.w;
  const double two_pi = 6.283185307179586;
  const double q03 = __dadd_rn(__dmul_rn(w, w), __dmul_rn(z, z));
  const double q12 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
  const double chi = sqrt(__dmul_rn(q03, q12));
  double e1, e2, e3;
  if (chi < 1e-14) {
    e1 = q12 <= q03 ? atan2(__dmul_rn(__dmul_rn(-2.0, w), z), __dsub_rn(__dmul_rn(w, w), __dmul_rn(z, z)))
                    : atan2(__dmul_rn(__dmul_rn(2.0, x), y), __dsub_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
    e2 = q12 <= q03 ? 0.0 : 3.141592653589793;
    e3 = 0.0;
  } else {
    e1 = atan2(__ddiv_rn(__dsub_rn(__dmul_rn(x, z), __dmul_rn(w, y)), chi),
               __ddiv_rn(__dsub_rn(__dmul_rn(-w, x), __dmul_rn(y, z)), chi));
    e2 = atan2(__dmul_rn(2.0, chi), __dsub_rn(q03, q12));
    e3 = atan2(__ddiv_rn(__dadd_rn(__dmul_rn(w, y), __dmul_rn(x, z)), chi),
               __ddiv_rn(__dsub_rn(__dmul_rn(y, z), __dmul_rn(w, x)), chi));
  }
  if (e1 < 0.0) e1 = __dadd_rn(e1, two_pi);
  if (e3 < 0.0) e3 = __dadd_rn(e3, two_pi);
  e[0] = __double2float_rn(e1); e[1] = __double2float_rn(e2); e[2] = __double2float_rn(e3);
}

// bunge (optional): each reduced orientation's Bunge angles, from its FP32-rounded quaternion as
// the host's landing would take it
__global__ void k_records_fz(const float* __restrict__ recs, int n, const double4* __restrict__ ops, int n_ops,
                             float* __restrict__ fz, float* __restrict__ bunge) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = recs + (size_t)i * 8;
  const double4 q = make_double4((double)r[0], (double)r[1], (double)r[2], (double)r[3]);
  double4 best = qstd_d(q);
  double bw = best.x;
  for (int k = 0; k < n_ops; ++k) {
    const double4 c = qstd_d(qmul_d(ops[k], q));
    if (c.x > bw + 1e-12) {
      best = c;
      bw = c.x;
    }
  }
  float* o = fz + (size_t)i * 4;
  o[0] = __double2float_rn(best.x); o[1] = __double2float_rn(best.y);
  o[2] = __double2float_rn(best.z); o[3] = __double2float_rn(best.w);
  if (bunge) bunge_d(make_double4((double)o[0], (double)o[1], (double)o[2], (double)o[3]), bunge + (size_t)i * 3);
}

static bool fill_frame(DetArgs& a, const zeb_frame_t* fr) {
  if (!fr || fr->h < 2 || fr->w < 2) return false;
  a.h = fr->h; a.w = fr->w;
  a.c0 = make_float3(fr->c0[0], fr->c0[1], fr->c0[2]);
  a.c1 = make_float3(fr->c1[0], fr->c1[1], fr->c1[2]);
  a.c2 = make_float3(fr->c2[0], fr->c2[1], fr->c2[2]);
  for (int k = 0; k < 3; ++k) a.mask[k] = fr->mask[k];
  return true;
}

// the compacted-pixel kernels while their list of masked pixels fits (12 800 of them: a 127 × 127
// pattern under the circular mask)
constexpr size_t DET_LIST_SMEM = 200 * 1024;

static size_t det_smem(DetArgs& a) {
  size_t hw = (size_t)a.h * a.w;
  a.pat_smem = hw * 4 <= 100 * 1024;
  a.sim_smem = a.pat_smem && hw * 8 <= 180 * 1024;
  return (a.pat_smem ? hw * 4 : 0) + (a.sim_smem ? hw * 4 : 0);
}

// ── the refinement over a precomputed pixel list ──
//
// The frame's masked pixels, in raster order, come as one list shared by every item (packed
// (row << 16) | col, zeb_mask_list); a block of 128 threads per item keeps only the pattern's
// values along the list in shared memory (4 bytes a pixel, 8 with NMI's simulated values), so
// that six items share an SM and one item's serial phase (the reduction and thread 0's step)
// overlaps the others' pixel passes (256 or 512 threads where those values pass 36 or 72 KB, so
// that the warps an SM holds stay about as many for a large detector's list).  Each pass recomputes the detector ray of every pixel (nine
// FMAs and a reciprocal square root) instead of keeping it; the sums per pixel are those of
// k_refine.

// the block size for a list whose pattern values and simulated values take `smem` bytes
inline int rl_threads(size_t smem) { return smem <= 36 * 1024 ? 128 : (smem <= 72 * 1024 ? 256 : 512); }

__device__ __forceinline__ float3 list_ray(const DetArgs& a, float3 t, uint32_t v) {
  return ray_dir(a, t, (int)(v >> 16), (int)(v & 0xffffu));
}

// the NMI over the list (detector.wgsl:744-832); sims (shared, npix floats) keeps the simulated
// values of the first pass for the histogram pass
__device__ float nmi_list(const DetArgs& a, const uint32_t* __restrict__ list, const float* pv, float* sims,
                          int npix, float3 t, float4 q, int nbins, uint32_t* hist, float* red) {
  float ext[4] = {3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f};
#pragma unroll 4
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const float e = pv[k];
    const float sv = master_at_pair(a.vpair, qrot(q, list_ray(a, t, __ldg(list + k))), a.side);
    sims[k] = sv;
    ext[0] = fminf(ext[0], e); ext[1] = fmaxf(ext[1], e);
    ext[2] = fminf(ext[2], sv); ext[3] = fmaxf(ext[3], sv);
  }
  for (int i = threadIdx.x; i < nbins * nbins; i += blockDim.x) hist[i] = 0u;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ext[0] = fminf(ext[0], __shfl_xor_sync(0xffffffffu, ext[0], o));
    ext[1] = fmaxf(ext[1], __shfl_xor_sync(0xffffffffu, ext[1], o));
    ext[2] = fminf(ext[2], __shfl_xor_sync(0xffffffffu, ext[2], o));
    ext[3] = fmaxf(ext[3], __shfl_xor_sync(0xffffffffu, ext[3], o));
  }
  if (lane == 0)
    for (int k = 0; k < 4; ++k) red[k * nw + wid] = ext[k];
  __syncthreads();
  float r[4] = {3.4e38f, -3.4e38f, 3.4e38f, -3.4e38f};
  for (int w = 0; w < nw; ++w) {
    r[0] = fminf(r[0], red[0 * nw + w]); r[1] = fmaxf(r[1], red[1 * nw + w]);
    r[2] = fminf(r[2], red[2 * nw + w]); r[3] = fmaxf(r[3], red[3 * nw + w]);
  }
  __syncthreads();
  const float ke = (float)nbins / fmaxf(r[1] - r[0], 1e-20f);
  const float ks = (float)nbins / fmaxf(r[3] - r[2], 1e-20f);
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const uint32_t be = min((uint32_t)((pv[k] - r[0]) * ke), (uint32_t)(nbins - 1));
    const uint32_t bs = min((uint32_t)((sims[k] - r[2]) * ks), (uint32_t)(nbins - 1));
    atomicAdd(&hist[be * nbins + bs], 1u);
  }
  __syncthreads();
  float acc[3] = {0.f, 0.f, 0.f};  // −Σ c log c (joint), −Σ (marginals), N
  for (int i = threadIdx.x; i < nbins * nbins; i += blockDim.x) {
    float c = (float)hist[i];
    acc[2] += c;
    if (c > 0.f) acc[0] -= c * logf(c);
  }
  if ((int)threadIdx.x < nbins) {
    float rs = 0.f, cs = 0.f;
    for (int k = 0; k < nbins; ++k) {
      rs += (float)hist[threadIdx.x * nbins + k];
      cs += (float)hist[k * nbins + threadIdx.x];
    }
    if (rs > 0.f) acc[1] -= rs * logf(rs);
    if (cs > 0.f) acc[1] -= cs * logf(cs);
  }
  block_sums<3>(acc, red);
  const float nn = fmaxf(acc[2], 1.f);
  const float h_joint = logf(nn) + acc[0] / nn;
  const float h_marg = 2.f * logf(nn) + acc[1] / nn;
  return h_marg > 1e-12f ? 2.f * (h_marg - h_joint) / h_marg : 0.f;
}

// QUAD: the lookups from the FP16 neighbourhood records (a.gpair holds zeb_master_quads' table)
// TH threads a pattern: 128 (six patterns an SM) while the list is small; a list whose shared
// memory leaves fewer blocks an SM takes 256 or 512, so that an SM keeps its warps
template <bool QUAD, int TH>
__global__ void __launch_bounds__(TH, TH == 128 ? 6 : (TH == 256 ? 3 : 1)) k_refine_list(DetArgs a, const uint32_t* __restrict__ list,
                                                                 int npix) {
  extern __shared__ float pv[];  // [npix] pattern values, then [npix] simulated values (NMI)
  __shared__ float red[20 * (TH / 32)];
  __shared__ uint32_t hist[32 * 32];
  __shared__ float4 sh_q;
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int NW = TH / 32;
  const float4 it = a.items[b];
  const float3 t = make_float3(it.x, it.y, it.z);
  const float* gpat = a.pats + (size_t)(int)it.w * a.h * a.w;
  for (int k = threadIdx.x; k < npix; k += TH) {
    const uint32_t v = __ldg(list + k);
    pv[k] = __ldg(gpat + (int)(v >> 16) * a.w + (int)(v & 0xffffu));
  }
  // refinement state (thread 0's registers): detector.wgsl:73-77
  const float* sd0 = a.seeds + (size_t)b * a.seed_stride;
  float4 q_best = make_float4(sd0[0], sd0[1], sd0[2], sd0[3]);
  float best = -2.f, mu = a.o.scale0, g_best[3] = {0.f, 0.f, 0.f}, h_best[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float last_good = 0.f, promised = 0.f, step_len = 0.f, accepted = 0.f;
  if (threadIdx.x == 0) sh_q = q_best;
  __syncthreads();

  for (int iter = 0; iter <= a.o.iters; ++iter) {
    const float4 q = sh_q;
    // the frame turned by q once a pass: q·(u/|u|) = (R u)/|R u| with R u = row·R c0 + col·R c1 + R t
    const float3 rc0 = qrot(q, a.c0), rc1 = qrot(q, a.c1), rt = qrot(q, t);
    float s[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) s[k] = 0.f;
#pragma unroll 4
    for (int k = threadIdx.x; k < npix; k += TH) {
      const uint32_t v = __ldg(list + k);
      const float row = (float)(int)(v >> 16), col = (float)(int)(v & 0xffffu);
      const float3 c = normalize3(make_float3(fmaf(rc0.x, row, fmaf(rc1.x, col, rt.x)),
                                              fmaf(rc0.y, row, fmaf(rc1.y, col, rt.y)),
                                              fmaf(rc0.z, row, fmaf(rc1.z, col, rt.z))));
      const float4 m = QUAD ? grad_at_quad(a.gpair, c, a.side) : grad_at_pair(a.gpair, c, a.side);
      const float3 d = cross3(c, make_float3(m.x, m.y, m.z));
      const float e = pv[k];
      s[1] += m.w; s[2] += m.w * m.w; s[3] += m.w * e;
      s[4] += d.x; s[5] += d.y; s[6] += d.z;
      s[7] += m.w * d.x; s[8] += m.w * d.y; s[9] += m.w * d.z;
      s[10] += e * d.x; s[11] += e * d.y; s[12] += e * d.z;
      s[13] += d.x * d.x; s[14] += d.y * d.y; s[15] += d.z * d.z;
      s[16] += d.x * d.y; s[17] += d.x * d.z; s[18] += d.y * d.z;
    }
    // each warp's sums (16 of them by a transposing reduction: each exchange halves the values a
    // lane holds, so lane pair i ends with sum 1 + i's total in 16 shuffles instead of 80), then
    // warp 0 alone adds the warps' (lane k: sum k) and takes the step
    {
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const bool up = (lane & 16) != 0;
        const float send = up ? s[1 + i] : s[9 + i];
        v[i] = (up ? s[9 + i] : s[1 + i]) + __shfl_xor_sync(0xffffffffu, send, 16);
      }
#pragma unroll
      for (int o = 8, n = 4; o >= 2; o >>= 1, n >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < n; ++i) {
          const float send = up ? v[i] : v[i + n];
          v[i] = (up ? v[i + n] : v[i]) + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
      const int idx = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
      if ((lane & 1) == 0) red[(1 + idx) * NW + wid] = v[0];
      const float w17 = warp_sum(s[17]), w18 = warp_sum(s[18]);
      if (lane == 0) {
        red[17 * NW + wid] = w17;
        red[18 * NW + wid] = w18;
      }
    }
    __syncthreads();
    if (wid == 0) {
      float tot = 0.f;
      if (lane >= 1 && lane < 19)
#pragma unroll
        for (int w = 0; w < NW; ++w) tot += red[lane * NW + w];
#pragma unroll
      for (int k = 1; k < 19; ++k) s[k] = __shfl_sync(0xffffffffu, tot, k);
      s[0] = (float)npix;
      if (lane == 0) {
        float4 qn = q_best;
        refine_step(a.o, iter, q, s, best, mu, g_best, h_best, last_good, promised, step_len, accepted, q_best, qn);
        sh_q = qn;
      }
    }
    __syncthreads();
  }
  const float4 qf = sh_q;
  const float v = nmi_list(a, list, pv, pv + npix, npix, t, qf, a.o.nmi_bins, hist, red);
  if (threadIdx.x == 0) {
    float* r = a.records + (size_t)b * 8;
    r[0] = qf.x; r[1] = qf.y; r[2] = qf.z; r[3] = qf.w;
    r[4] = best; r[5] = v; r[6] = last_good; r[7] = a.o.stamp;
  }
}

// the frame's masked pixels in raster order, (row << 16) | col: one block, a chunk of 256 pixels
// at a time (ballots and a running count keep the order)
__global__ void k_mask_list(DetArgs a, uint32_t* __restrict__ list) {
  __shared__ int wcnt[8];
  const int hw = a.h * a.w;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int out = 0;
  for (int base = 0; base < hw; base += 256) {
    const int i = base + threadIdx.x;
    const int row = i / a.w, col = i - row * a.w;
    const bool m = i < hw && in_mask(a, row, col);
    const unsigned bal = __ballot_sync(0xffffffffu, m);
    if (lane == 0) wcnt[wid] = __popc(bal);
    __syncthreads();
    int off = out, tot = 0;
    for (int w = 0; w < 8; ++w) {
      if (w < wid) off += wcnt[w];
      tot += wcnt[w];
    }
    if (m) list[off + __popc(bal & ((1u << lane) - 1u))] = ((uint32_t)row << 16) | (uint32_t)col;
    out += tot;
    __syncthreads();
  }
}

template <bool QUAD, int TH>
void rl_launch_th(const DetArgs& a, const uint32_t* list, int npix, size_t smem, cudaStream_t st) {
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_refine_list<QUAD, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_refine_list<QUAD, TH><<<a.n, TH, smem, st>>>(a, list, npix);
}

template <bool QUAD>
void rl_launch(const DetArgs& a, const uint32_t* list, int npix, size_t smem, cudaStream_t st) {
  const int th = rl_threads(smem);
  if (th == 128) rl_launch_th<QUAD, 128>(a, list, npix, smem, st);
  else if (th == 256) rl_launch_th<QUAD, 256>(a, list, npix, smem, st);
  else rl_launch_th<QUAD, 512>(a, list, npix, smem, st);
}

}  // namespace zeb

using namespace zeb;

extern "C" int zeb_refine(const float* pats, const float* items, const float* seeds, int seed_stride, int n,
                          const zeb_frame_t* fr, const float* vpair, const float* gpair, int side,
                          const zeb_refine_opts_t* o, float* records, void* stream) {
  ZEB_REQUIRE(pats && items && seeds && vpair && gpair && o && records, ZEB_EARG, "refine: null argument");
  ZEB_REQUIRE(((uintptr_t)gpair & 31) == 0 && ((uintptr_t)vpair & 7) == 0, ZEB_EARG, "refine: pair tables misaligned");
  ZEB_REQUIRE(seed_stride >= 4 && side >= 3 && o->iters >= 0 && o->iters <= 1000 && o->nmi_bins >= 2 &&
                  o->nmi_bins <= 32,
              ZEB_EARG, "refine: bad arguments");
  if (n <= 0) return ZEB_OK;
  DetArgs a{};
  ZEB_REQUIRE(fill_frame(a, fr), ZEB_EARG, "refine: bad frame");
  a.pats = pats; a.items = (const float4*)items; a.seeds = seeds; a.seed_stride = seed_stride; a.n = n;
  a.vpair = (const float2*)vpair; a.gpair = gpair; a.side = side; a.o = *o; a.records = records;
  const size_t list = (size_t)zeb_mask_count(fr) * sizeof(float4);
  if (list <= DET_LIST_SMEM) {
    cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)list);
    k_refine<<<n, 256, list, (cudaStream_t)stream>>>(a);
  } else {
    size_t smem = det_smem(a);
    cudaFuncSetAttribute(k_refine_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_refine_direct<<<n, 256, smem, (cudaStream_t)stream>>>(a);
  }
  return zeb_launch_check("refine");
}

extern "C" int zeb_mask_pixels(const zeb_frame_t* fr) {
  if (!fr || fr->h <= 0 || fr->w <= 0) return 0;
  return zeb_mask_count(fr);
}

extern "C" int zeb_mask_list(const zeb_frame_t* fr, uint32_t* list, void* stream) {
  ZEB_REQUIRE(fr && list, ZEB_EARG, "mask_list: null argument");
  ZEB_REQUIRE(fr->h > 0 && fr->w > 0 && fr->h < 65536 && fr->w < 65536, ZEB_EARG, "mask_list: bad frame size");
  DetArgs a{};
  ZEB_REQUIRE(fill_frame(a, fr), ZEB_EARG, "mask_list: bad frame");
  k_mask_list<<<1, 256, 0, (cudaStream_t)stream>>>(a, list);
  return zeb_launch_check("mask_list");
}

extern "C" int zeb_refine_list(const float* pats, const float* items, const float* seeds, int seed_stride, int n,
                               const zeb_frame_t* fr, const uint32_t* list, int npix, const float* vpair,
                               const float* gpair, int side, const zeb_refine_opts_t* o, float* records,
                               void* stream) {
  ZEB_REQUIRE(pats && items && seeds && list && vpair && gpair && o && records, ZEB_EARG,
              "refine_list: null argument");
  ZEB_REQUIRE(((uintptr_t)gpair & 31) == 0 && ((uintptr_t)vpair & 7) == 0, ZEB_EARG,
              "refine_list: pair tables misaligned");
  ZEB_REQUIRE(seed_stride >= 4 && side >= 3 && o->iters >= 0 && o->iters <= 1000 && o->nmi_bins >= 2 &&
                  o->nmi_bins <= 32,
              ZEB_EARG, "refine_list: bad arguments");
  ZEB_REQUIRE(fr && npix == zeb_mask_count(fr), ZEB_EARG, "refine_list: %d pixels listed, the frame masks %d", npix,
              fr ? zeb_mask_count(fr) : -1);
  const size_t smem = (size_t)npix * 2 * sizeof(float);
  ZEB_REQUIRE(npix >= 1 && smem <= DET_LIST_SMEM, ZEB_ESIZE, "refine_list: %d pixels (at most %zu)", npix,
              DET_LIST_SMEM / 8);
  if (n <= 0) return ZEB_OK;
  DetArgs a{};
  ZEB_REQUIRE(fill_frame(a, fr), ZEB_EARG, "refine_list: bad frame");
  a.pats = pats; a.items = (const float4*)items; a.seeds = seeds; a.seed_stride = seed_stride; a.n = n;
  a.vpair = (const float2*)vpair; a.gpair = gpair; a.side = side; a.o = *o; a.records = records;
  rl_launch<false>(a, list, npix, smem, (cudaStream_t)stream);
  return zeb_launch_check("refine_list");
}

extern "C" int zeb_refine_list_h(const float* pats, const float* items, const float* seeds, int seed_stride, int n,
                                 const zeb_frame_t* fr, const uint32_t* list, int npix, const float* vpair,
                                 const void* quads, int side, const zeb_refine_opts_t* o, float* records,
                                 void* stream) {
  ZEB_REQUIRE(pats && items && seeds && list && vpair && quads && o && records, ZEB_EARG,
              "refine_list_h: null argument");
  ZEB_REQUIRE(((uintptr_t)quads & 31) == 0 && ((uintptr_t)vpair & 7) == 0, ZEB_EARG,
              "refine_list_h: tables misaligned");
  ZEB_REQUIRE(seed_stride >= 4 && side >= 3 && o->iters >= 0 && o->iters <= 1000 && o->nmi_bins >= 2 &&
                  o->nmi_bins <= 32,
              ZEB_EARG, "refine_list_h: bad arguments");
  ZEB_REQUIRE(fr && npix == zeb_mask_count(fr), ZEB_EARG, "refine_list_h: %d pixels listed, the frame masks %d", npix,
              fr ? zeb_mask_count(fr) : -1);
  const size_t smem = (size_t)npix * 2 * sizeof(float);
  ZEB_REQUIRE(npix >= 1 && smem <= DET_LIST_SMEM, ZEB_ESIZE, "refine_list_h: %d pixels (at most %zu)", npix,
              DET_LIST_SMEM / 8);
  if (n <= 0) return ZEB_OK;
  DetArgs a{};
  ZEB_REQUIRE(fill_frame(a, fr), ZEB_EARG, "refine_list_h: bad frame");
  a.pats = pats; a.items = (const float4*)items; a.seeds = seeds; a.seed_stride = seed_stride; a.n = n;
  a.vpair = (const float2*)vpair; a.gpair = (const float*)quads; a.side = side; a.o = *o; a.records = records;
  rl_launch<true>(a, list, npix, smem, (cudaStream_t)stream);
  return zeb_launch_check("refine_list_h");
}

extern "C" int zeb_chance(const float* pats, const float* items, int n, int draws, const zeb_frame_t* fr,
                          const float* vpair, int side, int nmi_bins, float* out, void* stream) {
  ZEB_REQUIRE(pats && items && vpair && out && draws >= 1 && draws <= 65535 && nmi_bins >= 2 && nmi_bins <= 32,
              ZEB_EARG, "chance: bad arguments");
  ZEB_REQUIRE(((uintptr_t)vpair & 7) == 0, ZEB_EARG, "chance: value pairs misaligned");
  if (n <= 0) return ZEB_OK;
  DetArgs a{};
  ZEB_REQUIRE(fill_frame(a, fr), ZEB_EARG, "chance: bad frame");
  a.pats = pats; a.items = (const float4*)items; a.n = n; a.vpair = (const float2*)vpair; a.side = side;
  a.o.nmi_bins = nmi_bins; a.chance = out; a.draws = draws;
  dim3 g(n, draws);
  const size_t list = (size_t)zeb_mask_count(fr) * sizeof(float4);
  if (list <= DET_LIST_SMEM) {
    cudaFuncSetAttribute(k_chance, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)list);
    k_chance<<<g, 256, list, (cudaStream_t)stream>>>(a);
  } else {
    size_t smem = det_smem(a);
    cudaFuncSetAttribute(k_chance_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_chance_direct<<<g, 256, smem, (cudaStream_t)stream>>>(a);
  }
  return zeb_launch_check("chance");
}

extern "C" int zeb_project(const float* master, int side, const float* poses, int n, const zeb_frame_t* fr,
                           float* sims, void* stream) {
  ZEB_REQUIRE(master && poses && sims && side >= 3, ZEB_EARG, "project: bad arguments");
  if (n <= 0) return ZEB_OK;
  DetArgs a{};
  ZEB_REQUIRE(fill_frame(a, fr), ZEB_EARG, "project: bad frame");
  a.n = n; a.master = master; a.side = side;
  long long total = (long long)n * a.h * a.w;
  k_project<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a, poses, sims);
  return zeb_launch_check("project");
}

extern "C" int zeb_records_fz(const float* records, int n, const double* ops, int n_ops, float* fz, void* stream) {
  return zeb_records_fz_bunge(records, n, ops, n_ops, fz, nullptr, stream);
}

extern "C" int zeb_records_fz_bunge(const float* records, int n, const double* ops, int n_ops, float* fz, float* bunge,
                                    void* stream) {
  ZEB_REQUIRE(records && ops && fz && n_ops >= 1 && n_ops <= 48, ZEB_EARG, "records_fz: bad arguments");
  if (n <= 0) return ZEB_OK;
  k_records_fz<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(records, n, (const double4*)ops, n_ops, fz, bunge);
  return zeb_launch_check("records_fz");
}
