// (b, first stage) The spectrum of each item along b, in plain FP32 on the CUDA cores:
//
//   U[b][j][m'][iq] = Σ_{l ≥ m'} conj(g_b[l, m']) · Y[pair(m', l)][j·nc + iq]
//
// a complex GEMM per order m' (M = items, N = nb·nc columns, K = L − m'), where Y is the master's
// correlation table: the Wigner-d contraction with the master's weights and the transform along b
// folded in (zeb_correlation_table). This is the reference's `spectrum` kernel (so3.wgsl:147-277:
// l-sums of W·conj(g)·d per k, then an FFT along k) written as one GEMM against a table that
// already holds both.
//
// Tile: 64 items × 64 columns per block, K in steps of 8, each thread 4 × 4 complex outputs.
#include "abi_util.cuh"

namespace zeb {

#define SP_BM 64
#define SP_BN 64
#define SP_BK 8

__global__ void __launch_bounds__(256) k_spectrum_f32(const float2* __restrict__ alm, int n_items,
                                                        zeb_so3_dims_t d, const float2* __restrict__ Y,
                                                        float2* __restrict__ U) {
  __shared__ float2 As[SP_BK][SP_BM];
  __shared__ float2 Bs[SP_BK][SP_BN];
  const int L = d.L, nc = d.nc, nb = d.nb;
  const int N = nb * nc;
  const int mp = blockIdx.z;
  const int n0 = blockIdx.x * SP_BN;
  const int b0 = blockIdx.y * SP_BM;
  const int K = L - mp;
  const int p0 = mp * L - (mp * (mp - 1)) / 2;  // pair(m', m')
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);

  for (int k0 = 0; k0 < K; k0 += SP_BK) {
    // A: conj(g[b][p0 + k]) for 64 items × 8 k (2 per thread)
    for (int e = threadIdx.x; e < SP_BM * SP_BK; e += 256) {
      int i = e / SP_BK, kk = e - i * SP_BK;
      int b = b0 + i, k = k0 + kk;
      float2 v = make_float2(0.f, 0.f);
      if (b < n_items && k < K) {
        v = __ldg(alm + (size_t)b * d.n_pairs + p0 + k);
        v.y = -v.y;
      }
      As[kk][i] = v;
    }
    // B: Y rows p0 + k, columns n0 …
    for (int e = threadIdx.x; e < SP_BK * SP_BN; e += 256) {
      int kk = e / SP_BN, c = e - kk * SP_BN;
      int k = k0 + kk, n = n0 + c;
      float2 v = make_float2(0.f, 0.f);
      if (k < K && n < N) v = __ldg(Y + (size_t)(p0 + k) * N + n);
      Bs[kk][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < SP_BK; ++kk) {
      float2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fmaf(av[i].x, bv[j].x, fmaf(-av[i].y, bv[j].y, acc[i][j].x));
          acc[i][j].y = fmaf(av[i].x, bv[j].y, fmaf(av[i].y, bv[j].x, acc[i][j].y));
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int b = b0 + ty + 16 * i;
    if (b >= n_items) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      int jj = n / nc, iq = n - jj * nc;
      U[(((size_t)b * nb + jj) * L + mp) * nc + iq] = acc[i][j];
    }
  }
}

}  // namespace zeb

using namespace zeb;

static bool so3_dims_ok(const zeb_so3_dims_t* d) {
  return d && d->L >= 2 && d->L <= 256 && d->n >= 2 * d->L - 1 && d->nb == d->n / 2 + 1 && d->fold >= 1 &&
         d->nc == d->n / d->fold && d->mu_max == (d->L - 1) / d->fold && d->n_pairs == d->L * (d->L + 1) / 2;
}

extern "C" size_t zeb_spectrum_bytes(const zeb_so3_dims_t* d, int n_items) {
  if (!so3_dims_ok(d) || n_items <= 0) return 0;
  return (size_t)n_items * d->nb * d->L * d->nc * sizeof(float2);
}

extern "C" int zeb_spectrum_f32(const float* alm, int n_items, const zeb_so3_dims_t* d, const float* Y, float* U,
                                void* stream) {
  ZEB_REQUIRE(alm && Y && U, ZEB_EARG, "spectrum_f32: null argument");
  ZEB_REQUIRE(so3_dims_ok(d), ZEB_EARG, "spectrum_f32: inconsistent dims");
  if (n_items <= 0) return ZEB_OK;
  const int N = d->nb * d->nc;
  dim3 g((N + SP_BN - 1) / SP_BN, (n_items + SP_BM - 1) / SP_BM, d->L);
  ZEB_REQUIRE(g.y <= 65535, ZEB_ESIZE, "spectrum_f32: %d items in one call", n_items);
  k_spectrum_f32<<<g, 256, 0, (cudaStream_t)stream>>>((const float2*)alm, n_items, *d, (const float2*)Y, (float2*)U);
  return zeb_launch_check("spectrum_f32");
}
