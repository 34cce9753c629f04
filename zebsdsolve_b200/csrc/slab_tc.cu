// (b, second stage, the BF16 form) The correlation volume's transform along a on the tcgen05
// tensor cores, over the spectrum kept in FP16.
//
// U (transformed along b and c by the spectrum GEMM) arrives as s·U in FP16, laid out
// [item tile][(j, c)][m'][re|im][128 items] (k_spectrum_tc<true>).  For one (j, c) the real transform
// along a (so3.wgsl:279-315, 396-593),
//
//   C(a) = Re V[0] + 2 Re Σ_{m'>0} V[m'] e^{−2πi m' a/n} = Σ_κ V_κ F[a][κ],  κ = 2m' + (re|im),
//   F[a][2m'] = f_m' cos(2π m' a/n),  F[a][2m'+1] = f_m' sin(2π m' a/n),  f_0 = 1, f_m'>0 = 2,
//
// is then one GEMM per (j, c) over a tile of 128 items: D[item][a] = Σ_κ A[item][κ] F[a][κ] with
// M = 128 items, N = n, K = 2L, FP16 operands and FP32 accumulation in tensor memory.  A is the
// tile of U as it lies in memory (items contiguous: an MN-major operand, brought in by two 5-D
// tensor loads with the 128-byte swizzle); F, the same for every tile, is built once per CTA in
// shared memory (K-major, 128-byte swizzle).  The epilogue scales each value by the shared
// denominator volume, rden[j][c][a]/s, and keeps each item's largest with its volume index
// (j·nc + c)·n + a (first index of equal values) over the nc tiles of j: the candidate of slab
// (item, j), as zeb_correlate_peaks's slab kernels give it.  U never returns to HBM once read.
//
// k_peak_finish (slab.cu's, with an FP16 reader) then reduces the candidates and fits the vertex
// from direct sums over m' at the peak and its six neighbours.
//
// One persistent CTA per SM: warp 0 issues the tensor loads (a ring of ST_STAGES tiles) and the
// bulk copies of each tile's row of rden (a ring of ST_RSLOTS), warp 1 the MMAs into ST_ACC
// accumulators of n columns, warps 2-9 drain them (two warps per TMEM lane quadrant, each half of
// the n columns).  Every wait is bounded: on a timeout the CTA records the
// failure, waits (bounded) for what it issued, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "abi_util.cuh"
#include "tc_util.cuh"

namespace zeb {

constexpr int ST_BM = 128;                  // items per tile (MMA M)
constexpr int ST_STAGES = 4;                // tiles of U in flight
constexpr int ST_EPI = 8;                   // epilogue warps
constexpr int ST_THREADS = 64 + 32 * ST_EPI;
constexpr int ST_HALF_BYTES = 16384;        // one 64-item half of a tile: 2L rows of 128 B (L <= 64)

struct SlabTcArgs {
  int n_items, L, n, nb, nc, ptiles;
  float rscale;       // 1/s: rden × rscale turns s·C into the normalized score
  const float* rden;  // [nb][nc][n], shared by every item
  float2* cand;       // [item][nb]: (value, bits of the volume index)
  int* status;
  long long limit;
  long long stall;  // > 0: the failure test (the MMA thread first waits on `never`)
};

constexpr int ST_ACC = 4;    // accumulators in tensor memory (4 × 128 columns)
constexpr int ST_RSLOTS = 8;  // rows of rden staged ahead of the epilogue

struct SlabTcShared {
  uint8_t f[2][16384];                        // F: n rows × 2L FP16, K-major, in 64-wide K blocks
  uint8_t a[ST_STAGES][2][ST_HALF_BYTES];     // tiles of U: [half][κ][64 items]
  float rden[ST_RSLOTS][128];                 // each tile's row rden[j][c][0 … n)
  float bestv[2][ST_BM];                      // the second half's best, handed to the first
  uint32_t besti[2][ST_BM];
  uint64_t full[ST_STAGES], empty[ST_STAGES], acc_full[ST_ACC], acc_empty[ST_ACC], rfull[ST_RSLOTS],
      rempty[ST_RSLOTS], mma_done, never;
  uint32_t tmem;
};

// the n × 2L transform matrix in FP16, K-major with the 128-byte swizzle; the angle's fraction of
// a turn is exact ((m'·a) mod n over n), its sine and cosine from sincospif
__device__ void build_dft(uint8_t (*f)[16384], int n, int L) {
  const int K = 2 * L;
  for (int e = threadIdx.x; e < n * K; e += blockDim.x) {
    const int row = e / K, k = e - row * K;
    const int mp = k >> 1;
    const float frac = 2.f * (float)((mp * row) & (n - 1)) / (float)n;  // angle / π
    float sv, cv;
    sincospif(frac, &sv, &cv);
    const float fac = mp == 0 ? 1.f : 2.f;
    const float v = fac * ((k & 1) ? sv : cv);
    *(__half*)(f[k >> 6] + sw128(row, k & 63)) = __float2half_rn(v);
  }
}

__global__ void __launch_bounds__(ST_THREADS, 1) k_slab_tc(SlabTcArgs a, const __grid_constant__ CUtensorMap umap) {
  extern __shared__ __align__(1024) uint8_t st_smem_raw[];
  SlabTcShared& s = *reinterpret_cast<SlabTcShared*>((void*)(((uintptr_t)st_smem_raw + 1023) & ~(uintptr_t)1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = a.n, nc = a.nc, nb = a.nb;
  const long long items = (long long)a.ptiles * nb;  // work items (ptile, j), j-major
  // this CTA's items: blockIdx.x, + gridDim.x, …; each is nc tiles (c = 0 … nc − 1)
  const long long my_items = items > blockIdx.x ? (items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long long total = my_items * nc;
  if (threadIdx.x == 0) {
    for (int i = 0; i < ST_STAGES; ++i) {
      mbar_init(&s.full[i], 1);
      mbar_init(&s.empty[i], 1);
    }
    for (int i = 0; i < ST_ACC; ++i) {
      mbar_init(&s.acc_full[i], 1);
      mbar_init(&s.acc_empty[i], ST_EPI);
    }
    for (int i = 0; i < ST_RSLOTS; ++i) {
      mbar_init(&s.rfull[i], 1);
      mbar_init(&s.rempty[i], ST_EPI);
    }
    mbar_init(&s.mma_done, 1);
    mbar_init(&s.never, 1);  // nothing arrives: the failure test's wait
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  build_dft(s.f, n, a.L);
  fence_proxy_async();  // F, written by these threads, is read by the tensor cores (async proxy)
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem)),
                 "r"(128 * ST_ACC));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s.tmem;
  const long long lim = a.limit;
  const uint32_t tile_bytes = 2u * (uint32_t)(2 * a.L) * 128u;

  if (warp == 0) {
    if (lane == 0) {
      long long it = 0, rit = 0;  // tiles of U and rows of rden issued
      bool ok = true;
      for (long long mi = 0; mi < my_items && ok; ++mi) {
        const long long item = blockIdx.x + mi * gridDim.x;
        const int j = (int)(item / a.ptiles), pt = (int)(item - (long long)j * a.ptiles);
        for (int c = 0; c < nc; ++c, ++it) {
          const int st = (int)(it % ST_STAGES);
          if (!mbar_wait(&s.empty[st], (uint32_t)((it / ST_STAGES) & 1) ^ 1u, lim)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&s.full[st], tile_bytes);
          // the 2L × 256 contiguous bytes of (j, c) and this tile, as two halves of 64 items
          tma_load_5d(&umap, s.a[st][0], &s.full[st], 0, 0, 0, j * nc + c, pt);
          tma_load_5d(&umap, s.a[st][1], &s.full[st], 64, 0, 0, j * nc + c, pt);
          // and the tile's row of rden, for the epilogue
          const int rs = (int)(it % ST_RSLOTS);
          if (!mbar_wait(&s.rempty[rs], (uint32_t)((it / ST_RSLOTS) & 1) ^ 1u, lim)) {
            ok = false;
            ++it;  // its tile of U is in flight
            break;
          }
          mbar_expect_tx(&s.rfull[rs], (uint32_t)n * 4u);
          bulk_g2s(s.rden[rs], a.rden + (size_t)(j * nc + c) * n, (uint32_t)n * 4u, &s.rfull[rs]);
          rit = it + 1;
        }
      }
      if (!ok) atomicOr(a.status, 1);
      // the loads still in flight land before the CTA may leave (bounded waits on their phases; a
      // phase already consumed reads as complete)
      for (long long i = (it > ST_STAGES ? it - ST_STAGES : 0); i < it; ++i)
        mbar_wait(&s.full[i % ST_STAGES], (uint32_t)((i / ST_STAGES) & 1), kDrainNs);
      for (long long i = (rit > ST_RSLOTS ? rit - ST_RSLOTS : 0); i < rit; ++i)
        mbar_wait(&s.rfull[i % ST_RSLOTS], (uint32_t)((i / ST_RSLOTS) & 1), kDrainNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // kind::f16: F32 accumulate, FP16 A (MN-major) and B (K-major), M = 128, N = n
      const uint32_t idesc = (1u << 4) | (0u << 7) | (0u << 10) | (1u << 15) | ((uint32_t)(n >> 3) << 17) |
                             ((uint32_t)(ST_BM >> 4) << 24);
      const int ksteps = (2 * a.L) / 16;
      const uint32_t fbase = smem_addr(s.f[0]);
      bool ok = true;
      if (a.stall > 0 && !mbar_wait(&s.never, 0, a.stall)) ok = false;  // the failure test
      long long t = 0;
      for (; t < total && ok; ++t) {
        const int acc = (int)(t % ST_ACC);
        const int st = (int)(t % ST_STAGES);
        ok = mbar_wait(&s.acc_empty[acc], (uint32_t)((t / ST_ACC) & 1) ^ 1u, lim);
        if (ok) ok = mbar_wait(&s.full[st], (uint32_t)((t / ST_STAGES) & 1), lim);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * 128);
        const uint32_t abase = smem_addr(s.a[st][0]);
        for (int ks = 0; ks < ksteps; ++ks) {
          // A: 16 K rows (2 groups of 8, 1024 B apart) from row 16·ks; the item halves 16 KB apart
          const uint64_t da = umma_desc_mn(abase + (uint32_t)ks * 2048u, ST_HALF_BYTES, 1024);
          const uint64_t db = umma_desc(fbase + (uint32_t)(ks >> 2) * 16384u + (uint32_t)(ks & 3) * 32u);
          umma_f16(d, da, db, idesc, ks != 0);
        }
        umma_commit(&s.empty[st]);   // the stage is free once these MMAs have read it
        umma_commit(&s.acc_full[acc]);
      }
      if (!ok) atomicOr(a.status, 2);
      umma_commit(&s.mma_done);  // every MMA issued has finished before TMEM may be freed
      if (!mbar_wait(&s.mma_done, 0, kDrainNs)) atomicOr(a.status, 8);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32·(w mod 4) …; warps w and w + 4 take the two halves of
    // the n columns. Thread = one item (row of the tile) × half the a values of each tile. Each
    // warp follows the accumulators on its own (the MMAs run up to ST_ACC tiles ahead); the eight
    // meet once per item, where the halves' bests merge.
    const int ew = warp & 3;
    const int row = ew * 32 + lane;
    const int half = (warp - 2) >> 2;
    const int hn = n >> 1;  // columns per half: 16, 32 or 64
    const uint32_t lanes = (uint32_t)(ew * 32) << 16;
    const float rsc = a.rscale;
    float bv = -3.4e38f;
    uint32_t bi = 0xffffffffu;
    long long t = 0;
    bool ok = true;
    for (long long mi = 0; mi < my_items; ++mi) {
      const long long item = blockIdx.x + mi * gridDim.x;
      const int j = (int)(item / a.ptiles), pt = (int)(item - (long long)j * a.ptiles);
      for (int c = 0; c < nc && ok; ++c, ++t) {
        const int acc = (int)(t % ST_ACC);
        const int rs = (int)(t % ST_RSLOTS);
        // lane 0 waits (try_wait suspends it in hardware until the phase completes); the warp follows
        int got = 1;
        if (lane == 0)
          got = mbar_wait(&s.acc_full[acc], (uint32_t)((t / ST_ACC) & 1), lim) &&
                mbar_wait(&s.rfull[rs], (uint32_t)((t / ST_RSLOTS) & 1), lim);
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
          if (lane == 0) atomicOr(a.status, 4);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t c0 = tmem + lanes + (uint32_t)(acc * 128 + half * hn);
        uint32_t v[64];
        TMEM_LD32(c0, v);
        if (hn > 32) TMEM_LD32(c0 + 32, (v + 32));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.acc_empty[acc]);  // the MMAs of tile t + ST_ACC may start
        // the values s·C·rden (s a power of two: the order, and every product's rounding, are those
        // of C·rden; the candidate is scaled by 1/s once, exactly); their largest by a tree
        const float* rrow = s.rden[rs] + half * hn;
        float x[64];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          if (4 * q < hn) {
            const float4 r = *reinterpret_cast<const float4*>(rrow + 4 * q);
            x[4 * q + 0] = __uint_as_float(v[4 * q + 0]) * r.x;
            x[4 * q + 1] = __uint_as_float(v[4 * q + 1]) * r.y;
            x[4 * q + 2] = __uint_as_float(v[4 * q + 2]) * r.z;
            x[4 * q + 3] = __uint_as_float(v[4 * q + 3]) * r.w;
          } else {
            x[4 * q + 0] = x[4 * q + 1] = x[4 * q + 2] = x[4 * q + 3] = -3.4e38f;
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.rempty[rs]);  // this warp is done with the staged row
        float m4[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          float m = x[k];
#pragma unroll
          for (int q = 1; q < 16; ++q) m = fmaxf(m, x[4 * q + k]);
          m4[k] = m;
        }
        const float m = fmaxf(fmaxf(m4[0], m4[1]), fmaxf(m4[2], m4[3]));
        if (m > bv) {  // a new best: its first position in the tile (indices grow along the tile)
          int kk = 0;
#pragma unroll
          for (int k = 63; k >= 0; --k)
            if (x[k] == m) kk = k;
          bv = m;
          bi = (uint32_t)(j * nc + c) * (uint32_t)n + (uint32_t)(half * hn + kk);
        }
      }
      // the item's end: the eight warps agree on the outcome, and the second half's best joins the
      // first's (lower index on equal values)
      const int par = (int)(mi & 1);
      if (half == 1) {
        s.bestv[par][row] = bv;
        s.besti[par][row] = bi;
      }
      ok = bar_and(2, 32 * ST_EPI, ok);
      if (!ok) break;
      if (half == 0) {
        const float ov = s.bestv[par][row];
        const uint32_t oi = s.besti[par][row];
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        const int p = pt * ST_BM + row;
        if (p < a.n_items) a.cand[(size_t)p * nb + j] = make_float2(bv * rsc, __uint_as_float(bi));
      }
      bv = -3.4e38f;
      bi = 0xffffffffu;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128 * ST_ACC));
}

}  // namespace zeb

using namespace zeb;

// U16 as the 5-D tensor (items within the tile, re|im, order, (j, c), tile); boxes of 64 items × re|im
// × every order of one (j, c) and one tile, landing as [order][re|im][64 items] with the 128-byte
// swizzle
static bool st_u16_map(CUtensorMap* m, const void* U16, const zeb_so3_dims_t* d, int n_items) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  if (!fn) return false;
  const cuuint64_t ptiles = (cuuint64_t)((n_items + ST_BM - 1) / ST_BM);
  const cuuint64_t L = (cuuint64_t)d->L, jc = (cuuint64_t)d->nb * d->nc;
  cuuint64_t dims[5] = {ST_BM, 2, L, jc, ptiles};
  cuuint64_t strides[4] = {ST_BM * 2, ST_BM * 4, ST_BM * 4 * L, ST_BM * 4 * L * jc};
  cuuint32_t box[5] = {64, 2, (cuuint32_t)d->L, 1, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 5, const_cast<void*>(U16), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// dims the tensor-core transform along a takes: n = 2L a power of two, 32 ≤ n ≤ 128 (one tile of U
// and the transform matrix fit the stages), nc a power of two
static bool st_dims_ok(const zeb_so3_dims_t* d) {
  return d && d->L >= 16 && d->L <= 64 && d->n == 2 * d->L && (d->n & (d->n - 1)) == 0 && d->nb == d->n / 2 + 1 &&
         d->fold >= 1 && d->nc == d->n / d->fold && (d->nc & (d->nc - 1)) == 0 &&
         d->n_pairs == d->L * (d->L + 1) / 2 && 2 * d->nb * d->nc >= 128;
}

extern "C" int zeb_peak_finish_h(const void* U16, int n_items, const zeb_so3_dims_t* d, float scale, const float* rden,
                                 const float2* cand, float* peaks, void* stream);

extern "C" int zeb_correlate_peaks_h(const void* U16, int n_items, const zeb_so3_dims_t* d, float scale,
                                     const float* rden, float* peaks, void* scratch, int* status, void* stream) {
  ZEB_REQUIRE(U16 && rden && peaks && scratch && status, ZEB_EARG, "correlate_peaks_h: null argument");
  ZEB_REQUIRE(st_dims_ok(d), ZEB_EARG, "correlate_peaks_h: unsupported dims (L=%d)", d ? d->L : -1);
  ZEB_REQUIRE(scale > 0.f && scale < 1e30f, ZEB_EARG, "correlate_peaks_h: scale %g", (double)scale);
  ZEB_REQUIRE(((uintptr_t)U16 & 127) == 0 && ((uintptr_t)rden & 15) == 0, ZEB_EARG,
              "correlate_peaks_h: U16 must be 128-byte and rden 16-byte aligned");
  if (n_items <= 0) return ZEB_OK;
  CUtensorMap umap;
  ZEB_REQUIRE(st_u16_map(&umap, U16, d, n_items), ZEB_ECUDA, "correlate_peaks_h: tensor map for U16 refused");
  SlabTcArgs a{};
  a.n_items = n_items;
  a.L = d->L; a.n = d->n; a.nb = d->nb; a.nc = d->nc;
  a.ptiles = (n_items + ST_BM - 1) / ST_BM;
  a.rscale = 1.f / scale;
  a.rden = rden;
  a.cand = (float2*)scratch;
  a.status = status;
  a.stall = test_stall_ns();
  a.limit = a.stall > 0 ? a.stall : kWaitNs;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = sizeof(SlabTcShared) + 1024;
  cudaFuncSetAttribute(k_slab_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long items = (long long)a.ptiles * d->nb;
  const int grid = (int)std::min<long long>(items, sms);
  k_slab_tc<<<grid, ST_THREADS, smem, st>>>(a, umap);
  int rc = zeb_launch_check("correlate slab (tensor cores)");
  if (rc) return rc;
  return zeb_peak_finish_h(U16, n_items, d, scale, rden, (const float2*)scratch, peaks, stream);
}
