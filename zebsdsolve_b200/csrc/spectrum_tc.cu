// (b, first stage) The spectrum GEMM on the tcgen05 tensor cores: BF16 operands, FP32
// accumulation in tensor memory (TMEM).
//
//   U[b][j][m'][iq] = Σ_l conj(g_b[l,m']) · Y[pair(m',l)][j·nc + iq]
//
// as one real GEMM per order m':  D[ν][b] = Σ_κ A_m'[ν][κ] · B_m'[b][κ], with ν = 2(j·nc+iq) + (re|im)
// (the rows, M) and κ = 2(l−m') + (re|im) (the reduction, K):
//   A[2n][2l'] = Re Y,  A[2n][2l'+1] = Im Y,  A[2n+1][2l'] = Im Y,  A[2n+1][2l'+1] = −Re Y
//   B[b][2l'] = Re g,   B[b][2l'+1] = Im g
// (conj(g)·Y = (gr·Yr + gi·Yi) + i(gr·Yi − gi·Yr)).
//
// Accuracy: every operand is split x = hi + lo into two BF16 values; for the orders l ≤ split
// (the low orders, which carry most of the energy of a pattern and of a master) the product takes
// hi·hi + hi·lo + lo·hi, as two more K segments of the same GEMM (K' = K + 2·K_split); above,
// hi·hi alone (2^-9 relative per operand).  split = 16 keeps the low orders near FP32; split =
// L − 1 makes the whole product so (relative error ~2^-16).  A per-order scale would only shift
// exponents, of which BF16 has as many as FP32, so none is applied.
//
// Operands live in HBM already in the shared-memory layout the MMA reads (K-major, 128-byte
// rows, the 16-byte chunks of row r XOR-swizzled by r mod 8, 8-row groups 1024 B apart), in
// blocks of 64 K-elements: a block is one bulk async copy. The master's A is built once per phase
// (k_pack_master, FP64 → BF16 hi/lo); the patterns' B per batch (k_pack_patterns).
//
// k_spectrum_tc: one CTA per (pattern tile of 128, order m'), 6 warps: warp 0 issues the bulk
// copies (B once, then A block by block through a ring of stages: TC_STAGES for the FP32 U,
// TCH_STAGES for the FP16 one), warp 1 allocates TMEM and one of its threads issues the MMAs
// (M = 128 rows of ν, N = 128 patterns, K = 16 a step) into two accumulators of 128 columns, warps
// 2-5 drain an accumulator (tcgen05.ld) while the next one fills: the FP32 U 32 patterns at a time
// through shared memory into a tensor store, the FP16 U a whole tile at once (scattered 128-byte
// stores from four warps cap an SM near 13 GB/s; the tensor store does not). Every wait is
// bounded: on a timeout the CTA records the failure, drains what it issued, frees its TMEM and
// returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>

#include "abi_util.cuh"
#include "tc_util.cuh"

namespace zeb {

constexpr int TC_BN = 128;            // patterns per tile (MMA N)
constexpr int TC_BM = 128;            // rows ν per tile (MMA M)
constexpr int TC_KB = 64;             // K-elements per block (one 128-byte swizzled row)
constexpr int TC_A_BLOCK = TC_BM * 128;  // bytes of one A block (16 KB)
constexpr int TC_B_BLOCK = TC_BN * 128;  // bytes of one B block (16 KB)
constexpr int TC_MAX_KB = 6;          // K' ≤ 384: B stays resident (96 KB)
constexpr int TC_STAGES = 5;          // A ring: 5 blocks of 16 KB
constexpr int TC_THREADS = 192;

// K' of order m': 2(L − m') + 4·(number of l in [m', split])
__host__ __device__ inline int tc_k0(int L, int mp) { return 2 * (L - mp); }
__host__ __device__ inline int tc_k1(int L, int mp, int split) {
  int hi = split < L - 1 ? split : L - 1;
  return mp <= hi ? 2 * (hi - mp + 1) : 0;
}
__host__ __device__ inline int tc_kblocks(int L, int mp, int split) {
  int k = tc_k0(L, mp) + 2 * tc_k1(L, mp, split);
  return (k + TC_KB - 1) / TC_KB;
}

// (segment, l, re|im) of K-element κ of order m' (segment 0: hi·hi over all l; 1: hi(A)·lo(B) for
// l ≤ split; 2: lo(A)·hi(B) for l ≤ split; 3: padding)
struct KSlot {
  int seg, l, part;
};
__device__ __forceinline__ KSlot k_slot(int L, int mp, int split, int k) {
  const int k0 = tc_k0(L, mp), k1 = tc_k1(L, mp, split);
  KSlot s;
  if (k < k0) {
    s.seg = 0; s.l = mp + (k >> 1); s.part = k & 1;
  } else if (k < k0 + k1) {
    s.seg = 1; s.l = mp + ((k - k0) >> 1); s.part = (k - k0) & 1;
  } else if (k < k0 + 2 * k1) {
    s.seg = 2; s.l = mp + ((k - k0 - k1) >> 1); s.part = (k - k0 - k1) & 1;
  } else {
    s.seg = 3; s.l = 0; s.part = 0;
  }
  return s;
}

struct TcLayout {
  int L, nb, nc, rows, mtiles, ptiles, split;
};

// byte offset of order m''s blocks: Σ over the lower orders of tiles · K-blocks · block bytes
__host__ __device__ inline long long tc_offset(int L, int split, int mp, int tiles, int block_bytes) {
  long long o = 0;
  for (int q = 0; q < mp; ++q) o += (long long)tiles * tc_kblocks(L, q, split) * block_bytes;
  return o;
}

// A_m'[ν][κ] from Y (FP64 complex [pair][nb·nc]), one thread per 16-byte chunk of a block row.
__global__ void k_pack_master(const double2* __restrict__ Y, TcLayout t, int mp, long long a_off,
                              uint8_t* __restrict__ A) {
  const int kb = tc_kblocks(t.L, mp, t.split);
  const long long chunks = (long long)t.mtiles * kb * TC_BM * 8;
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= chunks) return;
  const int c16 = (int)(e & 7);
  const int row = (int)((e >> 3) % TC_BM);
  const long long blk = (e >> 3) / TC_BM;  // mtile·kb + kblock
  const int kblock = (int)(blk % kb), mtile = (int)(blk / kb);
  const int nu = mtile * TC_BM + row;
  const int ncols = t.nb * t.nc;
  const int p0 = mp * t.L - (mp * (mp - 1)) / 2;
  uint16_t v[8];
  for (int i = 0; i < 8; ++i) {
    const int k = kblock * TC_KB + c16 * 8 + i;
    KSlot s = k_slot(t.L, mp, t.split, k);
    float out = 0.f;
    if (s.seg < 3 && nu < 2 * ncols) {
      const double2 y = Y[(size_t)(p0 + s.l - mp) * ncols + (nu >> 1)];
      // rows re: (Yr, Yi); rows im: (Yi, −Yr)
      double val = (nu & 1) == 0 ? (s.part == 0 ? y.x : y.y) : (s.part == 0 ? y.y : -y.x);
      float hi = bf16_value(bf16_bits((float)val));
      out = s.seg == 2 ? (float)(val - (double)hi) : (float)val;
    }
    v[i] = bf16_bits(out);
  }
  uint8_t* blkp = A + a_off + (size_t)blk * TC_A_BLOCK;
  uint4 w;
  w.x = v[0] | ((uint32_t)v[1] << 16);
  w.y = v[2] | ((uint32_t)v[3] << 16);
  w.z = v[4] | ((uint32_t)v[5] << 16);
  w.w = v[6] | ((uint32_t)v[7] << 16);
  *(uint4*)(blkp + sw128(row, c16 * 8)) = w;
}

// B_m'[b][κ] from the coefficients (complex f32 [b][pair]), every order, one thread per chunk.
__global__ void k_pack_patterns(const float2* __restrict__ alm, int n_items, int n_pairs, TcLayout t,
                                uint8_t* __restrict__ B) {
  const int mp = blockIdx.y;
  __shared__ long long b_off;
  if (threadIdx.x == 0) b_off = tc_offset(t.L, t.split, mp, t.ptiles, TC_B_BLOCK);
  __syncthreads();
  const int kb = tc_kblocks(t.L, mp, t.split);
  const long long chunks = (long long)t.ptiles * kb * TC_BN * 8;
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= chunks) return;
  const int c16 = (int)(e & 7);
  const int row = (int)((e >> 3) % TC_BN);
  const long long blk = (e >> 3) / TC_BN;  // ptile·kb + kblock
  const int kblock = (int)(blk % kb), ptile = (int)(blk / kb);
  const int b = ptile * TC_BN + row;
  const int p0 = mp * t.L - (mp * (mp - 1)) / 2;
  uint16_t v[8];
  for (int i = 0; i < 8; ++i) {
    const int k = kblock * TC_KB + c16 * 8 + i;
    KSlot s = k_slot(t.L, mp, t.split, k);
    float out = 0.f;
    if (s.seg < 3 && b < n_items) {
      const float2 g = alm[(size_t)b * n_pairs + p0 + s.l - mp];
      const float x = s.part == 0 ? g.x : g.y;
      const float hi = bf16_value(bf16_bits(x));
      out = s.seg == 1 ? x - hi : x;  // the lo part pairs with A's hi in segment 1
    }
    v[i] = bf16_bits(out);
  }
  uint8_t* blkp = B + b_off + (size_t)blk * TC_B_BLOCK;
  uint4 w;
  w.x = v[0] | ((uint32_t)v[1] << 16);
  w.y = v[2] | ((uint32_t)v[3] << 16);
  w.z = v[4] | ((uint32_t)v[5] << 16);
  w.w = v[6] | ((uint32_t)v[7] << 16);
  *(uint4*)(blkp + sw128(row, c16 * 8)) = w;
}

struct TcArgs {
  TcLayout t;
  const uint8_t* A;
  const uint8_t* B;
  int n_items;
  float2* U;
  int* status;      // nonzero after a timed-out wait (what the CTA was waiting on)
  long long limit;  // nanoseconds before a wait gives up
  long long stall;  // > 0: the failure test (the MMA thread first waits on `never`)
  int per;          // row tiles per CTA (blockIdx.z picks the group)
  float scale;      // HALF: U is stored as scale·U in FP16
};

struct TcShared {
  uint8_t b[TC_MAX_KB][TC_B_BLOCK];   // 96 KB, 1024-aligned
  uint8_t a[TC_STAGES][TC_A_BLOCK];   // 80 KB
  float stage[2][32 * TC_BM];          // 2 × 16 KB: a 32-pattern chunk of the tile, [pattern][row]
  uint64_t b_full, a_full[TC_STAGES], a_empty[TC_STAGES], acc_full[2], acc_empty[2], mma_done, never;
  long long a_off, b_off;
  uint32_t tmem;
  int failed;
};

// The FP16 form: K' <= 256 (split <= 16 at L <= 64), so 4 B blocks; 6 A stages (a tile of the
// low orders takes 4, so the next tile's loads start while its MMAs run; 225 KB in all); the drain
// stages a whole tile (128 rows × 128 items in FP16: two 16 KB store boxes) at once, two tiles deep.
constexpr int TCH_MAX_KB = 4;
constexpr int TCH_STAGES = 6;
constexpr int TCH_BOX = 64 * TC_BM * 2;  // bytes of one store box: 64 items × 128 rows
struct TcSharedH {
  uint8_t b[TCH_MAX_KB][TC_B_BLOCK];   // 64 KB, 1024-aligned
  uint8_t a[TCH_STAGES][TC_A_BLOCK];   // 64 KB
  uint8_t stage[2][2 * TCH_BOX];       // 2 × 32 KB: a tile, items 0-63 then 64-127, [ν][64 items]
  uint64_t b_full, a_full[TCH_STAGES], a_empty[TCH_STAGES], acc_full[2], acc_empty[2], mma_done, never;
  long long a_off, b_off;
  uint32_t tmem;
  int failed;
};

// 64 accumulator columns of one row ν (two TMEM loads of 32) × scale → FP16 → the row's 128 bytes
// of a store box, 16-byte chunks XOR-swizzled by ν mod 8 (the tensor map's 128-byte swizzle)
__device__ __forceinline__ void tch_row(uint8_t* box, int row, const uint32_t (&v)[32], const uint32_t (&w)[32],
                                        float sc) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 o;
    o.x = pack_half2(__uint_as_float(v[8 * q + 0]) * sc, __uint_as_float(v[8 * q + 1]) * sc);
    o.y = pack_half2(__uint_as_float(v[8 * q + 2]) * sc, __uint_as_float(v[8 * q + 3]) * sc);
    o.z = pack_half2(__uint_as_float(v[8 * q + 4]) * sc, __uint_as_float(v[8 * q + 5]) * sc);
    o.w = pack_half2(__uint_as_float(v[8 * q + 6]) * sc, __uint_as_float(v[8 * q + 7]) * sc);
    *(uint4*)(box + sw128(row, 8 * q)) = o;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint4 o;
    o.x = pack_half2(__uint_as_float(w[8 * q + 0]) * sc, __uint_as_float(w[8 * q + 1]) * sc);
    o.y = pack_half2(__uint_as_float(w[8 * q + 2]) * sc, __uint_as_float(w[8 * q + 3]) * sc);
    o.z = pack_half2(__uint_as_float(w[8 * q + 4]) * sc, __uint_as_float(w[8 * q + 5]) * sc);
    o.w = pack_half2(__uint_as_float(w[8 * q + 6]) * sc, __uint_as_float(w[8 * q + 7]) * sc);
    *(uint4*)(box + sw128(row, 32 + 8 * q)) = o;
  }
}

// HALF = false: U in FP32 as [item][j][m'][c] (re, im); true: scale·U in FP16 as
// [item tile][(j, c)][m'][re|im][128 items] (items padded to whole tiles of 128), the layout the
// tensor-core transform along a (slab_tc.cu) loads its operand tiles from.
template <bool HALF>
__global__ void __launch_bounds__(TC_THREADS, 1) k_spectrum_tc(TcArgs a, const __grid_constant__ CUtensorMap umap) {
  using Sh = std::conditional_t<HALF, TcSharedH, TcShared>;
  constexpr int NST = HALF ? TCH_STAGES : TC_STAGES;
  extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
  Sh& s = *reinterpret_cast<Sh*>((void*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ptile = blockIdx.x, mp = blockIdx.y;
  const TcLayout& t = a.t;
  const int kb = tc_kblocks(t.L, mp, t.split);
  // this CTA's row tiles: [mt0, mt0 + mtiles) of the order's t.mtiles
  const int mt0 = blockIdx.z * a.per;
  const int mtiles = max(0, min(t.mtiles - mt0, a.per));
  if (threadIdx.x == 0) {
    mbar_init(&s.b_full, 1);
    mbar_init(&s.mma_done, 1);
    mbar_init(&s.never, 1);  // nothing arrives: the failure test's wait
    s.a_off = tc_offset(t.L, t.split, mp, t.mtiles, TC_A_BLOCK);
    s.b_off = tc_offset(t.L, t.split, mp, t.ptiles, TC_B_BLOCK);
    for (int i = 0; i < NST; ++i) {
      mbar_init(&s.a_full[i], 1);
      mbar_init(&s.a_empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.acc_full[i], 1);
      mbar_init(&s.acc_empty[i], 4);
    }
    s.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem)),
                 "r"(2 * TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s.tmem;
  const long long lim = a.limit;

  if (warp == 0) {
    if (lane == 0) {
      // B once; then A block by block through the ring (block it of the CTA goes to stage it mod S)
      const uint8_t* bsrc = a.B + s.b_off + (size_t)ptile * kb * TC_B_BLOCK;
      mbar_expect_tx(&s.b_full, kb * TC_B_BLOCK);
      for (int k = 0; k < kb; ++k) bulk_g2s(s.b[k], bsrc + (size_t)k * TC_B_BLOCK, TC_B_BLOCK, &s.b_full);
      const uint8_t* asrc = a.A + s.a_off + (size_t)mt0 * kb * TC_A_BLOCK;
      const int total = mtiles * kb;  // this CTA's blocks of the order's A, [mtile][kblock]
      int it = 0;
      for (; it < total; ++it) {
        const int st = it % NST;
        if (!mbar_wait(&s.a_empty[st], ((it / NST) & 1) ^ 1, lim)) break;
        mbar_expect_tx(&s.a_full[st], TC_A_BLOCK);
        bulk_g2s(s.a[st], asrc + (size_t)it * TC_A_BLOCK, TC_A_BLOCK, &s.a_full[st]);
      }
      if (it < total) {
        atomicOr(a.status, 1);
        s.failed = 1;
      }
      // the copies still in flight land before the CTA may leave, whether or not the MMAs took
      // them (bounded waits on their phases; a phase already consumed reads as complete)
      mbar_wait(&s.b_full, 0, kDrainNs);
      for (int i = (it > NST ? it - NST : 0); i < it; ++i)
        mbar_wait(&s.a_full[i % NST], (i / NST) & 1, kDrainNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // kind::f16: F32 accumulate, BF16 A and B, both K-major, N = 128, M = 128
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
      bool ok = mbar_wait(&s.b_full, 0, lim);
      if (a.stall > 0 && !mbar_wait(&s.never, 0, a.stall)) ok = false;  // the failure test
      int it = 0;
      for (int mt = 0; mt < mtiles && ok; ++mt) {
        const int acc = mt & 1;
        ok = mbar_wait(&s.acc_empty[acc], ((mt >> 1) & 1) ^ 1, lim);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * TC_BN);
        for (int k = 0; k < kb; ++k, ++it) {
          const int st = it % NST;
          ok = mbar_wait(&s.a_full[st], (it / NST) & 1, lim);
          if (!ok) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t abase = smem_addr(s.a[st]), bbase = smem_addr(s.b[k]);
#pragma unroll
          for (int ks = 0; ks < TC_KB / 16; ++ks)
            umma_f16(d, umma_desc(abase + ks * 32), umma_desc(bbase + ks * 32), idesc, (k | ks) != 0);
          umma_commit(&s.a_empty[st]);  // the stage is free once these MMAs have read it
        }
        if (!ok) break;
        umma_commit(&s.acc_full[acc]);
      }
      if (!ok) {
        atomicOr(a.status, 2);
        s.failed = 1;
      }
      // every MMA issued has finished before TMEM may be freed
      umma_commit(&s.mma_done);
      if (!mbar_wait(&s.mma_done, 0, kDrainNs)) atomicOr(a.status, 8);
    }
  } else {
    // epilogue (warps 2-5): a warp may reach only its TMEM lane quadrant, so warp w drains tile
    // rows 32·(w mod 4) …  Each 32-pattern chunk goes TMEM → registers → a staging buffer laid
    // out [pattern][row] (the tensor-store box: rows ν of a tile are whole (j, m') lines of U)
    // → one 16 KB tensor store; rows and patterns past the ends are clipped by the store.
    const int ew = warp & 3;
    const int row = ew * 32 + lane;
    const bool leader = warp == 2 && lane == 0;
    const int two_nc = 2 * t.nc;
    int chunk = 0;
    for (int mt = 0; mt < mtiles; ++mt) {
      if constexpr (HALF) {
        // the whole tile at once: four TMEM loads (128 items of row ν), the accumulator handed back
        // to the MMAs, FP16 rows into the tile's staging buffer, two 16 KB tensor stores; the
        // buffer of two tiles back has been read by its stores (the last group may still read)
        const int acc = mt & 1;
        // the leader polls (no backoff: a sleep would outlast the MMAs of a tile), the others wait at
        // the barrier
        if (!bar_and(1, 128, leader ? mbar_wait(&s.acc_full[acc], (mt >> 1) & 1, lim) : true)) {
          if (leader) {
            atomicOr(a.status, 4);
            s.failed = 1;
          }
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r0 = (mt0 + mt) * TC_BM;  // first row ν of the tile
        const uint32_t ta = tmem + ((uint32_t)(ew * 32) << 16) + (uint32_t)(acc * TC_BN);
        uint32_t v0[32], v1[32], v2[32], v3[32];
        TMEM_LD32(ta, v0);
        TMEM_LD32(ta + 32, v1);
        TMEM_LD32(ta + 64, v2);
        TMEM_LD32(ta + 96, v3);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.acc_empty[acc]);
        uint8_t* stg = s.stage[mt & 1];
        if (leader) bulk_wait_read1();
        bar_sync(1, 128);
        const float sc = a.scale;
        tch_row(stg, row, v0, v1, sc);
        tch_row(stg + TCH_BOX, row, v2, v3, sc);
        fence_proxy_async();
        bar_sync(1, 128);
        if (leader) {
          if (ptile * TC_BN < a.n_items) tma_store_5d(&umap, stg, 0, 0, mp, r0 >> 1, ptile);
          if (ptile * TC_BN + 64 < a.n_items) tma_store_5d(&umap, stg + TCH_BOX, 64, 0, mp, r0 >> 1, ptile);
          bulk_commit();
        }
      } else {
        const int acc = mt & 1;
        // the four warps agree on the outcome (a barrier that ANDs their results)
        // one thread waits for the accumulator (sleeping between polls); the barrier hands the
        // outcome to the others, which wait there without taking issue slots
        if (!bar_and(1, 128, leader ? mbar_wait_sleep(&s.acc_full[acc], (mt >> 1) & 1, lim) : true)) {
          if (leader) {
            atomicOr(a.status, 4);
            s.failed = 1;
          }
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r0 = (mt0 + mt) * TC_BM;  // first row ν of the tile
        const int j0 = r0 / two_nc, x0 = two_nc <= TC_BM ? 0 : r0 % two_nc;
#pragma unroll 1
        for (int c0 = 0; c0 < TC_BN; c0 += 32, ++chunk) {
          uint32_t v[32];
          TMEM_LD32(tmem + ((uint32_t)(ew * 32) << 16) + (uint32_t)(acc * TC_BN + c0), v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (c0 + 32 == TC_BN) {  // the accumulator is read out: the next tile's MMAs may start
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&s.acc_empty[acc]);
          }
          float* stg = s.stage[chunk & 1];
          if (leader) bulk_wait_read1();  // the store that last used this buffer has read it
          bar_sync(1, 128);
#pragma unroll
          for (int c = 0; c < 32; ++c) stg[c * TC_BM + row] = __uint_as_float(v[c]);
          fence_proxy_async();
          bar_sync(1, 128);
          if (leader) {
            if (ptile * TC_BN + c0 < a.n_items) tma_store_4d(&umap, stg, x0, mp, j0, ptile * TC_BN + c0);
            bulk_commit();
          }
        }
      }
    }
    if (leader) bulk_wait_all();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_BN));
}

}  // namespace zeb

using namespace zeb;

static bool tc_dims_ok(const zeb_so3_dims_t* d, int split) {
  return d && d->L >= 2 && d->L <= 256 && d->n >= 2 * d->L - 1 && d->nb == d->n / 2 + 1 && d->fold >= 1 &&
         d->nc == d->n / d->fold && d->mu_max == (d->L - 1) / d->fold && d->n_pairs == d->L * (d->L + 1) / 2 &&
         split >= -1 && tc_kblocks(d->L, 0, split) <= TC_MAX_KB;
}

static TcLayout tc_layout(const zeb_so3_dims_t* d, int split, int n_items) {
  TcLayout t{};
  t.L = d->L; t.nb = d->nb; t.nc = d->nc; t.rows = 2 * d->nb * d->nc;
  t.mtiles = (t.rows + TC_BM - 1) / TC_BM;
  t.ptiles = (n_items + TC_BN - 1) / TC_BN;
  t.split = split;
  return t;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tc_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// U as a 4-D tensor [item][j][m'][2·nc floats]; the box is one tile's rows for 32 items
static bool tc_u_map(CUtensorMap* m, float* U, const zeb_so3_dims_t* d, int n_items) {
  auto fn = tc_encode_fn();
  if (!fn) return false;
  const cuuint64_t two_nc = 2 * (cuuint64_t)d->nc;
  cuuint64_t dims[4] = {two_nc, (cuuint64_t)d->L, (cuuint64_t)d->nb, (cuuint64_t)n_items};
  cuuint64_t strides[3] = {two_nc * 4, two_nc * 4 * d->L, two_nc * 4 * d->L * d->nb};
  cuuint32_t box[4] = {(cuuint32_t)(two_nc <= TC_BM ? two_nc : TC_BM), 1,
                       (cuuint32_t)(two_nc <= TC_BM ? TC_BM / two_nc : 1), 32};
  cuuint32_t es[4] = {1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, U, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

extern "C" size_t zeb_tc_master_bytes(const zeb_so3_dims_t* d, int split) {
  if (!tc_dims_ok(d, split)) return 0;
  TcLayout t = tc_layout(d, split, 1);
  return (size_t)tc_offset(d->L, split, d->L, t.mtiles, TC_A_BLOCK);
}

extern "C" size_t zeb_tc_patterns_bytes(const zeb_so3_dims_t* d, int split, int n_items) {
  if (!tc_dims_ok(d, split) || n_items <= 0) return 0;
  TcLayout t = tc_layout(d, split, n_items);
  return (size_t)tc_offset(d->L, split, d->L, t.ptiles, TC_B_BLOCK);
}

extern "C" int zeb_tc_pack_master(const zeb_so3_dims_t* d, int split, const double* Y, void* A, void* stream) {
  ZEB_REQUIRE(Y && A, ZEB_EARG, "tc_pack_master: null argument");
  ZEB_REQUIRE(tc_dims_ok(d, split), ZEB_EARG, "tc_pack_master: unsupported dims (L=%d, split=%d)", d ? d->L : -1,
              split);
  TcLayout t = tc_layout(d, split, 1);
  cudaStream_t st = (cudaStream_t)stream;
  for (int mp = 0; mp < d->L; ++mp) {
    long long chunks = (long long)t.mtiles * tc_kblocks(d->L, mp, split) * TC_BM * 8;
    k_pack_master<<<(unsigned)((chunks + 255) / 256), 256, 0, st>>>(
        (const double2*)Y, t, mp, tc_offset(d->L, split, mp, t.mtiles, TC_A_BLOCK), (uint8_t*)A);
  }
  return zeb_launch_check("tc_pack_master");
}

extern "C" int zeb_spectrum_bf16(const float* alm, int n_items, const zeb_so3_dims_t* d, int split, const void* A,
                                 void* B, float* U, int* status, void* stream) {
  ZEB_REQUIRE(alm && A && B && U && status, ZEB_EARG, "spectrum_bf16: null argument");
  ZEB_REQUIRE(tc_dims_ok(d, split), ZEB_EARG, "spectrum_bf16: unsupported dims (L=%d, split=%d)", d ? d->L : -1,
              split);
  if (n_items <= 0) return ZEB_OK;
  TcLayout t = tc_layout(d, split, n_items);
  cudaStream_t st = (cudaStream_t)stream;
  long long chunks = (long long)t.ptiles * tc_kblocks(d->L, 0, split) * TC_BN * 8;
  dim3 gp((unsigned)((chunks + 255) / 256), d->L);
  k_pack_patterns<<<gp, 256, 0, st>>>((const float2*)alm, n_items, d->n_pairs, t, (uint8_t*)B);
  int rc = zeb_launch_check("pack_patterns");
  if (rc) return rc;
  CUtensorMap umap;
  ZEB_REQUIRE(((uintptr_t)U & 15) == 0, ZEB_EARG, "spectrum_bf16: U must be 16-byte aligned");
  ZEB_REQUIRE(tc_u_map(&umap, U, d, n_items), ZEB_ECUDA, "spectrum_bf16: tensor map for U refused");
  TcArgs a{};
  a.t = t; a.A = (const uint8_t*)A; a.B = (const uint8_t*)B; a.n_items = n_items; a.U = (float2*)U;
  a.status = status;
  a.stall = test_stall_ns();
  a.limit = a.stall > 0 ? a.stall : kWaitNs;
  size_t smem = sizeof(TcShared) + 1024;
  cudaFuncSetAttribute(k_spectrum_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // enough CTAs for several waves: row tiles split into groups when the pattern tiles are few
  int sms = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const long long base = (long long)t.ptiles * d->L;
  int groups = (int)std::min<long long>(t.mtiles, (8LL * sms + base - 1) / base);
  groups = std::max(1, std::min(groups, 65535));
  a.per = (t.mtiles + groups - 1) / groups;
  groups = (t.mtiles + a.per - 1) / a.per;  // no empty group: every CTA has at least one row tile
  dim3 g(t.ptiles, d->L, groups);
  k_spectrum_tc<false><<<g, TC_THREADS, smem, st>>>(a, umap);
  return zeb_launch_check("spectrum_bf16");
}

// scale·U in FP16 as [item tile][(j, c)][m'][re|im][128 items]: a 5-D tensor (items within the tile,
// re|im, order, (j, c), tile); a store box is 64 items × the 128 rows ν = 2(j·nc + c) + (re|im) of a
// row tile (64 (j, c) × re|im) of one order and one tile, with the staging buffer's 128-byte
// swizzle. One (j, c) of one tile of items is then 2L × 256 contiguous bytes: what the transform
// along a loads as one operand tile; and a CTA's stores (one tile, one order) stay within the
// tile's region of 2L × 256 bytes × (j, c).
static bool tc_u16_map(CUtensorMap* m, void* U16, const zeb_so3_dims_t* d, int n_items) {
  auto fn = tc_encode_fn();
  if (!fn) return false;
  const cuuint64_t ptiles = (cuuint64_t)((n_items + TC_BN - 1) / TC_BN);
  const cuuint64_t L = (cuuint64_t)d->L, jc = (cuuint64_t)d->nb * d->nc;
  cuuint64_t dims[5] = {TC_BN, 2, L, jc, ptiles};
  cuuint64_t strides[4] = {TC_BN * 2, TC_BN * 4, TC_BN * 4 * L, TC_BN * 4 * L * jc};
  cuuint32_t box[5] = {64, 2, 1, (cuuint32_t)TC_BM / 2, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 5, U16, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

extern "C" size_t zeb_spectrum_h_bytes(const zeb_so3_dims_t* d, int n_items) {
  if (!tc_dims_ok(d, -1) || n_items <= 0) return 0;
  const size_t ppad = (size_t)((n_items + TC_BN - 1) / TC_BN) * TC_BN;
  return (size_t)d->L * 2 * d->nb * d->nc * ppad * 2;
}

extern "C" int zeb_spectrum_bf16_h(const float* alm, int n_items, const zeb_so3_dims_t* d, int split, const void* A,
                                   void* B, void* U16, float scale, int* status, void* stream) {
  ZEB_REQUIRE(alm && A && B && U16 && status, ZEB_EARG, "spectrum_bf16_h: null argument");
  ZEB_REQUIRE(tc_dims_ok(d, split), ZEB_EARG, "spectrum_bf16_h: unsupported dims (L=%d, split=%d)", d ? d->L : -1,
              split);
  ZEB_REQUIRE(2 * d->nb * d->nc >= TC_BM, ZEB_EARG, "spectrum_bf16_h: bandwidth %d too small", d->L);
  ZEB_REQUIRE(tc_kblocks(d->L, 0, split) <= TCH_MAX_KB, ZEB_EARG,
              "spectrum_bf16_h: K' of %d blocks (L=%d, split=%d) exceeds the FP16 form's %d", tc_kblocks(d->L, 0, split),
              d->L, split, TCH_MAX_KB);
  ZEB_REQUIRE(scale > 0.f && scale < 1e30f, ZEB_EARG, "spectrum_bf16_h: scale %g", (double)scale);
  if (n_items <= 0) return ZEB_OK;
  TcLayout t = tc_layout(d, split, n_items);
  cudaStream_t st = (cudaStream_t)stream;
  long long chunks = (long long)t.ptiles * tc_kblocks(d->L, 0, split) * TC_BN * 8;
  dim3 gp((unsigned)((chunks + 255) / 256), d->L);
  k_pack_patterns<<<gp, 256, 0, st>>>((const float2*)alm, n_items, d->n_pairs, t, (uint8_t*)B);
  int rc = zeb_launch_check("pack_patterns");
  if (rc) return rc;
  CUtensorMap umap;
  ZEB_REQUIRE(((uintptr_t)U16 & 127) == 0, ZEB_EARG, "spectrum_bf16_h: U16 must be 128-byte aligned");
  ZEB_REQUIRE(tc_u16_map(&umap, U16, d, n_items), ZEB_ECUDA, "spectrum_bf16_h: tensor map for U16 refused");
  TcArgs a{};
  a.t = t; a.A = (const uint8_t*)A; a.B = (const uint8_t*)B; a.n_items = n_items; a.U = nullptr;
  a.status = status;
  a.stall = test_stall_ns();
  a.limit = a.stall > 0 ? a.stall : kWaitNs;
  a.scale = scale;
  size_t smem = sizeof(TcSharedH) + 1024;
  cudaFuncSetAttribute(k_spectrum_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int sms = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const long long base = (long long)t.ptiles * d->L;
  int groups = (int)std::min<long long>(t.mtiles, (8LL * sms + base - 1) / base);
  groups = std::max(1, std::min(groups, 65535));
  a.per = (t.mtiles + groups - 1) / groups;
  groups = (t.mtiles + a.per - 1) / a.per;
  dim3 g(t.ptiles, d->L, groups);
  k_spectrum_tc<true><<<g, TC_THREADS, smem, st>>>(a, umap);
  return zeb_launch_check("spectrum_bf16_h");
}
