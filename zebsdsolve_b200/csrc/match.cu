// Dictionary indexing: every pattern scored against every simulated pattern of an orientation
// dictionary (or against the dictionary's PCA coefficients), the best entry kept.
//
//   k_dict_sims   the dictionary's entries simulated at one detector position, zero mean and unit
//                 norm under the mask (detector.wgsl project_dict 266-273 + sim_norm 662-699)
//   k_pack_panel  FP32 rows → BF16 in the tensor cores' operand layout
//   k_match_tc    S = X·Dᵀ on the tcgen05 tensor cores (BF16 operands, FP32 accumulation in tensor
//                 memory), each pattern's eight largest scores kept by the epilogue as the tiles of
//                 S drain: S itself is never written (at 10⁵ patterns × 3·10⁵ entries it would be
//                 120 GB)
//   k_match_f32   the same scores in plain FP32 on the CUDA cores, the best per dictionary slice
//                 (the reference's dict_score / pca nearest, detector.wgsl:705-740, pca.wgsl:114-168)
//   k_match_best  each pattern's candidates scored again in FP32 against the FP32 rows, the best
//                 (ties to the lower index) written as a seed (q, score, index) for the refinement
//
// Panel layout (the operand layout of the MMA): blocks of 64 K-elements (one 128-byte row per
// matrix row), [k-block][row][128 B], the 16-byte chunks of row r XOR-swizzled by r mod 8; rows
// padded to a multiple of 256 with zeros, K to a multiple of 64.  A block of 128 (A) or 256 (B)
// consecutive rows of one k-block is then one contiguous bulk copy.
#include <algorithm>

#include "abi_util.cuh"
#include "tc_util.cuh"

namespace zeb {

constexpr int MT_BM = 128;               // patterns per tile (MMA M)
constexpr int MT_BN = 256;               // dictionary entries per tile (MMA N)
constexpr int MT_A_BLOCK = MT_BM * 128;  // 16 KB
constexpr int MT_B_BLOCK = MT_BN * 128;  // 32 KB
constexpr int MT_STAGES = 4;
constexpr int MT_EPI = 8;                          // epilogue warps: two per TMEM lane quadrant
constexpr int MT_THREADS = 64 + 32 * MT_EPI;       // + the copy warp and the MMA warp
constexpr int MT_TOP = 8;

__host__ __device__ inline int panel_rows(int rows) { return (rows + 255) / 256 * 256; }
__host__ __device__ inline int panel_kblocks(int cols) { return (cols + 63) / 64; }

// ── simulation of the dictionary ──

struct SimArgs {
  int h, w;
  float3 c0, c1, t0;
  float mask[3];
  const float2* vpair;
  int side;
  const float4* q;
  float* out;
};

__global__ void __launch_bounds__(256) k_dict_sims(SimArgs a) {
  extern __shared__ float sim_px[];
  __shared__ float red[2][8];
  const int e = blockIdx.x;
  const int hw = a.h * a.w;
  const float4 q = __ldg(a.q + e);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float sum = 0.f, cnt = 0.f;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    const int row = i / a.w, col = i - row * a.w;
    const float dr = (float)row - a.mask[0], dc = (float)col - a.mask[1];
    float v = 0.f;
    if (zeb_in_circle(dr, dc, a.mask[2])) {
      const float3 u = normalize3(make_float3(a.c0.x * row + a.c1.x * col + a.t0.x, a.c0.y * row + a.c1.y * col + a.t0.y,
                                              a.c0.z * row + a.c1.z * col + a.t0.z));
      v = master_at_pair(a.vpair, qrot(q, u), a.side);
      sum += v;
      cnt += 1.f;
    }
    sim_px[i] = v;
  }
  sum = warp_sum(sum);
  cnt = warp_sum(cnt);
  if (lane == 0) { red[0][wid] = sum; red[1][wid] = cnt; }
  __syncthreads();
  float tot = 0.f, n = 0.f;
  for (int k = 0; k < 8; ++k) { tot += red[0][k]; n += red[1][k]; }
  const float mean = tot / fmaxf(n, 1.f);
  __syncthreads();
  float ss = 0.f;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    const int row = i / a.w, col = i - row * a.w;
    const float dr = (float)row - a.mask[0], dc = (float)col - a.mask[1];
    const float d = zeb_in_circle(dr, dc, a.mask[2]) ? sim_px[i] - mean : 0.f;
    sim_px[i] = d;
    ss += d * d;
  }
  ss = warp_sum(ss);
  if (lane == 0) red[0][wid] = ss;
  __syncthreads();
  float tss = 0.f;
  for (int k = 0; k < 8; ++k) tss += red[0][k];
  const float inv = rsqrtf(fmaxf(tss, 1e-30f));
  float* o = a.out + (size_t)e * hw;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) o[i] = sim_px[i] * inv;
}

// ── BF16 panels ──

__global__ void k_pack_panel(const float* __restrict__ src, int rows, int cols, int ld, int rows_pad, int kblocks,
                             uint8_t* __restrict__ dst) {
  const long long chunks = (long long)kblocks * rows_pad * 8;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= chunks) return;
  const int c16 = (int)(e & 7);
  const int row = (int)((e >> 3) % rows_pad);
  const int kb = (int)((e >> 3) / rows_pad);
  const int k0 = kb * 64 + c16 * 8;
  uint16_t v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = k0 + i;
    v[i] = bf16_bits(row < rows && k < cols ? __ldg(src + (size_t)row * ld + k) : 0.f);
  }
  uint4 wv;
  wv.x = v[0] | ((uint32_t)v[1] << 16);
  wv.y = v[2] | ((uint32_t)v[3] << 16);
  wv.z = v[4] | ((uint32_t)v[5] << 16);
  wv.w = v[6] | ((uint32_t)v[7] << 16);
  *(uint4*)(dst + (size_t)kb * rows_pad * 128 + sw128(row, c16 * 8)) = wv;
}

// The panel of FP32 rows as three K segments of BF16 for a near-FP32 product on the tensor cores:
// x = hi + lo with hi = bf16(x), lo = bf16(x − hi); segment order (hi, hi, lo) for the left
// operand (role 0) and (hi, lo, hi) for the right one (role 1), so that the one GEMM over the
// three segments sums hi·hi + hi·lo + lo·hi.
__global__ void k_pack_panel_split(const float* __restrict__ src, int rows, int cols, int ld, int rows_pad,
                                   int kblocks, int role, uint8_t* __restrict__ dst) {
  const long long chunks = 3LL * kblocks * rows_pad * 8;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= chunks) return;
  const int c16 = (int)(e & 7);
  const int row = (int)((e >> 3) % rows_pad);
  const int kbs = (int)((e >> 3) / rows_pad);  // K-block of the whole panel
  const int seg = kbs / kblocks, kb = kbs - seg * kblocks;
  const bool lo = role == 0 ? seg == 2 : seg == 1;
  const int k0 = kb * 64 + c16 * 8;
  uint16_t v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = k0 + i;
    const float x = row < rows && k < cols ? __ldg(src + (size_t)row * ld + k) : 0.f;
    const float hi = bf16_value(bf16_bits(x));
    v[i] = bf16_bits(lo ? x - hi : x);
  }
  uint4 wv;
  wv.x = v[0] | ((uint32_t)v[1] << 16);
  wv.y = v[2] | ((uint32_t)v[3] << 16);
  wv.z = v[4] | ((uint32_t)v[5] << 16);
  wv.w = v[6] | ((uint32_t)v[7] << 16);
  *(uint4*)(dst + (size_t)kbs * rows_pad * 128 + sw128(row, c16 * 8)) = wv;
}

// ── top eight on the tensor cores ──

struct MatchArgs {
  const uint8_t* A;  // patterns' panel
  const uint8_t* B;  // dictionary's panel
  int rows_a, rows_b, kb;
  int n_exp, n_dict;
  int per;     // dictionary tiles per slice
  int slices;
  float* cand_v;
  int* cand_i;
  int* status;
  long long limit;
  long long stall;  // > 0: the failure test (the MMA thread first waits on `never`)
  float* out;       // PROJECT: the products themselves, out[p][entry] (n_exp × n_dict)
};

struct MatchShared {
  uint8_t a[MT_STAGES][MT_A_BLOCK];
  uint8_t b[MT_STAGES][MT_B_BLOCK];
  float stash[32][32 * MT_EPI];  // a chunk of each epilogue thread's scores, [column][thread]
  uint64_t full[MT_STAGES], empty[MT_STAGES], acc_full[2], acc_empty[2], mma_done, never;
  uint32_t tmem;
};

// (x, i) before (y, j): the larger score first, equal scores in index order
__device__ __forceinline__ bool top8_before(float x, int i, float y, int j) { return x > y || (x == y && i < j); }

// insert (x, i) into the list (v, id) of eight kept in that order
__device__ __forceinline__ void top8_insert(float (&v)[MT_TOP], int (&id)[MT_TOP], float x, int i) {
  if (!top8_before(x, i, v[MT_TOP - 1], id[MT_TOP - 1])) return;
  v[MT_TOP - 1] = x;
  id[MT_TOP - 1] = i;
#pragma unroll
  for (int k = MT_TOP - 1; k > 0; --k) {
    if (top8_before(v[k], id[k], v[k - 1], id[k - 1])) {
      const float tv = v[k]; v[k] = v[k - 1]; v[k - 1] = tv;
      const int ti = id[k]; id[k] = id[k - 1]; id[k - 1] = ti;
    }
  }
}

// push (x, i) into the descending list when it beats the last entry (equal scores keep the
// entry already there, which came first): every slot's new content from the comparisons with
// the old list at once, no chain of dependent swaps
__device__ __forceinline__ void top8_push(float (&v)[MT_TOP], int (&id)[MT_TOP], float x, int i) {
  bool gt[MT_TOP];
#pragma unroll
  for (int k = 0; k < MT_TOP; ++k) gt[k] = x > v[k];
#pragma unroll
  for (int k = MT_TOP - 1; k > 0; --k) {
    v[k] = gt[k - 1] ? v[k - 1] : (gt[k] ? x : v[k]);
    id[k] = gt[k - 1] ? id[k - 1] : (gt[k] ? i : id[k]);
  }
  v[0] = gt[0] ? x : v[0];
  id[0] = gt[0] ? i : id[0];
}

// PROJECT: the epilogue writes every product (the patterns' coefficients on the components of a
// PCA, zeb_project_bf16) instead of keeping each pattern's eight best
template <bool PROJECT>
__global__ void __launch_bounds__(MT_THREADS, 1) k_match_tc(MatchArgs a) {
  extern __shared__ __align__(1024) uint8_t mt_smem_raw[];
  MatchShared& s = *reinterpret_cast<MatchShared*>((void*)(((uintptr_t)mt_smem_raw + 1023) & ~(uintptr_t)1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.x, slice = blockIdx.y;
  const int ntiles = (a.n_dict + MT_BN - 1) / MT_BN;
  const int nt0 = slice * a.per;
  const int my_tiles = max(0, min(ntiles - nt0, a.per));
  if (threadIdx.x == 0) {
    for (int i = 0; i < MT_STAGES; ++i) {
      mbar_init(&s.full[i], 1);
      mbar_init(&s.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.acc_full[i], 1);
      mbar_init(&s.acc_empty[i], MT_EPI);
    }
    mbar_init(&s.mma_done, 1);
    mbar_init(&s.never, 1);  // nothing arrives: the failure test's wait
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem)),
                 "r"(2 * MT_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s.tmem;
  const long long lim = a.limit;
  const int total = my_tiles * a.kb;  // (tile, k-block) steps of this CTA

  if (warp == 0) {
    if (lane == 0) {
      const uint8_t* abase = a.A + (size_t)mt * MT_A_BLOCK;
      int it = 0;
      for (; it < total; ++it) {
        const int st = it % MT_STAGES;
        const int t = it / a.kb, k = it - t * a.kb;
        if (!mbar_wait(&s.empty[st], ((it / MT_STAGES) & 1) ^ 1, lim)) break;
        mbar_expect_tx(&s.full[st], MT_A_BLOCK + MT_B_BLOCK);
        bulk_g2s(s.a[st], abase + (size_t)k * a.rows_a * 128, MT_A_BLOCK, &s.full[st]);
        bulk_g2s(s.b[st], a.B + (size_t)k * a.rows_b * 128 + (size_t)(nt0 + t) * MT_B_BLOCK, MT_B_BLOCK, &s.full[st]);
      }
      if (it < total) atomicOr(a.status, 1);
      // the copies still in flight land before the CTA may leave (bounded waits on their phases;
      // a phase already consumed reads as complete)
      for (int i = (it > MT_STAGES ? it - MT_STAGES : 0); i < it; ++i)
        mbar_wait(&s.full[i % MT_STAGES], (i / MT_STAGES) & 1, kDrainNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // kind::f16: F32 accumulate, BF16 A and B, both K-major, N = 256, M = 128
      const uint32_t idesc =
          (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(MT_BN >> 3) << 17) | ((uint32_t)(MT_BM >> 4) << 24);
      bool ok = true;
      if (a.stall > 0 && !mbar_wait(&s.never, 0, a.stall)) ok = false;  // the failure test
      int it = 0;
      for (int t = 0; t < my_tiles && ok; ++t) {
        const int acc = t & 1;
        ok = mbar_wait(&s.acc_empty[acc], ((t >> 1) & 1) ^ 1, lim);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * MT_BN);
        for (int k = 0; k < a.kb; ++k, ++it) {
          const int st = it % MT_STAGES;
          ok = mbar_wait(&s.full[st], (it / MT_STAGES) & 1, lim);
          if (!ok) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t ab = smem_addr(s.a[st]), bb = smem_addr(s.b[st]);
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            umma_f16(d, umma_desc(ab + ks * 32), umma_desc(bb + ks * 32), idesc, (k | ks) != 0);
          umma_commit(&s.empty[st]);
        }
        if (!ok) break;
        umma_commit(&s.acc_full[acc]);
      }
      if (!ok) atomicOr(a.status, 2);
      umma_commit(&s.mma_done);
      if (!mbar_wait(&s.mma_done, 0, kDrainNs)) atomicOr(a.status, 8);
    }
  } else {
    // epilogue: warp w may read only TMEM lanes 32·(w mod 4) …, so warps w and w + 4 share a
    // quadrant and split the 256 columns: thread = one pattern (row of the tile) × one half of
    // the entries of each tile.  The two halves' lists merge at the end.
    const int ew = warp & 3;
    const int row = ew * 32 + lane;
    const int half = (warp - 2) >> 2;
    const int me = half * MT_BM + row;  // this thread's column of the stash
    const uint32_t lanes = (uint32_t)(ew * 32) << 16;
    float tv[MT_TOP];
    int ti[MT_TOP];
#pragma unroll
    for (int k = 0; k < MT_TOP; ++k) { tv[k] = -3.4e38f; ti[k] = -1; }
    // the scores v of entries e0 + j (j < 32; none past the dictionary's end) into the list: a
    // mask of the scores above the list's last entry first; only those (after the first tiles,
    // rarely any) go in, one at a time from the thread's own column of the stash (registers
    // cannot be indexed by a variable)
    auto take = [&](const uint32_t (&v)[32], int e0) {
      const int lim_c = min(32, a.n_dict - e0);
      const float th = tv[MT_TOP - 1];
      uint32_t mask = 0;
#pragma unroll
      for (int c = 0; c < 32; ++c) mask |= (c < lim_c && __uint_as_float(v[c]) > th) ? (1u << c) : 0u;
      if (mask) {
#pragma unroll
        for (int c = 0; c < 32; ++c) s.stash[c][me] = __uint_as_float(v[c]);
        while (mask) {
          const int c = __ffs(mask) - 1;
          mask &= mask - 1;
          top8_push(tv, ti, s.stash[c][me], e0 + c);
        }
      }
    };
    bool ok = true;
    for (int t = 0; t < my_tiles; ++t) {
      const int acc = t & 1;
      // one thread waits for the accumulator (sleeping between polls); the barrier hands the
      // outcome to the others, which wait there without taking issue slots
      const bool lead = warp == 2 && lane == 0;
      if (!bar_and(1, 32 * MT_EPI, lead ? mbar_wait_sleep(&s.acc_full[acc], (t >> 1) & 1, lim) : true)) {
        if (warp == 2 && lane == 0) atomicOr(a.status, 4);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int e0 = (nt0 + t) * MT_BN + half * 128;
      const uint32_t c0 = tmem + lanes + (uint32_t)(acc * MT_BN + half * 128);
      if constexpr (PROJECT) {
        // four chunks of 32 columns, each stored as it is read (the row's entries past n_dict and
        // the rows past n_exp not at all)
        const int p = mt * MT_BM + row;
        float* orow = a.out + (size_t)p * a.n_dict;
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
          uint32_t v[32];
          TMEM_LD32(c0 + 32 * q, v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (q == 3) {  // the accumulator is read out: the MMAs of tile t + 2 may start
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&s.acc_empty[acc]);
          }
          const int eq = e0 + 32 * q;
          if (p < a.n_exp) {
            if (eq + 32 <= a.n_dict && (a.n_dict & 3) == 0) {
#pragma unroll
              for (int c = 0; c < 32; c += 4)
                *(float4*)(orow + eq + c) = make_float4(__uint_as_float(v[c]), __uint_as_float(v[c + 1]),
                                                        __uint_as_float(v[c + 2]), __uint_as_float(v[c + 3]));
            } else {
#pragma unroll
              for (int c = 0; c < 32; ++c)
                if (eq + c < a.n_dict) orow[eq + c] = __uint_as_float(v[c]);
            }
          }
        }
        continue;
      }
      // four chunks of 32 columns, the next one's load in flight while one is taken
      uint32_t va[32], vb[32];
      TMEM_LD32(c0, va);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      TMEM_LD32(c0 + 32, vb);
      take(va, e0);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      TMEM_LD32(c0 + 64, va);
      take(vb, e0 + 32);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      TMEM_LD32(c0 + 96, vb);
      take(va, e0 + 64);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // the accumulator is read out: the MMAs of tile t + 2 may start
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&s.acc_empty[acc]);
      take(vb, e0 + 96);
    }
    // the second half's list joins the first's (through the stash, once every thread is done)
    if constexpr (!PROJECT) {
      bar_sync(1, 32 * MT_EPI);
      if (half == 1) {
#pragma unroll
        for (int k = 0; k < MT_TOP; ++k) {
          s.stash[k][row] = tv[k];
          s.stash[MT_TOP + k][row] = __int_as_float(ti[k]);
        }
      }
      bar_sync(1, 32 * MT_EPI);
      const int p = mt * MT_BM + row;
      if (half == 0) {
#pragma unroll 1
        for (int k = 0; k < MT_TOP; ++k)
          top8_insert(tv, ti, s.stash[k][row], __float_as_int(s.stash[MT_TOP + k][row]));
        if (ok && p < a.n_exp) {
          const size_t o = ((size_t)p * a.slices + slice) * MT_TOP;
#pragma unroll
          for (int k = 0; k < MT_TOP; ++k) {
            a.cand_v[o + k] = tv[k];
            a.cand_i[o + k] = ti[k];
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * MT_BN));
}

// ── the plain FP32 form ──
//
// 64 patterns × 128 entries per tile, K in steps of 16 through shared memory, 4 × 8 scores per
// thread; after each tile every pattern's best of its 128 entries joins its running best.
constexpr int MF_BM = 64, MF_BN = 128, MF_BK = 16;

// PROJECT: every product is written to out[p][entry] (the coefficients of a PCA projection,
// zeb_project_f32) instead of each pattern's best
template <bool PROJECT>
__global__ void __launch_bounds__(256) k_match_f32(const float* __restrict__ x, int n_exp, const float* __restrict__ d,
                                                   int n_dict, int cols, int per, int slices, float* cand_v,
                                                   int* cand_i, float* out = nullptr) {
  __shared__ float xs[MF_BK][MF_BM + 4];
  __shared__ float ds[MF_BK][MF_BN + 4];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;  // entry group (8 entries), pattern group (4 patterns)
  const int p0 = blockIdx.x * MF_BM;
  const int slice = blockIdx.y;
  const int ntiles = (n_dict + MF_BN - 1) / MF_BN;
  const int t0 = slice * per, t1 = min(ntiles, t0 + per);
  float bv[4];
  int bi[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) { bv[i] = -3.4e38f; bi[i] = -1; }
  for (int t = t0; t < t1; ++t) {
    const int e0 = t * MF_BN;
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
    for (int k0 = 0; k0 < cols; k0 += MF_BK) {
      // 64 × 16 pattern values and 128 × 16 entry values, transposed into shared memory
      for (int u = tid; u < MF_BM * MF_BK; u += 256) {
        const int r = u / MF_BK, k = u - r * MF_BK;
        const int p = p0 + r, kk = k0 + k;
        xs[k][r] = (p < n_exp && kk < cols) ? __ldg(x + (size_t)p * cols + kk) : 0.f;
      }
      for (int u = tid; u < MF_BN * MF_BK; u += 256) {
        const int r = u / MF_BK, k = u - r * MF_BK;
        const int e = e0 + r, kk = k0 + k;
        ds[k][r] = (e < n_dict && kk < cols) ? __ldg(d + (size_t)e * cols + kk) : 0.f;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < MF_BK; ++k) {
        float xv[4], dv[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) xv[i] = xs[k][ty * 4 + i];
#pragma unroll
        for (int j = 0; j < 8; ++j) dv[j] = ds[k][tx * 8 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(xv[i], dv[j], acc[i][j]);
      }
      __syncthreads();
    }
    if constexpr (PROJECT) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int p = p0 + ty * 4 + i;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int e = e0 + tx * 8 + j;
          if (p < n_exp && e < n_dict) out[(size_t)p * n_dict + e] = acc[i][j];
        }
      }
      continue;
    }
    // each pattern's best of this tile: over the thread's 8 entries, then across the 16 threads
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float v = -3.4e38f;
      int id = -1;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int e = e0 + tx * 8 + j;
        if (e < n_dict && acc[i][j] > v) { v = acc[i][j]; id = e; }
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, id, o);
        if (oi >= 0 && (ov > v || (ov == v && (id < 0 || oi < id)))) { v = ov; id = oi; }
      }
      if (id >= 0 && v > bv[i]) { bv[i] = v; bi[i] = id; }
    }
  }
  if (PROJECT) return;
  if (tx == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int p = p0 + ty * 4 + i;
      if (p < n_exp) {
        cand_v[(size_t)p * slices + slice] = bv[i];
        cand_i[(size_t)p * slices + slice] = bi[i];
      }
    }
  }
}

// ── candidates scored again in FP32 ──

__global__ void k_match_best(const float* __restrict__ x, int n_exp, const float* __restrict__ d, int n_dict,
                             int cols, const int* __restrict__ cand, int n_cand, const float4* __restrict__ dict_q,
                             float* __restrict__ seeds) {
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (p >= n_exp) return;
  const float* xp = x + (size_t)p * cols;
  float best = -3.4e38f;
  int bi = -1;
  for (int c = 0; c < n_cand; ++c) {
    const int id = __ldg(cand + (size_t)p * n_cand + c);
    if (id < 0 || id >= n_dict) continue;
    const float* dp = d + (size_t)id * cols;
    float s = 0.f;
    for (int k = lane; k < cols; k += 32) s = fmaf(__ldg(xp + k), __ldg(dp + k), s);
    s = warp_sum(s);
    if (bi < 0 || s > best || (s == best && id < bi)) { best = s; bi = id; }
  }
  if (lane == 0) {
    float* o = seeds + (size_t)p * 8;
    const float4 q = bi >= 0 ? __ldg(dict_q + bi) : make_float4(1.f, 0.f, 0.f, 0.f);
    o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
    o[4] = bi >= 0 ? best : -2.f;
    o[5] = (float)bi;
    o[6] = 0.f;
    o[7] = 0.f;
  }
}

}  // namespace zeb

using namespace zeb;

static int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

extern "C" size_t zeb_panel_bytes(int rows, int cols) {
  if (rows <= 0 || cols <= 0) return 0;
  return (size_t)panel_kblocks(cols) * panel_rows(rows) * 128;
}

extern "C" int zeb_pack_panel(const float* src, int rows, int cols, int ld, void* panel, void* stream) {
  ZEB_REQUIRE(src && panel && rows > 0 && cols > 0 && ld >= cols, ZEB_EARG, "pack_panel: bad arguments");
  ZEB_REQUIRE(((uintptr_t)panel & 15) == 0, ZEB_EARG, "pack_panel: panel must be 16-byte aligned");
  const int rp = panel_rows(rows), kb = panel_kblocks(cols);
  const long long chunks = (long long)kb * rp * 8;
  k_pack_panel<<<(unsigned)((chunks + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, rows, cols, ld, rp, kb,
                                                                                  (uint8_t*)panel);
  return zeb_launch_check("pack_panel");
}

extern "C" int zeb_dict_sims(const zeb_frame_t* fr, const float* vpair, int side, const float t0[3],
                             const float* dict_q, int n, float* out, void* stream) {
  ZEB_REQUIRE(fr && vpair && t0 && dict_q && out && side >= 2, ZEB_EARG, "dict_sims: bad arguments");
  ZEB_REQUIRE(((uintptr_t)vpair & 7) == 0 && ((uintptr_t)dict_q & 15) == 0, ZEB_EARG,
              "dict_sims: vpair must be 8-byte and dict_q 16-byte aligned");
  const long long hw = (long long)fr->h * fr->w;
  ZEB_REQUIRE(hw > 0 && hw * 4 <= 200 * 1024, ZEB_EARG, "dict_sims: %lld pixels per pattern (at most 51200)", hw);
  if (n <= 0) return ZEB_OK;
  SimArgs a;
  a.h = fr->h; a.w = fr->w;
  a.c0 = make_float3(fr->c0[0], fr->c0[1], fr->c0[2]);
  a.c1 = make_float3(fr->c1[0], fr->c1[1], fr->c1[2]);
  a.t0 = make_float3(t0[0], t0[1], t0[2]);
  for (int k = 0; k < 3; ++k) a.mask[k] = fr->mask[k];
  a.vpair = (const float2*)vpair;
  a.side = side;
  a.q = (const float4*)dict_q;
  a.out = out;
  const size_t smem = (size_t)hw * 4;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_dict_sims, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_dict_sims<<<n, 256, smem, (cudaStream_t)stream>>>(a);
  return zeb_launch_check("dict_sims");
}

extern "C" int zeb_match_slices(int n_exp, int n_dict, int cols, int form) {
  if (n_exp <= 0 || n_dict <= 0 || cols <= 0) return 1;
  const int sms = sm_count();
  const int mtiles = form ? (n_exp + MT_BM - 1) / MT_BM : (n_exp + MF_BM - 1) / MF_BM;
  const int ntiles = form ? (n_dict + MT_BN - 1) / MT_BN : (n_dict + MF_BN - 1) / MF_BN;
  const int want = form ? sms : 4 * sms;  // resident CTAs: one per SM (tensor cores), about four (FP32)
  int slices = std::max(1, (want + mtiles - 1) / mtiles);
  // a slice is a band of the dictionary that every pattern tile reads in turn (the pattern tiles
  // run fastest in the grid): at most ~48 MB of it, so that the band stays in L2 while a wave of
  // CTAs streams it
  const long long tile_bytes = form ? (long long)panel_kblocks(cols) * MT_B_BLOCK : (long long)MF_BN * cols * 4;
  const long long band = 48LL << 20;
  slices = std::max<long long>(slices, ((long long)ntiles * tile_bytes + band - 1) / band);
  slices = std::min(ntiles, slices);
  const int per = (ntiles + slices - 1) / slices;
  return (ntiles + per - 1) / per;
}

extern "C" int zeb_match_bf16(const void* x_panel, int n_exp, const void* d_panel, int n_dict, int cols, int slices,
                              float* cand_v, int* cand_i, int* status, void* stream) {
  ZEB_REQUIRE(x_panel && d_panel && cand_v && cand_i && status && cols > 0, ZEB_EARG, "match_bf16: bad arguments");
  ZEB_REQUIRE(((uintptr_t)x_panel & 127) == 0 && ((uintptr_t)d_panel & 127) == 0, ZEB_EARG,
              "match_bf16: panels must be 128-byte aligned");
  if (n_exp <= 0 || n_dict <= 0) return ZEB_OK;
  const int ntiles = (n_dict + MT_BN - 1) / MT_BN;
  ZEB_REQUIRE(slices >= 1 && slices <= ntiles, ZEB_EARG, "match_bf16: %d slices of %d dictionary tiles", slices, ntiles);
  MatchArgs a{};
  a.A = (const uint8_t*)x_panel;
  a.B = (const uint8_t*)d_panel;
  a.rows_a = panel_rows(n_exp);
  a.rows_b = panel_rows(n_dict);
  a.kb = panel_kblocks(cols);
  a.n_exp = n_exp;
  a.n_dict = n_dict;
  a.per = (ntiles + slices - 1) / slices;
  a.slices = slices;
  a.cand_v = cand_v;
  a.cand_i = cand_i;
  a.status = status;
  a.stall = test_stall_ns();
  a.limit = a.stall > 0 ? a.stall : kWaitNs;
  // every candidate reads as "none" until the kernel writes it (a CTA that gave up writes nothing)
  cudaMemsetAsync(cand_i, 0xFF, (size_t)n_exp * slices * MT_TOP * sizeof(int), (cudaStream_t)stream);
  const size_t smem = sizeof(MatchShared) + 1024;
  cudaFuncSetAttribute(k_match_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((n_exp + MT_BM - 1) / MT_BM, slices);
  k_match_tc<false><<<g, MT_THREADS, smem, (cudaStream_t)stream>>>(a);
  return zeb_launch_check("match_bf16");
}

extern "C" size_t zeb_panel_split_bytes(int rows, int cols) {
  if (rows <= 0 || cols <= 0) return 0;
  return 3 * (size_t)panel_kblocks(cols) * panel_rows(rows) * 128;
}

extern "C" int zeb_pack_panel_split(const float* src, int rows, int cols, int ld, int role, void* panel, void* stream) {
  ZEB_REQUIRE(src && panel && rows > 0 && cols > 0 && ld >= cols && (role == 0 || role == 1), ZEB_EARG,
              "pack_panel_split: bad arguments");
  ZEB_REQUIRE(((uintptr_t)panel & 127) == 0, ZEB_EARG, "pack_panel_split: panel must be 128-byte aligned");
  const int rp = panel_rows(rows), kb = panel_kblocks(cols);
  const long long chunks = 3LL * kb * rp * 8;
  k_pack_panel_split<<<(unsigned)((chunks + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, rows, cols, ld, rp, kb,
                                                                                        role, (uint8_t*)panel);
  return zeb_launch_check("pack_panel_split");
}

extern "C" int zeb_project_bf16(const void* x_split, int n_exp, const void* w_split, int k, int cols, float* out,
                                int* status, void* stream) {
  ZEB_REQUIRE(x_split && w_split && out && status && cols > 0 && k > 0, ZEB_EARG, "project_bf16: bad arguments");
  ZEB_REQUIRE(((uintptr_t)x_split & 127) == 0 && ((uintptr_t)w_split & 127) == 0 && ((uintptr_t)out & 15) == 0,
              ZEB_EARG, "project_bf16: panels must be 128-byte and out 16-byte aligned");
  if (n_exp <= 0) return ZEB_OK;
  const int ntiles = (k + MT_BN - 1) / MT_BN;
  MatchArgs a{};
  a.A = (const uint8_t*)x_split;
  a.B = (const uint8_t*)w_split;
  a.rows_a = panel_rows(n_exp);
  a.rows_b = panel_rows(k);
  a.kb = 3 * panel_kblocks(cols);  // the three segments: hi·hi + hi·lo + lo·hi
  a.n_exp = n_exp;
  a.n_dict = k;
  a.per = 1;  // a CTA per (pattern tile, tile of components)
  a.slices = ntiles;
  a.out = out;
  a.status = status;
  a.stall = test_stall_ns();
  a.limit = a.stall > 0 ? a.stall : kWaitNs;
  const size_t smem = sizeof(MatchShared) + 1024;
  cudaFuncSetAttribute(k_match_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((n_exp + MT_BM - 1) / MT_BM, ntiles);
  k_match_tc<true><<<g, MT_THREADS, smem, (cudaStream_t)stream>>>(a);
  return zeb_launch_check("project_bf16");
}

extern "C" int zeb_match_f32(const float* x, int n_exp, const float* d, int n_dict, int cols, int slices,
                             float* cand_v, int* cand_i, void* stream) {
  ZEB_REQUIRE(x && d && cand_v && cand_i && cols > 0, ZEB_EARG, "match_f32: bad arguments");
  if (n_exp <= 0 || n_dict <= 0) return ZEB_OK;
  const int ntiles = (n_dict + MF_BN - 1) / MF_BN;
  ZEB_REQUIRE(slices >= 1 && slices <= ntiles, ZEB_EARG, "match_f32: %d slices of %d dictionary tiles", slices, ntiles);
  const int per = (ntiles + slices - 1) / slices;
  dim3 g((n_exp + MF_BM - 1) / MF_BM, slices);
  k_match_f32<false><<<g, 256, 0, (cudaStream_t)stream>>>(x, n_exp, d, n_dict, cols, per, slices, cand_v, cand_i);
  return zeb_launch_check("match_f32");
}

extern "C" int zeb_project_f32(const float* x, int n_exp, const float* w, int k, int cols, float* out, void* stream) {
  ZEB_REQUIRE(x && w && out && cols > 0 && k > 0, ZEB_EARG, "project_f32: bad arguments");
  if (n_exp <= 0) return ZEB_OK;
  const int ntiles = (k + MF_BN - 1) / MF_BN;
  dim3 g((n_exp + MF_BM - 1) / MF_BM, ntiles);
  k_match_f32<true><<<g, 256, 0, (cudaStream_t)stream>>>(x, n_exp, w, k, cols, 1, ntiles, nullptr, nullptr, out);
  return zeb_launch_check("project_f32");
}

extern "C" int zeb_match_best(const float* x, int n_exp, const float* d, int n_dict, int cols, const int* cand,
                              int n_cand, const float* dict_q, float* seeds, void* stream) {
  ZEB_REQUIRE(x && d && cand && dict_q && seeds && cols > 0 && n_cand >= 1, ZEB_EARG, "match_best: bad arguments");
  ZEB_REQUIRE(((uintptr_t)dict_q & 15) == 0, ZEB_EARG, "match_best: dict_q must be 16-byte aligned");
  if (n_exp <= 0) return ZEB_OK;
  k_match_best<<<(n_exp + 7) / 8, 256, 0, (cudaStream_t)stream>>>(x, n_exp, d, n_dict, cols, cand, n_cand,
                                                                 (const float4*)dict_q, seeds);
  return zeb_launch_check("match_best");
}
