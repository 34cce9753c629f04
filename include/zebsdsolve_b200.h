/*
 * zebsdsolve_b200 — C ABI of the B200 (sm_100a) kernels of zebsdsolve's spherical
 * cross-correlation indexing path.
 *
 * Every entry point takes device pointers, plain sizes and a CUDA stream (cudaStream_t passed as
 * void*; NULL is the legacy default stream), enqueues its kernels and returns without waiting.
 * Return value: 0 on success, a negative ZEB_E* code on failure; zeb_error() then gives the
 * message (per thread, cleared by reading).  No entry point allocates device memory: the caller
 * owns every buffer, scratch included, and sizes it with the zeb_*_bytes helpers.
 *
 * The entry points replace the reference's GPU schedule functions (zebsdsolve 0.2.8, Zig +
 * WGSL), which record WGSL dispatches through its WebGPU layer; the file:line cited beside each
 * is the reference function it stands in for.  The reference's Python/C front end (ze.index,
 * ze.Solver, the ze_* engine calls) is mirrored one level up by the Python package
 * zebsdsolve_b200, which drives these entry points.
 */
#ifndef ZEBSDSOLVE_B200_H
#define ZEBSDSOLVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZEB_OK 0
#define ZEB_EARG (-1)   /* an argument is out of range or a pointer is missing */
#define ZEB_ECUDA (-2)  /* a CUDA launch or call failed */
#define ZEB_ESIZE (-3)  /* a size beyond what the kernels support */

/* Message of the last failure on this thread (cleared by the call); returns its length. */
size_t zeb_error(char* buf, size_t cap);
/* The library's version string: the reference version it is a drop-in for ("0.2.8"). */
const char* zeb_version(void);

/* ── tables in FP64 on the device ──────────────────────────────────────────────────────── */

/* Gauss–Legendre nodes x (descending) and weights w of order n.
 * Replaces sh.gaussLegendre (src/sh.zig:31-72). */
int zeb_gauss_legendre(int n, double* x, double* w, void* stream);

/* Normalized associated Legendre P̄_l^m(x_i) for every pair below L, plm[i][pair(m,l)].
 * Replaces sh.legendreAll (src/sh.zig:75-99) over a grid's rings (sh.Grid.init, sh.zig:111-125). */
int zeb_legendre_table(int L, int n_x, const double* x, double* plm, void* stream);

/* Wigner d^l_{k,m}(π/2) for 0 ≤ k, m, l < L at d[(k·L + m)·L + l] (zero for l < max(k,m)) by
 * the Jacobi three-term recursion. Replaces sh.wignerHalfPi (src/sh.zig:239-280). */
int zeb_wigner_half_pi(int L, double* d, void* stream);

/* ── the detector frame ─────────────────────────────────────────────────────────────────── */

typedef struct {
  int32_t h, w;       /* pattern rows, columns (pixels of the level being worked on) */
  float c0[3];        /* detector row direction in the sample frame */
  float c1[3];        /* detector column direction */
  float c2[3];        /* detector normal */
  float mask[3];      /* mask centre (row, col) and squared radius in pixels (≤ 0: none) */
} zeb_frame_t;        /* spherical.Frame (src/spherical.zig:81-90) */

/* ── preprocessing ──────────────────────────────────────────────────────────────────────── */

/* Unpack n stored patterns of h × w (pixel: 0 u8, 1 u16, 2 f32), subtract the static background
 * (h·w floats, or NULL), subtract (dynamic = 1) or divide by (2) a Gaussian blur of deviation
 * sigma pixels (0: none), then zero mean and unit norm under the mask (zero outside).
 * Replaces Prep.run / Prep.filter without CLAHE and band pass (src/prep.zig:143-204,263-272;
 * shaders/prep.wgsl load, background, blur_rows/cols, the wide blur, combine, normalize). */
int zeb_prep(const void* raw, int pixel, int n, int h, int w, const float* static_bg, int dynamic,
             float sigma, const float mask[3], int normalize, float* out, void* stream);
/* Device scratch bytes zeb_prep needs for a wide blur (sigma ≥ 12 pixels); 0 otherwise. */
size_t zeb_prep_scratch_bytes(int n, int h, int w, float sigma);
int zeb_prep_ex(const void* raw, int pixel, int n, int h, int w, const float* static_bg, int dynamic,
                float sigma, const float mask[3], int normalize, float* out, void* scratch, void* stream);
/* zeb_prep_ex on patterns stored at src_h × src_w and reduced by `factor` (settings.binning, 1 to
 * 64) as they are unpacked: a whole factor is the k × k blocks' means, any other the source area
 * each output pixel covers (area resampling); the output is floor(size / factor) each way, the
 * remainder dropped. static_bg, mask, sigma and out are at the reduced size. Replaces the host
 * reduction of reduce.zig:44-131 (which the reference runs on the CPU before the upload). */
int zeb_prep_reduced(const void* raw, int pixel, int n, int src_h, int src_w, double factor, const float* static_bg,
                     int dynamic, float sigma, const float mask[3], int normalize, float* out, void* scratch,
                     void* stream);

/* dynamic = 3 in the zeb_prep entries: the output is the Gaussian blur itself (the band pass's
 * two Gaussians; prep.zig:190-200). */

/* Contrast-limited adaptive histogram equalization of n images of h × w in place: each stretched
 * to [0, 1], padded by reflection to tiles × tiles whole tiles, each tile's histogram of `bins`
 * levels clipped at clip × the mean count per level and redistributed, the pixel read from the
 * four nearest tiles' tables between its two nearest levels. scratch: zeb_clahe_scratch_bytes.
 * Replaces Prep.filter's CLAHE (src/prep.zig:167-188; shaders/prep.wgsl stretch, clahe_hist,
 * clahe_cdf, clahe_apply). */
size_t zeb_clahe_scratch_bytes(int n, int tiles, int bins);
int zeb_clahe(float* img, int n, int h, int w, int tiles, int bins, float clip, void* scratch, void* stream);

/* out = a − b (op 0) or a / max(b, 1e-6) (op 1), elementwise over count floats. Replaces
 * combine (shaders/prep.wgsl; the band pass's difference, src/prep.zig:190-200). */
int zeb_combine(const float* a, const float* b, float* out, long long count, int op, void* stream);

/* Non-local pattern averaging (NLPAR; Brewick, Wright and Rowenhorst 2019) of a window of loaded
 * patterns (px floats each, f32, in the window's order: the wanted cells first, then ring after
 * ring around them; counts[d] (host, radius·passes + 2 entries) cells lie within d rings): passes
 * of weighted means over (2·radius + 1)² neighbours, each weight from the pair's mean squared
 * difference against the noise the pair's shares of the stored patterns give. nbr (device,
 * [n_win][(2·radius·passes + 1)²] rows first, 0xffffffff outside the map) lists each cell's
 * neighbours. Writes the counts[0] averages to out; `patterns` is working space (clobbered when
 * passes ≥ 3). sig_out (counts[rings − 1] floats) and shares_out (counts[0] × F) take the noise and
 * the final shares when not NULL. Replaces Nlpar.average (src/nlpar.zig:89-138; shaders/nlpar.wgsl
 * distance, sigma, weights, average, shares). */
size_t zeb_nlpar_scratch_bytes(int n_win, int px, int radius, int passes);
int zeb_nlpar(float* patterns, int px, const uint32_t* nbr, const int* counts, int radius, int passes, float lambda,
              float* out, float* sig_out, float* shares_out, void* scratch, void* stream);

/* ── the master on the sphere ───────────────────────────────────────────────────────────── */

/* The master's mean over its point group: dst at each sheet pixel's direction d is the mean of
 * src (bilinear) at g·d over the n_ops operators (ops: 3 × 3 row-major each). Replaces
 * Prep.symmetrize (src/prep.zig:240-249; shaders/mastersph.wgsl symmetrize 111-122). */
int zeb_master_symmetrize(const float* src, float* dst, int side, const float* ops, int n_ops, void* stream);

/* One pass of Gaussian smoothing on the sphere over a (2·radius+1)² tangent lattice of step
 * `step` radians with weights exp(−(a²+b²)·k). Replaces the sphere_blur pass of Prep.sphereBlur
 * (src/prep.zig:215-237; shaders/mastersph.wgsl:87-109). */
int zeb_master_blur_pass(const float* src, float* dst, int side, float step, float k, int radius, void* stream);

/* The master's tangent gradient with its value: grad4[i] = (∇M.xyz, M) at every sheet pixel.
 * Replaces Prep.gradient (src/prep.zig:253-260; shaders/mastersph.wgsl:124-138). */
int zeb_master_gradient(const float* sheets, float* grad4, int side, void* stream);

/* The sheets and the gradient table with each pixel's right-hand neighbour beside it:
 * vpair[i] = (M[i], M[i+1]) (2 floats), gpair[i] = (grad4[i], grad4[i+1]) (8 floats, 32-byte
 * records), [2][side][side] each. The detector kernels read these so that a bilinear lookup takes
 * one record per row. No counterpart in the reference (its lookups read the four texels). */
int zeb_master_pairs(const float* sheets, const float* grad4, int side, float* vpair, float* gpair, void* stream);

/* The master sampled (bilinear, FP64 arithmetic on the FP32 sheets) at every point of a
 * Gauss–Legendre grid of n_theta rings (cos θ in x) and n_phi points per ring: out[ring][j].
 * Replaces the sampling loop of master.Harmonics.init (src/master.zig:680-688). */
int zeb_master_sample_grid(const float* sheets, int side, const double* x, int n_theta, int n_phi,
                           double* out, void* stream);

/* ── (a) patterns → spherical-harmonic coefficients ─────────────────────────────────────── */

typedef struct {
  int32_t L, n_theta, n_phi, n_pairs;
  const float* ring;    /* [n_theta][4]: cos θ, sin θ, quadrature weight, 0 */
  const float* phi_cs;  /* [n_phi][2]: cos φ_j, sin φ_j */
  const float* wplm;    /* [n_theta/2][n_pairs]: w_y · P̄(cos θ_y) · 2π/n_phi */
  const float* tw;      /* [1024][2]: e^{−2πi t/1024} */
} zeb_sphere_tables_t;  /* spherical.Tables (src/spherical.zig:106-180) */

#define ZEB_FLAG_CENTER 1u
#define ZEB_FLAG_NORM 2u
#define ZEB_FLAG_WINDOW 4u

/* Scratch bytes for n_items items at these tables. */
size_t zeb_sphere_scratch_bytes(const zeb_sphere_tables_t* tb, int n_items);

/* Each item (items[b] = t.x, t.y, t.z in pixels, pattern index) sampled on the sphere, window-
 * mean centred (ZEB_FLAG_CENTER), analysed into alm[b][pair][re,im] and scaled to unit norm
 * (ZEB_FLAG_NORM); ZEB_FLAG_WINDOW projects the window itself. stats[b] = (window area,
 * window mean, harmonic norm, a_00). Replaces Spherical.coefficients
 * (src/spherical.zig:319-361; shaders/sphere.wgsl sphere_sums, rings, legendre, sh_norm). */
int zeb_sphere_coefficients(const float* pats, const float* items, int n_items, const zeb_frame_t* fr,
                            const zeb_sphere_tables_t* tb, unsigned flags, float* alm, float* stats,
                            void* scratch, void* stream);

/* The same, sampling each ring only over its span (zeb_sphere_spans): spans[2y], spans[2y+1] =
 * first φ sample and count (cyclic) of ring y. A ring whose span's end samples meet the detector
 * for an item is sampled whole for that item, so the result is that of full sampling whatever
 * the spans; spans NULL samples everything. Replaces Spherical.coefficients as above. */
int zeb_sphere_coefficients_spans(const float* pats, const float* items, int n_items, const zeb_frame_t* fr,
                                  const zeb_sphere_tables_t* tb, const int* spans, unsigned flags, float* alm,
                                  float* stats, void* scratch, void* stream);

/* Ring spans for the detector positions ts[k] (float4 t.x, t.y, t.z, unused; n_t <= 64): per ring
 * the shortest cyclic run of φ samples holding every sample on the masked detector for any of
 * them, widened by `margin` samples each side. spans: device int[n_theta][2]. No counterpart in
 * the reference (which samples every direction): the sampling work of the rings drops to the
 * detector's footprint. */
int zeb_sphere_spans(const zeb_frame_t* fr, const zeb_sphere_tables_t* tb, const float* ts, int n_t, int margin,
                     int* spans, void* stream);

/* ── (b) the SO(3) correlation ──────────────────────────────────────────────────────────── */

typedef struct {
  int32_t L, n, nb, nc, fold, mu_max, n_pairs;
} zeb_so3_dims_t;  /* spherical.PhaseGpu + Tables sizes (src/spherical.zig:192-242) */

/* The master's correlation table for one phase at one bandwidth, in FP64 on the device:
 * Y[pair(m',l)][j·nc + c] = Σ_μ e^{−2πi μ c/nc} i^{m'} Σ_k d^l_{k,m'} W[μ,l,k] β_{±}(k, j), the
 * Wigner-d contraction with the master's weights W (master.weights, src/master.zig:727-753) and
 * the transforms along b (so3.wgsl spectrum, :147-277; β_+ = 2cos(k b_j), β_− = −2i sin, by the
 * parity of m'+m; k = 0 once) and along c (so3.wgsl:396-430, m = fold·μ at the nc grid points
 * c) folded in, so that the spectrum U of an item is already transformed along b and c.
 * W is [mc][L][L] complex (re, im) FP64. */
int zeb_correlation_table(const zeb_so3_dims_t* d, const double* W, const double* wigner, double* Y, void* stream);

/* U[b][j][m'][c] = Σ_l conj(g_b[l,m']) Y[pair(m',l)][j·nc+c]: the spectrum of every item,
 * transformed along b and c, in plain FP32 (CUDA cores). alm as zeb_sphere_coefficients leaves it; Y in FP32.
 * Replaces Spherical.spectrum (src/spherical.zig:369-382; shaders/so3.wgsl spectrum). */
int zeb_spectrum_f32(const float* alm, int n_items, const zeb_so3_dims_t* d, const float* Y, float* U, void* stream);

/* Bytes of U for n_items items. */
size_t zeb_spectrum_bytes(const zeb_so3_dims_t* d, int n_items);

/* The same U on the tcgen05 tensor cores (the BF16 form): BF16 operands, FP32 accumulation in
 * tensor memory.  Every operand is split x = hi + lo into two BF16 values; for l <= split the
 * product keeps hi*hi + hi*lo + lo*hi (near FP32), above it hi*hi (2^-9 relative per operand);
 * split = -1: hi*hi everywhere, split >= L-1: the split product everywhere.
 * A is the master's table packed once per phase and split by zeb_tc_pack_master from the FP64 Y
 * of zeb_correlation_table (zeb_tc_master_bytes bytes); B is scratch of
 * zeb_tc_patterns_bytes(d, split, n_items) bytes that this call packs from alm.  status (one
 * int, zeroed by the caller) is left nonzero if a wait inside the kernel timed out (the kernel
 * then returns early and U is incomplete).  Supported while K of order 0,
 * 2L + 4(min(split, L-1) + 1), is at most 384 (L <= 64 with every order split; L <= 160 with none).
 * Replaces Spherical.spectrum (src/spherical.zig:369-382; shaders/so3.wgsl spectrum). */
int zeb_spectrum_bf16(const float* alm, int n_items, const zeb_so3_dims_t* d, int split, const void* A, void* B,
                      float* U, int* status, void* stream);
int zeb_tc_pack_master(const zeb_so3_dims_t* d, int split, const double* Y, void* A, void* stream);
/* Bytes of A, and of B for n_items items (0 for unsupported dims). */
size_t zeb_tc_master_bytes(const zeb_so3_dims_t* d, int split);
size_t zeb_tc_patterns_bytes(const zeb_so3_dims_t* d, int split, int n_items);

/* The BF16 form's spectrum kept in FP16 (half the bytes of U): zeb_spectrum_bf16's GEMM, its
 * accumulators scaled by `scale` and rounded to FP16 as they drain, stored as
 * U16[item / 128][j·nc + c][m'][re|im][item % 128] with the items padded to a multiple of 128
 * (zeb_spectrum_h_bytes bytes; U16 128-byte aligned). `scale` is a power of two with
 * scale·max|U| well inside FP16's range: the host takes it from the table, as 2^floor(log2(16384 /
 * y)) with y the largest column norm over l of any order's table (|U| <= y since the coefficients
 * have unit norm). Same A, B, split and status as zeb_spectrum_bf16; needs 2·nb·nc >= 128.
 * Replaces Spherical.spectrum (src/spherical.zig:369-382; shaders/so3.wgsl spectrum). */
size_t zeb_spectrum_h_bytes(const zeb_so3_dims_t* d, int n_items);
int zeb_spectrum_bf16_h(const float* alm, int n_items, const zeb_so3_dims_t* d, int split, const void* A, void* B,
                        void* U16, float scale, int* status, void* stream);

/* zeb_correlate_peaks over U16 (zeb_spectrum_bf16_h, the same `scale`), the transform along a on
 * the tcgen05 tensor cores: per (j, c) one GEMM of 128 items × n values of a × 2L (m', re|im),
 * FP16 operands (the transform matrix f_m'·cos / f_m'·sin of 2π m'a/n built on the device), FP32
 * accumulation in tensor memory, each value times rden (one volume shared by every item) and
 * each (item, j) slab's largest kept as the drain runs; then the vertex from direct sums over m'
 * at the peak and its six neighbours (the peak's score from the same sum). Supports 16 <= L <= 64
 * with n = 2L. scratch: zeb_peaks_scratch_bytes; status as zeb_spectrum_bf16 (a timed-out wait).
 * Replaces Spherical.correlate's a_peak_m, peak_reduce and peak_finish_m (src/spherical.zig:
 * 401-432; shaders/so3.wgsl :489-593, 631-663, 716-796). */
int zeb_correlate_peaks_h(const void* U16, int n_items, const zeb_so3_dims_t* d, float scale, const float* rden,
                          float* peaks, void* scratch, int* status, void* stream);

/* The correlation volume's transform along a (U comes transformed along b and c), times rden
 * (volume b / rden_div for item b), each (item, j, c) line's largest value, each item's largest, and its sub-grid vertex and
 * orientation: peaks[b] = (q.w, q.x, q.y, q.z, score, a, b, c). Replaces Spherical.correlate's
 * a_peak_m, peak_reduce and peak_finish_m (src/spherical.zig:401-432; shaders/so3.wgsl
 * :489-593, 631-663, 716-796). scratch: zeb_peaks_scratch_bytes. */
size_t zeb_peaks_scratch_bytes(const zeb_so3_dims_t* d, int n_items);
int zeb_correlate_peaks(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw, const float* rden,
                        int rden_div, float* peaks, void* scratch, void* stream);

/* zeb_correlate_peaks without caller scratch — this entry point has no counterpart in the
 * reference. It is for callers that cannot call cudaMalloc: hosts that reserve their device
 * memory once at start-up and forbid allocation afterwards (an allocator owns the rest of the
 * GPU), and latency-bound loops that must not let an allocation call synchronize the device.
 * The candidates' scratch is a file-scope __device__ array of ZEB_PEAKS_STATIC_SLABS (item, j)
 * slabs (4 MiB; every GPU that loads the library holds it until the process exits), so one call
 * takes at most ZEB_PEAKS_STATIC_SLABS / nb items (8065 at L = 64); larger calls fail with
 * ZEB_ESIZE and a message. The first call in a CUDA context looks the array's device address up
 * (cudaGetSymbolAddress, with that context current) and keeps it for that context, keyed by the
 * context's unique ID: after a cudaDeviceReset, or with another driver-API context current on the
 * device, the next call is again a first call. Make each context's first call before any stream
 * capture in it. Every call shares the one array and leaves its candidates in it:
 * calls that overlap on the GPU (other streams, other threads) race and must be serialized by
 * the caller. Nothing in it needs to start at zero: each call writes every candidate it reads.
 * Allocates nothing (no cudaMalloc, cudaFree or allocating library routine). */
#define ZEB_PEAKS_STATIC_SLABS (1 << 19)
int zeb_correlate_peaks_static(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw,
                               const float* rden, int rden_div, float* peaks, void* stream);

/* The full volumes (no peak) of n items: vol[b][j][c][ia]. Replaces a_volume
 * (shaders/so3.wgsl:595-612). */
int zeb_correlate_volume(const float* U, int n_items, const zeb_so3_dims_t* d, const float* tw, float* vol, void* stream);

/* rden = 1/sqrt(vol_f2 − vol_f²/area) where above 1e-6·area, else 0; area[b·4] per window.
 * Replaces rden_build (shaders/so3.wgsl:614-626). */
int zeb_rden_build(const float* vol_f, const float* vol_f2, const float* stats, int n, long long cells,
                   float* rden, void* stream);

/* The failure test of the tensor-core kernels (zeb_spectrum_bf16, zeb_spectrum_bf16_h,
 * zeb_correlate_peaks_h, zeb_match_bf16): while ns > 0, each of them launched makes its MMA thread
 * wait first on an mbarrier that nothing arrives at and gives every wait ns nanoseconds, so that the
 * kernel gives up as it would on a real timeout: it sets its status word, waits (up to 1 s) for its
 * own copies and MMAs in flight, frees its tensor memory and returns. 0 (the default) turns it off.
 * No counterpart in the reference (its waits are the WebGPU queue's). */
int zeb_set_test_stall(long long ns);

/* ── (c) refinement and scores on the detector ──────────────────────────────────────────── */

typedef struct {
  int32_t iters;        /* Gauss–Newton steps; iters + 1 passes of sums */
  float max_step;       /* largest rotation of one step, radians */
  float scale0, scale_min, scale_max;  /* curvature scale μ: start and bounds */
  int32_t nmi_bins;
  float stamp;          /* written into each record's last slot */
} zeb_refine_opts_t;    /* detector.RefineOptions (src/detector.zig:57-70) */

/* Seed each item with the orientation beginning seeds[b·seed_stride] (spherical peaks or
 * refinement records), refine it on the detector against its pattern (rotation-only
 * Gauss–Newton), score it (NCC, NMI) and write records[b] = (q.w, q.x, q.y, q.z, NCC, NMI,
 * last improving step, stamp). One thread block per item, the pattern resident in shared
 * memory across the passes. Replaces Detector.seed + Detector.refine (src/detector.zig:178-212;
 * shaders/detector.wgsl seed, refine_init, sums_rot, refine_rot_step, nmi, collect). */
int zeb_refine(const float* pats, const float* items, const float* seeds, int seed_stride, int n,
               const zeb_frame_t* fr, const float* vpair, const float* gpair, int side,
               const zeb_refine_opts_t* o, float* records, void* stream);  /* tables: zeb_master_pairs */

/* NMI of each item's pattern against the master at `draws` random orientations (Shoemake from
 * a hash of the item and draw): out[draw][b]. Replaces Detector.chanceOf (src/detector.zig:
 * 216-229; shaders/detector.wgsl decoy, nmi). */
int zeb_chance(const float* pats, const float* items, int n, int draws, const zeb_frame_t* fr,
               const float* vpair, int side, int nmi_bins, float* out, void* stream);  /* vpair: zeb_master_pairs */

/* The records' orientations (records[b][0..3]) in the fundamental zone of a group of n_ops
 * rotations (ops[k] = w, x, y, z, FP64, identity first): fz[b] = the g·q of largest w, unit norm,
 * w >= 0, ties within 1e-12 keeping the first, in FP64 rounded once to FP32. The landing's
 * reduction (engine.zig:2392-2419 with sym.zig:120-131), moved from the host to the device. */
int zeb_records_fz(const float* records, int n, const double* ops, int n_ops, float* fz, void* stream);
/* zeb_records_fz with each reduced orientation's Bunge angles too: bunge[b] = (φ1, Φ, φ2) in radians
 * ([0, 2π), [0, π], [0, 2π)) of the FP32 quaternion fz[b], by the formulas of rot.zig:151-173 in
 * FP64 rounded once to FP32 — the landing's conversion (engine.zig:2392-2419), moved to the device. */
int zeb_records_fz_bunge(const float* records, int n, const double* ops, int n_ops, float* fz, float* bunge,
                         void* stream);

/* Six unknowns per item: x[b] = (δt: the rays' origin moved, 3 floats in pixels, sample axes;
 * φ: a rotation vector applied on the left of q0[b], radians), the detector projection
 * v = c0·row + c1·col + t + δt, c = (exp(φ)·q0)·v/|v| and the normalized cross-correlation of
 * the pattern with the master there. One block per item, the masked pixels listed in shared
 * memory. mode 0: out[b] = NCC (the forward). mode 1: out[b][0..5] = ∂NCC/∂x by the exact
 * derivatives of the forward (the bilinear lookup's slopes through the square-Lambert map, the
 * rotation and the ray's normalization), out[b][6] = NCC: the adjoint, which recomputes the
 * projection. mode 2: out[b][0..42] = the 43 sums of detector.wgsl:435-499 (sums), with the
 * directions from the gradient table gpair (the reference's Gauss–Newton Jacobian), from which
 * planefit.zig:176-200 (localOf) forms NCC, gradient and GN matrix. mode 3: out[b][0..60] =
 * mode 2's 43 sums, then from the same pass mode 1's exact derivatives D' summed as ΣD' (43-48),
 * ΣM·D' (49-54) and Σe·D' (55-60): one pass a round for the adjoint settle (GN matrix from the
 * table, gradient from the adjoint). vpair/gpair: zeb_master_pairs. Replaces Detector's `sums`
 * schedule (src/planefit.zig:523-558 eval). */
int zeb_det6(int mode, const float* pats, const float* items, int n, const zeb_frame_t* fr, const float* vpair,
             const float* gpair, int side, const float* x, const float* q0, float* out, void* stream);

/* x[b] = A[b]⁻¹ b[b] for n systems of 6 (A: [n][6][6], b: [n][6], FP64) by elimination with
 * partial pivoting; ok[b] = 0 where a pivot falls below 1e-300 (x[b] = 0). Replaces the host
 * solve of planefit.zig:203-233 (the damped Levenberg–Marquardt step of settle). */
/* zeb_det6 over the frame's masked-pixel list (zeb_mask_list, npix = zeb_mask_pixels entries, at
 * most 51200): 128 threads per pattern keep only the pattern's values in shared memory and
 * recompute each pixel's ray, so that four or five patterns share an SM; the same outputs. */
int zeb_det6_list(int mode, const float* pats, const float* items, int n, const zeb_frame_t* fr, const uint32_t* list,
                  int npix, const float* vpair, const float* gpair, int side, const float* x, const float* q0,
                  float* out, void* stream);

int zeb_solve6(const double* A, const double* b, int n, double* x, int* ok, void* stream);

/* ── dictionary indexing ────────────────────────────────────────────────────────────────── */

/* The dictionary's entries simulated at detector position t0 (pixels): out[e][h·w] = the master
 * (value pairs of zeb_master_pairs) at dict_q[e]·(c0·row + c1·col + t0)/|…|, then zero mean and
 * unit norm under the mask (zero outside). h·w ≤ 51200. Replaces Detector.dictSims
 * (src/detector.zig:250-260; shaders/detector.wgsl project_dict 266-273, sim_norm 662-699). */
int zeb_dict_sims(const zeb_frame_t* fr, const float* vpair, int side, const float t0[3], const float* dict_q,
                  int n, float* out, void* stream);

/* Bytes of the BF16 operand panel of `rows` rows of `cols` values: ⌈cols/64⌉ blocks of
 * [rows rounded up to 256][128 B], the 16-byte chunks of row r XOR-swizzled by r mod 8. */
size_t zeb_panel_bytes(int rows, int cols);

/* FP32 rows (src[r·ld + k]) rounded to BF16 into a panel; padding rows and columns are zero. */
int zeb_pack_panel(const float* src, int rows, int cols, int ld, void* panel, void* stream);

/* How many dictionary slices the match kernels split the entries into for n_exp patterns of cols
 * values (form 0: FP32, 1: BF16 tensor cores): enough CTAs to fill the GPU, and bands of the
 * dictionary small enough to stay in L2 while the pattern tiles stream them. The candidate
 * buffers hold n_exp × slices (FP32) or n_exp × slices × 8 (BF16) entries. */
int zeb_match_slices(int n_exp, int n_dict, int cols, int form);

/* Per pattern and dictionary slice the eight largest inner products of the pattern's panel row
 * with the dictionary's panel rows (BF16 operands, FP32 accumulation on the tensor cores),
 * descending, equal scores in index order: cand_v/cand_i[p][slice][8] (index −1 where a slice has
 * fewer than eight entries). status gets a nonzero bit when a wait inside the kernel timed out.
 * Replaces the scoring of Detector.dictChunk and Pca.match (src/detector.zig:262-271,
 * src/pca.zig:166-171; shaders/detector.wgsl dict_score 705-740, pca.wgsl nearest 114-168). */
int zeb_match_bf16(const void* x_panel, int n_exp, const void* d_panel, int n_dict, int cols, int slices,
                   float* cand_v, int* cand_i, int* status, void* stream);

/* The same in plain FP32 (CUDA cores) from row-major x[n_exp][cols] and d[n_dict][cols]: per
 * pattern and slice the best entry, ties to the lower index: cand_v/cand_i[p][slice]. */
int zeb_match_f32(const float* x, int n_exp, const float* d, int n_dict, int cols, int slices, float* cand_v,
                  int* cand_i, void* stream);

/* The patterns' coefficients on a PCA's components: out[p][c] = Σ_k x[p][k]·w[c][k] (the batch's
 * projection of Pca.project, src/pca.zig:159-162; shaders/pca.wgsl project). The BF16 form on the
 * tcgen05 tensor cores from split panels (zeb_pack_panel_split: each operand x = hi + lo in BF16,
 * the product hi·hi + hi·lo + lo·hi, near FP32), role 0 for the patterns and 1 for the components
 * (zeb_panel_split_bytes bytes each); status as zeb_match_bf16. The plain FP32 form from row-major
 * x [n_exp][cols] and w [k][cols] on the CUDA cores. out is n_exp × k FP32, 16-byte aligned. */
size_t zeb_panel_split_bytes(int rows, int cols);
int zeb_pack_panel_split(const float* src, int rows, int cols, int ld, int role, void* panel, void* stream);
int zeb_project_bf16(const void* x_split, int n_exp, const void* w_split, int k, int cols, float* out, int* status,
                     void* stream);
int zeb_project_f32(const float* x, int n_exp, const float* w, int k, int cols, float* out, void* stream);

/* Each pattern's n_cand candidate entries scored again in FP32 (x·d over cols; indices outside
 * [0, n_dict) skipped), the best (ties to the lower index) written as a seed: seeds[p] = (dict_q[best] (w, x, y, z), score, best, 0, 0).
 * Replaces Detector.seedDict (src/detector.zig:231-235; shaders/detector.wgsl seed_dict 311-317). */
int zeb_match_best(const float* x, int n_exp, const float* d, int n_dict, int cols, const int* cand, int n_cand,
                   const float* dict_q, float* seeds, void* stream);

/* The number of pixels of an h × w frame inside its circular mask (all of them without one), and
 * their list in raster order, list[k] = (row << 16) | col (zeb_mask_pixels entries). Both use the
 * same test as the kernels (dr² + dc² ≤ r², each product and the sum rounded on its own). */
int zeb_mask_pixels(const zeb_frame_t* fr);
int zeb_mask_list(const zeb_frame_t* fr, uint32_t* list, void* stream);

/* zeb_refine over the frame's pixel list (zeb_mask_list, npix = zeb_mask_pixels entries, at most
 * 25600): a block of 128 threads per item keeps only the pattern's values along the list in shared
 * memory, so that six items share an SM (256 or 512 threads where those values pass 36 or 72 KB, so
 * that an SM keeps about as many warps for a large detector's list). The same records as
 * zeb_refine. */
int zeb_refine_list(const float* pats, const float* items, const float* seeds, int seed_stride, int n,
                    const zeb_frame_t* fr, const uint32_t* list, int npix, const float* vpair, const float* gpair,
                    int side, const zeb_refine_opts_t* o, float* records, void* stream);

/* The BF16 form's refinement table: for every texel of the [2][side][side] sheets its 2 × 2
 * neighbourhood (the texel, the one right of it, the one below, the one below right) in one
 * 32-byte record of FP16 values — per texel (gx, gy) and (gz, master) as two half2 — from the
 * gradient table grad4 of zeb_master_gradient (quads: 32 × 2·side² bytes, 32-byte aligned). No
 * counterpart in the reference (its lookups read the four texels in FP32). */
int zeb_master_quads(const float* grad4, int side, void* quads, void* stream);

/* zeb_refine_list with every lookup of the Gauss–Newton passes from the FP16 records of
 * zeb_master_quads (one 32-byte record a pixel instead of two; the bilinear interpolation in
 * packed FP16, every sum in FP32; the NMI from vpair in FP32 as before). The same records as
 * zeb_refine_list to FP16's rounding of the master's values and gradients and of the
 * interpolation. */
int zeb_refine_list_h(const float* pats, const float* items, const float* seeds, int seed_stride, int n,
                      const zeb_frame_t* fr, const uint32_t* list, int npix, const float* vpair, const void* quads,
                      int side, const zeb_refine_opts_t* o, float* records, void* stream);

/* Simulated patterns: the master at q·ray for every pixel of item b (poses[b] = t.xyz, pattern
 * index, q.wxyz): sims[b][h][w]. Replaces Detector.project (src/detector.zig:138-142;
 * shaders/detector.wgsl:254-263). */
int zeb_project(const float* master, int side, const float* poses, int n, const zeb_frame_t* fr, float* sims,
                void* stream);

/* The 43 Gauss–Newton sums of zeb_det6_list (mode 2) with the master taken by `interp`: 0 the
 * gradient table (gpair, bilinear), 1 bicubic (Catmull–Rom) or 2 Keys' six-point cubic convolution
 * of the sheets themselves (sheets [2][side][side]), each with its own surface's gradient on the
 * sphere. Replaces Detector.sumsOf with settings.plane_interp (src/detector.zig:145-159;
 * shaders/detector.wgsl sums 435-499, grad_at_cubic / grad_at_keys6 146-248). */
int zeb_sums6_list(const float* pats, const float* items, int n, const zeb_frame_t* fr, const uint32_t* list,
                   int npix, const float* sheets, const float* gpair, int side, int interp, const float* x,
                   const float* q0, float* out, void* stream);

/* The pattern-centre vote's density (host function, no GPU): n_ballots ballots at integer
 * candidate coordinates at[b] = (x, y, z) with weights w[b], each spread by a Gaussian of sigma[a]
 * candidate steps along axis a out to ceil(3 sigma) (clipped to the n[0] × n[1] × n[2] grid) and
 * added in float32, ballot by ballot: out[x + n0 (y + n1 z)]. Replaces splat
 * (src/pcfit.zig:210-236). */
int zeb_pc_splat(const int* at, const double* w, int n_ballots, const int* n, const double* sigma, float* out);

#ifdef __cplusplus
}
#endif
#endif
