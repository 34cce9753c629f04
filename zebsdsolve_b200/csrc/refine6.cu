// (c, config 3) Six unknowns per pattern: the source's shift (the rays' origin, pixels in the
// sample's axes) and the crystal's rotation, and the score they give: the normalized cross-
// correlation of the pattern with the master projected through them.
//
// k_det6<MODE>: one block per pattern. The masked pixels are listed once per block as (row, col,
// pattern value) in shared memory; with the pattern's parameters x = (δt, φ) the block projects
// every listed pixel, v = c0·row + c1·col + t + δt, c = (exp(φ)·q0)·v/|v| (the frame turned by the
// rotation once a block), and sums over the pixels:
//   MODE 0 (forward): n, ΣM, ΣM², ΣM·e → the NCC;
//   MODE 1 (adjoint): with the exact derivatives D = ∂M/∂x of the forward — the bilinear
//     lookup's slopes in the sheet, through the square-Lambert map's Jacobian, the rotation and
//     the normalization of the ray — also ΣD, ΣM·D, Σe·D → ∂NCC/∂x (the projection is recomputed,
//     nothing of the forward is stored);
//   MODE 2 (the reference's Gauss–Newton sums, detector.wgsl:435-499): with D from the master's
//     gradient table instead (q⁻¹·∇M/|v|, c × ∇M), all 43 sums (n, ΣM, ΣM², ΣM·e, ΣD, ΣM·D, Σe·D,
//     ΣDᵢDⱼ) from which planefit.zig:176-200 forms the NCC, its gradient and its GN matrix.
//   MODE 3 (the adjoint settle's one pass a round): MODE 2's 43 sums and, from the same ray and
//     rotation, MODE 1's exact derivatives D' with their ΣD', ΣM·D', Σe·D' (61 sums): the GN
//     matrix from the table and the gradient from the adjoint, as two passes would give them.
// k_solve6: a damped 6 × 6 system per pattern in FP64 by elimination with partial pivoting
// (planefit.zig:203-248).
#include "abi_util.cuh"

namespace zeb {

struct Det6Args {
  const float* pats;
  const float4* items;
  int n, h, w;
  float3 c0, c1, c2;
  float mask[3];
  const float2* vpair;
  const float* gpair;
  int side;
  const float* x;   // [n][6]: δt (3, pixels), φ (3, radians)
  const float* q0;  // [n][4] (w, x, y, z)
  float* out;       // MODE 0: [n]; MODE 1: [n][7] (∂NCC/∂x, NCC); MODE 2: [n][43]; MODE 3: [n][61]
  const float* sheets;  // MODE 2 with interp 1 or 2: the master's two sheets [2][side][side]
  int interp;           // MODE 2: 0 the gradient table (bilinear), 1 bicubic, 2 Keys' six-point
};

// ── the master sampled by a smooth kernel, with that surface's own gradient on the sphere ──
//
// The plane fit's sums may take the master by bicubic (Catmull–Rom) or by Keys' six-point cubic
// convolution (Keys 1981, fourth-order accurate) instead of the bilinear gradient table
// (detector.wgsl grad_at_cubic / grad_at_keys6, 146-248): the intensity is then smooth across the
// sheet's pixels, and the gradient is the derivative of the same surface. The sheet's
// coordinates are carried onto the sphere by central differences of the square-Lambert map
// along two tangent directions, 1e-3 rad either way.

// one texel of the hemisphere's sheet at offset o, the indices held inside the sheet
__device__ __forceinline__ float sheet_texel(const float* __restrict__ s, int o, int r, int c, int side) {
  r = min(max(r, 0), side - 1);
  c = min(max(c, 0), side - 1);
  return __ldg(s + o + r * side + c);
}

// Catmull–Rom weights of the four texels at −1, 0, 1, 2 from the cell's corner, and their slopes
__device__ __forceinline__ void catmull_rom(float t, float (&w)[4], float (&d)[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = 0.5f * (-t3 + 2.f * t2 - t);
  w[1] = 0.5f * (3.f * t3 - 5.f * t2 + 2.f);
  w[2] = 0.5f * (-3.f * t3 + 4.f * t2 + t);
  w[3] = 0.5f * (t3 - t2);
  d[0] = 0.5f * (-3.f * t2 + 4.f * t - 1.f);
  d[1] = 0.5f * (9.f * t2 - 10.f * t);
  d[2] = 0.5f * (-9.f * t2 + 8.f * t + 1.f);
  d[3] = 0.5f * (3.f * t2 - 2.f * t);
}

// Keys' six-point kernel at distance a ≥ 0 and its slope (cubic pieces on [0,1), [1,2), [2,3))
__device__ __forceinline__ float2 keys_kernel(float a) {
  if (a < 1.f) return make_float2((4.f / 3.f * a - 7.f / 3.f) * a * a + 1.f, (4.f * a - 14.f / 3.f) * a);
  if (a < 2.f)
    return make_float2(((-7.f / 12.f * a + 3.f) * a - 59.f / 12.f) * a + 2.5f, (-1.75f * a + 6.f) * a - 59.f / 12.f);
  if (a < 3.f)
    return make_float2(((1.f / 12.f * a - 2.f / 3.f) * a + 1.75f) * a - 1.5f, (0.25f * a - 4.f / 3.f) * a + 1.75f);
  return make_float2(0.f, 0.f);
}

__device__ __forceinline__ float3 unit3(float3 v) {
  const float r = rsqrtf(dot3(v, v));
  return make_float3(v.x * r, v.y * r, v.z * r);
}

// (intensity, gradient on the sphere) of the master at direction v by the smooth kernel KIND
// (1 Catmull–Rom, 2 Keys' six-point): .xyz the gradient, .w the intensity
template <int KIND>
__device__ float4 grad_smooth(const float* __restrict__ sheets, float3 v, int side) {
  const float2 uv = sphere_to_square(v);
  const float last = (float)(side - 1);
  const float fj = fminf(fmaxf((uv.x + 1.f) * 0.5f * last, 0.f), last);
  const float fi = fminf(fmaxf((uv.y + 1.f) * 0.5f * last, 0.f), last);
  const int c0 = min((int)fj, side - 2), r0 = min((int)fi, side - 2);
  const int o = v.z < 0.f ? side * side : 0;
  const float tj = fj - (float)c0, ti = fi - (float)r0;
  float val = 0.f, gj = 0.f, gi = 0.f;
  if (KIND == 1) {
    float wj[4], dj[4], wi[4], di[4];
    catmull_rom(tj, wj, dj);
    catmull_rom(ti, wi, di);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      float row = 0.f, drow = 0.f;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const float t = sheet_texel(sheets, o, r0 - 1 + a, c0 - 1 + b, side);
        row += wj[b] * t;
        drow += dj[b] * t;
      }
      val += wi[a] * row;
      gj += wi[a] * drow;
      gi += di[a] * row;
    }
  } else {
    float wj[6], dj[6], wi[6], di[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const float sj = tj - (float)(m - 2), si = ti - (float)(m - 2);
      const float2 kj = keys_kernel(fabsf(sj)), ki = keys_kernel(fabsf(si));
      wj[m] = kj.x;
      dj[m] = sj < 0.f ? -kj.y : (sj > 0.f ? kj.y : 0.f);
      wi[m] = ki.x;
      di[m] = si < 0.f ? -ki.y : (si > 0.f ? ki.y : 0.f);
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      float row = 0.f, drow = 0.f;
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        const float t = sheet_texel(sheets, o, r0 - 2 + a, c0 - 2 + b, side);
        row += wj[b] * t;
        drow += dj[b] * t;
      }
      val += wi[a] * row;
      gj += wi[a] * drow;
      gi += di[a] * row;
    }
  }
  // two directions across v, and how the sheet's coordinates move along them
  float3 e1 = cross3(v, make_float3(0.f, 0.f, 1.f));
  if (dot3(e1, e1) < 1e-4f) e1 = cross3(v, make_float3(1.f, 0.f, 0.f));
  e1 = unit3(e1);
  const float3 e2 = cross3(v, e1);
  const float h = 1e-3f, k = 0.5f * last / (2.f * h);
  const float2 p1 = sphere_to_square(unit3(make_float3(v.x + h * e1.x, v.y + h * e1.y, v.z + h * e1.z)));
  const float2 m1 = sphere_to_square(unit3(make_float3(v.x - h * e1.x, v.y - h * e1.y, v.z - h * e1.z)));
  const float2 p2 = sphere_to_square(unit3(make_float3(v.x + h * e2.x, v.y + h * e2.y, v.z + h * e2.z)));
  const float2 m2 = sphere_to_square(unit3(make_float3(v.x - h * e2.x, v.y - h * e2.y, v.z - h * e2.z)));
  const float2 d1 = make_float2((p1.x - m1.x) * k, (p1.y - m1.y) * k);
  const float2 d2 = make_float2((p2.x - m2.x) * k, (p2.y - m2.y) * k);
  const float a1 = gj * d1.x + gi * d1.y, a2 = gj * d2.x + gi * d2.y;
  return make_float4(e1.x * a1 + e2.x * a2, e1.y * a1 + e2.y * a2, e1.z * a1 + e2.z * a2, val);
}

// ∂(fj, fi)/∂c of the sheet coordinates fj = (U + 1)/2·last, fi = (W + 1)/2·last of direction c
// (sphere_to_square, common.wgsl:44-57), from the map's own formula and the intermediates its
// evaluation left (square_map: ρ², 1/(1 + |z|), 1/√q, xn = √q, the fitted arctangent); zero where
// clamped or at the poles of the map (x = y = 0).
__device__ __forceinline__ void sheet_jacobian_of(const SquareMap& m, float3 c, int side, float3& dfj, float3& dfi) {
  const float ax = fabsf(c.x), ay = fabsf(c.y);
  const float sx = c.x < 0.f ? -1.f : 1.f, sy = c.y < 0.f ? -1.f : 1.f, sz = c.z < 0.f ? -1.f : 1.f;
  const float rho2 = m.rho2;
  dfj = make_float3(0.f, 0.f, 0.f);
  dfi = make_float3(0.f, 0.f, 0.f);
  if (rho2 < 1e-20f) return;
  const float rden = m.rden, rrho2 = __fdividef(1.f, rho2);
  const float xn = m.xn;
  // ∂xn = ∂q / (2 xn); ∂q = (π x/den, π y/den, −(π/2) ρ² sgn(z)/den²)
  const float k = 0.5f * m.rq;
  const float3 dxn = make_float3(k * ZEB_PI * c.x * rden, k * ZEB_PI * c.y * rden, -k * 0.5f * ZEB_PI * rho2 * sz * rden * rden);
  const float four_pi = 4.f / ZEB_PI;
  // the angle as the lookup's map takes it (the fitted arctangent of the smaller over the larger
  // coordinate)
  const float ang = m.at;
  float3 du, dw;
  if (ax >= ay) {
    const float al = ang;
    const float3 dal = make_float3(-ay * sx * rrho2, ax * sy * rrho2, 0.f);
    du = dxn;
    dw = make_float3(four_pi * (dxn.x * al + xn * dal.x), four_pi * (dxn.y * al + xn * dal.y), four_pi * dxn.z * al);
  } else {
    const float be = ang;
    const float3 dbe = make_float3(ay * sx * rrho2, -ax * sy * rrho2, 0.f);
    du = make_float3(four_pi * (dxn.x * be + xn * dbe.x), four_pi * (dxn.y * be + xn * dbe.y), four_pi * dxn.z * be);
    dw = dxn;
  }
  const float sc = 0.79788456080286536f;  // 1 / sqrt(π / 2)
  const float last = (float)(side - 1);
  const float kj = 0.5f * last * sc * sx, ki = 0.5f * last * sc * sy;
  dfj = make_float3(kj * du.x, kj * du.y, kj * du.z);
  dfi = make_float3(ki * dw.x, ki * dw.y, ki * dw.z);
}

// The bilinear master value at c and its gradient along the sphere (the exact derivative of the
// lookup, projected on the tangent plane at c).
__device__ __forceinline__ float master_and_slope(const float2* __restrict__ vp, float3 c, int side, float3& grad) {
  const SquareMap sm = square_map(c);
  const float2 uv = sm.uv;
  const float last = (float)(side - 1);
  const float fj0 = (uv.x + 1.f) * 0.5f * last, fi0 = (uv.y + 1.f) * 0.5f * last;
  const float fj = fminf(fmaxf(fj0, 0.f), last), fi = fminf(fmaxf(fi0, 0.f), last);
  const uint32_t cj = min((uint32_t)fj, (uint32_t)(side - 2)), ri = min((uint32_t)fi, (uint32_t)(side - 2));
  uint32_t o = ri * side + cj;
  if (c.z < 0.f) o += side * side;
  const float tj = fj - (float)cj, ti = fi - (float)ri;
  const float2 t = __ldg(vp + o), u = __ldg(vp + o + side);
  const float top = lerpf(t.x, t.y, tj), bot = lerpf(u.x, u.y, tj);
  const float m = lerpf(top, bot, ti);
  const float dmj = (fj0 > 0.f && fj0 < last) ? (1.f - ti) * (t.y - t.x) + ti * (u.y - u.x) : 0.f;
  const float dmi = (fi0 > 0.f && fi0 < last) ? bot - top : 0.f;
  float3 dfj, dfi;
  sheet_jacobian_of(sm, c, side, dfj, dfi);
  float3 g = make_float3(dmj * dfj.x + dmi * dfi.x, dmj * dfj.y + dmi * dfi.y, dmj * dfj.z + dmi * dfi.z);
  const float r = dot3(g, c);
  grad = make_float3(g.x - r * c.x, g.y - r * c.y, g.z - r * c.z);
  return m;
}

// Both lookups of MODE 3 from the gradient table alone: its 2 × 2 records' value slots are the
// sheet's texels, so the bilinear value and its exact slopes (master_and_slope's) come with the
// table's interpolated gradient (grad_at_pair's), from one map to the square and one pair of loads.
__device__ __forceinline__ float4 grad_and_slope(const float* __restrict__ gp, float3 c, int side, float3& grad) {
  const SquareMap sm = square_map(c);
  const float2 uv = sm.uv;
  const float last = (float)(side - 1);
  const float fj0 = (uv.x + 1.f) * 0.5f * last, fi0 = (uv.y + 1.f) * 0.5f * last;
  const float fj = fminf(fmaxf(fj0, 0.f), last), fi = fminf(fmaxf(fi0, 0.f), last);
  const uint32_t cj = min((uint32_t)fj, (uint32_t)(side - 2)), ri = min((uint32_t)fi, (uint32_t)(side - 2));
  uint32_t o = ri * side + cj;
  if (c.z < 0.f) o += side * side;
  const float tj = fj - (float)cj, ti = fi - (float)ri;
  float4 ta, tb, tc, td;
  ldg_v8(gp + 8 * (size_t)o, ta, tb);
  ldg_v8(gp + 8 * ((size_t)o + side), tc, td);
  const float4 top = lerp4(ta, tb, tj), bot = lerp4(tc, td, tj);
  const float4 gm = lerp4(top, bot, ti);
  const float dmj = (fj0 > 0.f && fj0 < last) ? (1.f - ti) * (tb.w - ta.w) + ti * (td.w - tc.w) : 0.f;
  const float dmi = (fi0 > 0.f && fi0 < last) ? bot.w - top.w : 0.f;
  float3 dfj, dfi;
  sheet_jacobian_of(sm, c, side, dfj, dfi);
  const float3 g = make_float3(dmj * dfj.x + dmi * dfi.x, dmj * dfj.y + dmi * dfi.y, dmj * dfj.z + dmi * dfi.z);
  const float r = dot3(g, c);
  grad = make_float3(g.x - r * c.x, g.y - r * c.y, g.z - r * c.z);
  return gm;
}

// One pixel's share of the sums, from its ray already turned by the pattern's rotation R:
// rv = R·v, v = u + δt (pixels), and its pattern value e. The derivatives along the shift,
// R⁻¹·∇M/|v|, are summed in the turned frame as ∇M/|v| (det6_unturn takes the sums back once a
// pattern: R⁻¹ on the vectors, R⁻¹·(·)·R and R⁻¹·(·) on the blocks of products); those along the
// rotation, c × ∇M, need no turning.
template <int MODE, int NS>
__device__ __forceinline__ void det6_pixel(const Det6Args& a, float3 rv, float e, float (&s)[NS]) {
  const float inv = rsqrtf(dot3(rv, rv));  // 1/|v|
  const float3 c = make_float3(rv.x * inv, rv.y * inv, rv.z * inv);
  float m;
  float d[6], dx[6];
  if (MODE == 0) {
    m = master_at_pair(a.vpair, c, a.side);
  } else {
    float3 g;
    if (MODE == 1) {
      m = master_and_slope(a.vpair, c, a.side, g);
    } else if (MODE == 2) {
      const float4 gm = a.interp == 0   ? grad_at_pair(a.gpair, c, a.side)
                        : a.interp == 1 ? grad_smooth<1>(a.sheets, c, a.side)
                                        : grad_smooth<2>(a.sheets, c, a.side);
      m = gm.w;
      g = make_float3(gm.x, gm.y, gm.z);
    } else {
      float3 ge;
      const float4 gm = grad_and_slope(a.gpair, c, a.side, ge);
      m = gm.w;
      g = make_float3(gm.x, gm.y, gm.z);
      const float3 re = cross3(c, ge);
      dx[0] = ge.x * inv; dx[1] = ge.y * inv; dx[2] = ge.z * inv;
      dx[3] = re.x; dx[4] = re.y; dx[5] = re.z;
    }
    const float3 r = cross3(c, g);
    d[0] = g.x * inv; d[1] = g.y * inv; d[2] = g.z * inv;
    d[3] = r.x; d[4] = r.y; d[5] = r.z;
  }
  s[0] += 1.f;
  s[1] += m;
  s[2] += m * m;
  s[3] += m * e;
  if (MODE >= 1) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      s[4 + i] += d[i];
      s[10 + i] += m * d[i];
      s[16 + i] += e * d[i];
    }
  }
  if (MODE >= 2) {
    int o = 22;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j) s[o++] += d[i] * d[j];
  }
  if (MODE == 3) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      s[43 + i] += dx[i];
      s[49 + i] += m * dx[i];
      s[55 + i] += e * dx[i];
    }
  }
}

// offset of the product (i, j), i <= j, among the 21 of the GN sums
__host__ __device__ constexpr int det6_pair(int i, int j) { return 22 + i * 6 - (i * (i - 1)) / 2 + (j - i); }

// the summed shift derivatives back from the turned frame (thread 0, once a pattern): with R's
// columns r_k = R·e_k, a vector w becomes (r_k · w)_k, the shift × shift block M becomes
// r_kᵀ·M·r_l, the shift × rotation block N becomes r_kᵀ·N
template <int MODE, int NS>
__device__ __forceinline__ void det6_unturn(float4 q, float (&s)[NS]) {
  if (MODE == 0) return;
  const float3 r[3] = {qrot(q, make_float3(1.f, 0.f, 0.f)), qrot(q, make_float3(0.f, 1.f, 0.f)),
                       qrot(q, make_float3(0.f, 0.f, 1.f))};
  auto vec = [&](int o) {
    const float3 w = make_float3(s[o], s[o + 1], s[o + 2]);
    s[o] = dot3(r[0], w); s[o + 1] = dot3(r[1], w); s[o + 2] = dot3(r[2], w);
  };
  vec(4); vec(10); vec(16);
  if (MODE == 3) { vec(43); vec(49); vec(55); }
  if (MODE >= 2) {
    float M[3][3], N[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        M[i][j] = s[det6_pair(i < j ? i : j, i < j ? j : i)];
        N[i][j] = s[det6_pair(i, 3 + j)];
      }
    float MR[3][3];  // M·r_l
    for (int i = 0; i < 3; ++i)
      for (int l = 0; l < 3; ++l) MR[i][l] = M[i][0] * r[l].x + M[i][1] * r[l].y + M[i][2] * r[l].z;
    for (int k = 0; k < 3; ++k)
      for (int l = k; l < 3; ++l)
        s[det6_pair(k, l)] = r[k].x * MR[0][l] + r[k].y * MR[1][l] + r[k].z * MR[2][l];
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) s[det6_pair(k, 3 + l)] = r[k].x * N[0][l] + r[k].y * N[1][l] + r[k].z * N[2][l];
  }
}

// the pattern's outputs from its summed sums (thread 0): MODE 2 the 43 sums; MODE 0 the NCC;
// MODE 1 the NCC and its gradient (planefit.zig:176-200)
template <int MODE, int NS>
__device__ __forceinline__ void det6_finish(const Det6Args& a, int b, const float (&s)[NS]) {
  if (MODE >= 2) {
    for (int k = 0; k < NS; ++k) a.out[(size_t)b * NS + k] = s[k];
    return;
  }
  // planefit.zig:176-200: NCC and (MODE 1) its gradient
  const float n = fmaxf(s[0], 1.f);
  const float mean = s[1] / n;
  const float var_n = s[2] - n * mean * mean;
  float ncc = -2.f, g[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (var_n > 1e-12f) {
    const float inv = rsqrtf(var_n);
    ncc = s[3] * inv;
    if (MODE == 1)
      for (int i = 0; i < 6; ++i) {
        const float au = (s[10 + i] - mean * s[4 + i]) * inv;
        g[i] = (s[16 + i] - ncc * au) * inv;
      }
  }
  if (MODE == 0) {
    a.out[b] = ncc;
  } else {
    float* o = a.out + (size_t)b * 7;
    for (int i = 0; i < 6; ++i) o[i] = g[i];
    o[6] = ncc;
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_det6(Det6Args a) {
  constexpr int NS = MODE == 0 ? 4 : (MODE == 1 ? 22 : (MODE == 2 ? 43 : 61));
  extern __shared__ float4 px6[];
  __shared__ float red[NS * 8];
  __shared__ int wcnt[8];
  __shared__ float4 sh_q;
  __shared__ float3 sh_t;
  const int b = blockIdx.x;
  const int hw = a.h * a.w;
  const float4 it = a.items[b];
  const float* gpat = a.pats + (size_t)(int)it.w * hw;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // the masked pixels in raster order: (c0·row + c1·col + t, value)
  int npix = 0;
  for (int base = 0; base < hw; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int row = i / a.w, col = i - row * a.w;
    float dr = (float)row - a.mask[0], dc = (float)col - a.mask[1];
    const bool m = i < hw && zeb_in_circle(dr, dc, a.mask[2]);
    const unsigned bal = __ballot_sync(0xffffffffu, m);
    if (lane == 0) wcnt[wid] = __popc(bal);
    __syncthreads();
    int off = npix, tot = 0;
    for (int w2 = 0; w2 < nw; ++w2) {
      if (w2 < wid) off += wcnt[w2];
      tot += wcnt[w2];
    }
    if (m) px6[off + __popc(bal & ((1u << lane) - 1u))] = make_float4((float)row, (float)col, 0.f, __ldg(gpat + i));
    npix += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float* x = a.x + (size_t)b * 6;
    const float* q0 = a.q0 + (size_t)b * 4;
    float4 q = qmul(qexp(make_float3(x[3], x[4], x[5])), make_float4(q0[0], q0[1], q0[2], q0[3]));
    const float nq = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    sh_q = make_float4(q.x * nq, q.y * nq, q.z * nq, q.w * nq);
    sh_t = make_float3(x[0], x[1], x[2]);
  }
  __syncthreads();
  const float4 q = sh_q;
  const float3 dt = sh_t;
  // the frame turned once: R·v = row·R c0 + col·R c1 + R (t + δt)
  const float3 rc0 = qrot(q, a.c0), rc1 = qrot(q, a.c1);
  const float3 rt = qrot(q, make_float3(it.x + dt.x, it.y + dt.y, it.z + dt.z));
  float s[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) s[k] = 0.f;
  // unrolled: several master lookups of a thread in flight at once
#pragma unroll 2
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const float4 p = px6[k];
    const float3 rv = make_float3(fmaf(rc0.x, p.x, fmaf(rc1.x, p.y, rt.x)), fmaf(rc0.y, p.x, fmaf(rc1.y, p.y, rt.y)),
                                  fmaf(rc0.z, p.x, fmaf(rc1.z, p.y, rt.z)));
    det6_pixel<MODE, NS>(a, rv, p.w, s);
  }
  block_sums<NS>(s, red);
  if (threadIdx.x != 0) return;
  det6_unturn<MODE, NS>(q, s);
  det6_finish<MODE, NS>(a, b, s);
}

// The same over the frame's masked-pixel list (zeb_mask_list, shared by every pattern): 128
// threads per pattern keep only the pattern's values along the list in shared memory and
// recompute each pixel's ray, so that several patterns share an SM (a list of (ray, value) per
// block fills an SM's shared memory for one 120 × 120 pattern).
// (the one-pass mode: five blocks an SM at 96 registers, one pixel a thread at a time, measured
// 11 % faster than four blocks with two pixels in flight: the table loads' latency is hidden by
// the warps rather than by unrolling; the other modes keep four blocks, which mode 2's smooth
// kernels need to run without spilling)
template <int MODE>
__global__ void __launch_bounds__(128, MODE == 3 ? 5 : 4) k_det6_list(Det6Args a, const uint32_t* __restrict__ list,
                                                                     int npix) {
  constexpr int NS = MODE == 0 ? 4 : (MODE == 1 ? 22 : (MODE == 2 ? 43 : 61));
  extern __shared__ float pv6[];
  __shared__ float red[NS * 4];
  __shared__ float4 sh_q;
  __shared__ float3 sh_t;
  const int b = blockIdx.x;
  const float4 it = a.items[b];
  const float* gpat = a.pats + (size_t)(int)it.w * a.h * a.w;
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const uint32_t v = __ldg(list + k);
    pv6[k] = __ldg(gpat + (int)(v >> 16) * a.w + (int)(v & 0xffffu));
  }
  if (threadIdx.x == 0) {
    const float* x = a.x + (size_t)b * 6;
    const float* q0 = a.q0 + (size_t)b * 4;
    float4 q = qmul(qexp(make_float3(x[3], x[4], x[5])), make_float4(q0[0], q0[1], q0[2], q0[3]));
    const float nq = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    sh_q = make_float4(q.x * nq, q.y * nq, q.z * nq, q.w * nq);
    sh_t = make_float3(x[0], x[1], x[2]);
  }
  __syncthreads();
  const float4 q = sh_q;
  const float3 dt = sh_t;
  // the frame turned once: R·v = row·R c0 + col·R c1 + R (t + δt)
  const float3 rc0 = qrot(q, a.c0), rc1 = qrot(q, a.c1);
  const float3 rt = qrot(q, make_float3(it.x + dt.x, it.y + dt.y, it.z + dt.z));
  float s[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) s[k] = 0.f;
  auto pixel = [&](int k) {
    const uint32_t v = __ldg(list + k);
    const float row = (float)(int)(v >> 16), col = (float)(int)(v & 0xffffu);
    const float3 rv = make_float3(fmaf(rc0.x, row, fmaf(rc1.x, col, rt.x)), fmaf(rc0.y, row, fmaf(rc1.y, col, rt.y)),
                                  fmaf(rc0.z, row, fmaf(rc1.z, col, rt.z)));
    det6_pixel<MODE, NS>(a, rv, pv6[k], s);
  };
  if constexpr (MODE == 3) {
#pragma unroll 1
    for (int k = threadIdx.x; k < npix; k += blockDim.x) pixel(k);
  } else {
#pragma unroll 2
    for (int k = threadIdx.x; k < npix; k += blockDim.x) pixel(k);
  }
  block_sums<NS>(s, red);
  if (threadIdx.x != 0) return;
  det6_unturn<MODE, NS>(q, s);
  det6_finish<MODE, NS>(a, b, s);
}

// x = A⁻¹ b for a (6 × 6, 6) system per item in FP64 (planefit.zig:203-233); ok[b] = 0 where a
// pivot is below 1e-300 (x left 0).
__global__ void k_solve6(const double* __restrict__ A, const double* __restrict__ bvec, int n, double* __restrict__ x,
                         int* __restrict__ ok) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  double M[36], r[6];
  for (int i = 0; i < 36; ++i) M[i] = A[(size_t)b * 36 + i];
  for (int i = 0; i < 6; ++i) r[i] = bvec[(size_t)b * 6 + i];
  bool good = true;
  for (int c = 0; c < 6 && good; ++c) {
    int piv = c;
    for (int rr = c + 1; rr < 6; ++rr)
      if (fabs(M[rr * 6 + c]) > fabs(M[piv * 6 + c])) piv = rr;
    if (fabs(M[piv * 6 + c]) < 1e-300) {
      good = false;
      break;
    }
    if (piv != c) {
      for (int k = 0; k < 6; ++k) {
        const double t = M[c * 6 + k];
        M[c * 6 + k] = M[piv * 6 + k];
        M[piv * 6 + k] = t;
      }
      const double t = r[c];
      r[c] = r[piv];
      r[piv] = t;
    }
    for (int rr = c + 1; rr < 6; ++rr) {
      const double f = M[rr * 6 + c] / M[c * 6 + c];
      if (f == 0.0) continue;
      for (int k = c; k < 6; ++k) M[rr * 6 + k] -= f * M[c * 6 + k];
      r[rr] -= f * r[c];
    }
  }
  double y[6] = {0, 0, 0, 0, 0, 0};
  if (good) {
    for (int rr = 5; rr >= 0; --rr) {
      double acc = r[rr];
      for (int k = rr + 1; k < 6; ++k) acc -= M[rr * 6 + k] * y[k];
      y[rr] = acc / M[rr * 6 + rr];
    }
  }
  for (int i = 0; i < 6; ++i) x[(size_t)b * 6 + i] = y[i];
  ok[b] = good ? 1 : 0;
}

}  // namespace zeb

using namespace zeb;

extern "C" int zeb_det6(int mode, const float* pats, const float* items, int n, const zeb_frame_t* fr,
                        const float* vpair, const float* gpair, int side, const float* x, const float* q0, float* out,
                        void* stream) {
  ZEB_REQUIRE(mode >= 0 && mode <= 3, ZEB_EARG, "det6: mode %d", mode);
  ZEB_REQUIRE(pats && items && vpair && x && q0 && out && fr && side >= 3 && (mode < 2 || gpair), ZEB_EARG,
              "det6: bad arguments");
  ZEB_REQUIRE(((uintptr_t)gpair & 31) == 0 && ((uintptr_t)vpair & 7) == 0, ZEB_EARG, "det6: pair tables misaligned");
  if (n <= 0) return ZEB_OK;
  Det6Args a{};
  ZEB_REQUIRE(fr->h >= 2 && fr->w >= 2, ZEB_EARG, "det6: bad frame");
  a.h = fr->h; a.w = fr->w;
  a.c0 = make_float3(fr->c0[0], fr->c0[1], fr->c0[2]);
  a.c1 = make_float3(fr->c1[0], fr->c1[1], fr->c1[2]);
  a.c2 = make_float3(fr->c2[0], fr->c2[1], fr->c2[2]);
  for (int k = 0; k < 3; ++k) a.mask[k] = fr->mask[k];
  a.pats = pats; a.items = (const float4*)items; a.n = n; a.vpair = (const float2*)vpair; a.gpair = gpair;
  a.side = side; a.x = x; a.q0 = q0; a.out = out;
  const size_t list = (size_t)zeb_mask_count(fr) * sizeof(float4);
  ZEB_REQUIRE(list <= 200 * 1024, ZEB_ESIZE, "det6: the %d x %d pattern's masked pixels exceed the shared-memory list",
              a.h, a.w);
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 0) {
    cudaFuncSetAttribute(k_det6<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)list);
    k_det6<0><<<n, 256, list, st>>>(a);
  } else if (mode == 1) {
    cudaFuncSetAttribute(k_det6<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)list);
    k_det6<1><<<n, 256, list, st>>>(a);
  } else if (mode == 2) {
    cudaFuncSetAttribute(k_det6<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)list);
    k_det6<2><<<n, 256, list, st>>>(a);
  } else {
    cudaFuncSetAttribute(k_det6<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)list);
    k_det6<3><<<n, 256, list, st>>>(a);
  }
  return zeb_launch_check("det6");
}

extern "C" int zeb_det6_list(int mode, const float* pats, const float* items, int n, const zeb_frame_t* fr,
                             const uint32_t* list, int npix, const float* vpair, const float* gpair, int side,
                             const float* x, const float* q0, float* out, void* stream) {
  ZEB_REQUIRE(mode >= 0 && mode <= 3, ZEB_EARG, "det6_list: mode %d", mode);
  ZEB_REQUIRE(pats && items && list && vpair && x && q0 && out && fr && side >= 3 && (mode < 2 || gpair), ZEB_EARG,
              "det6_list: bad arguments");
  ZEB_REQUIRE(((uintptr_t)gpair & 31) == 0 && ((uintptr_t)vpair & 7) == 0, ZEB_EARG,
              "det6_list: pair tables misaligned");
  ZEB_REQUIRE(npix == zeb_mask_count(fr), ZEB_EARG, "det6_list: %d pixels listed, the frame masks %d", npix,
              zeb_mask_count(fr));
  const size_t smem = (size_t)npix * sizeof(float);
  ZEB_REQUIRE(npix >= 1 && smem <= 200 * 1024, ZEB_ESIZE, "det6_list: %d pixels (at most 51200)", npix);
  if (n <= 0) return ZEB_OK;
  Det6Args a{};
  ZEB_REQUIRE(fr->h >= 2 && fr->w >= 2 && fr->h < 65536 && fr->w < 65536, ZEB_EARG, "det6_list: bad frame");
  a.h = fr->h; a.w = fr->w;
  a.c0 = make_float3(fr->c0[0], fr->c0[1], fr->c0[2]);
  a.c1 = make_float3(fr->c1[0], fr->c1[1], fr->c1[2]);
  a.c2 = make_float3(fr->c2[0], fr->c2[1], fr->c2[2]);
  for (int k = 0; k < 3; ++k) a.mask[k] = fr->mask[k];
  a.pats = pats; a.items = (const float4*)items; a.n = n; a.vpair = (const float2*)vpair; a.gpair = gpair;
  a.side = side; a.x = x; a.q0 = q0; a.out = out;
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 0) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_det6_list<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_det6_list<0><<<n, 128, smem, st>>>(a, list, npix);
  } else if (mode == 1) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_det6_list<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_det6_list<1><<<n, 128, smem, st>>>(a, list, npix);
  } else if (mode == 2) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_det6_list<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_det6_list<2><<<n, 128, smem, st>>>(a, list, npix);
  } else {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_det6_list<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_det6_list<3><<<n, 128, smem, st>>>(a, list, npix);
  }
  return zeb_launch_check("det6_list");
}

extern "C" int zeb_sums6_list(const float* pats, const float* items, int n, const zeb_frame_t* fr,
                              const uint32_t* list, int npix, const float* sheets, const float* gpair, int side,
                              int interp, const float* x, const float* q0, float* out, void* stream) {
  ZEB_REQUIRE(interp >= 0 && interp <= 2, ZEB_EARG, "sums6_list: interp %d", interp);
  ZEB_REQUIRE(pats && items && list && x && q0 && out && fr && side >= 3 && (interp != 0 || gpair) &&
                  (interp == 0 || sheets),
              ZEB_EARG, "sums6_list: bad arguments");
  ZEB_REQUIRE(((uintptr_t)gpair & 31) == 0, ZEB_EARG, "sums6_list: gradient pairs misaligned");
  ZEB_REQUIRE(npix == zeb_mask_count(fr), ZEB_EARG, "sums6_list: %d pixels listed, the frame masks %d", npix,
              zeb_mask_count(fr));
  const size_t smem = (size_t)npix * sizeof(float);
  ZEB_REQUIRE(npix >= 1 && smem <= 200 * 1024, ZEB_ESIZE, "sums6_list: %d pixels (at most 51200)", npix);
  if (n <= 0) return ZEB_OK;
  Det6Args a{};
  ZEB_REQUIRE(fr->h >= 2 && fr->w >= 2 && fr->h < 65536 && fr->w < 65536, ZEB_EARG, "sums6_list: bad frame");
  a.h = fr->h; a.w = fr->w;
  a.c0 = make_float3(fr->c0[0], fr->c0[1], fr->c0[2]);
  a.c1 = make_float3(fr->c1[0], fr->c1[1], fr->c1[2]);
  a.c2 = make_float3(fr->c2[0], fr->c2[1], fr->c2[2]);
  for (int k = 0; k < 3; ++k) a.mask[k] = fr->mask[k];
  a.pats = pats; a.items = (const float4*)items; a.n = n; a.gpair = gpair; a.sheets = sheets; a.interp = interp;
  a.side = side; a.x = x; a.q0 = q0; a.out = out;
  cudaStream_t st = (cudaStream_t)stream;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_det6_list<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_det6_list<2><<<n, 128, smem, st>>>(a, list, npix);
  return zeb_launch_check("sums6_list");
}

extern "C" int zeb_solve6(const double* A, const double* b, int n, double* x, int* ok, void* stream) {
  ZEB_REQUIRE(A && b && x && ok, ZEB_EARG, "solve6: null argument");
  if (n <= 0) return ZEB_OK;
  k_solve6<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(A, b, n, x, ok);
  return zeb_launch_check("solve6");
}
