// The pattern-centre vote's density of ballots, on the host (no GPU): each ballot spread over
// the candidate grid by a Gaussian, summed in float32 ballot by ballot.
//
// Replaces splat (src/pcfit.zig:210-236). The vote's other steps are host arithmetic over a few
// hundred values per grid; this is the one with a loop per ballot and per candidate cell.
#include <cmath>
#include <vector>

#include "abi_util.cuh"

#pragma STDC FP_CONTRACT OFF

extern "C" int zeb_pc_splat(const int* at, const double* w, int n_ballots, const int* n, const double* sigma,
                            float* out) {
  ZEB_REQUIRE(n_ballots >= 0 && n && sigma && out && (n_ballots == 0 || (at && w)), ZEB_EARG,
              "pc_splat: bad arguments");
  for (int a = 0; a < 3; ++a) ZEB_REQUIRE(n[a] >= 1 && sigma[a] > 0, ZEB_EARG, "pc_splat: bad grid or sigma");
  const long long cells = (long long)n[0] * n[1] * n[2];
  for (long long i = 0; i < cells; ++i) out[i] = 0.0f;
  int r[3];
  double inv[3];
  for (int a = 0; a < 3; ++a) {
    // out to three sigma, never beyond the grid
    const double reach = std::fmin(std::ceil(3.0 * sigma[a]), (double)(n[a] - 1));
    r[a] = (int)reach;
    inv[a] = 1.0 / (2.0 * sigma[a] * sigma[a]);
  }
  // exp(−Σ d²/(2σ²)) depends on the offsets alone: once per offset, the same for every ballot
  const int sx = 2 * r[0] + 1, sy = 2 * r[1] + 1, sz = 2 * r[2] + 1;
  std::vector<double> g((size_t)sx * sy * sz);
  for (int dz = -r[2]; dz <= r[2]; ++dz)
    for (int dy = -r[1]; dy <= r[1]; ++dy)
      for (int dx = -r[0]; dx <= r[0]; ++dx) {
        const double fx = (double)dx, fy = (double)dy, fz = (double)dz;
        const double ex = fx * fx * inv[0];
        const double ey = fy * fy * inv[1];
        const double ez = fz * fz * inv[2];
        const double e = (ex + ey) + ez;
        g[(size_t)(dx + r[0]) + (size_t)sx * ((dy + r[1]) + (size_t)sy * (dz + r[2]))] = std::exp(-e);
      }
  for (int b = 0; b < n_ballots; ++b) {
    const int cx = at[3 * b], cy = at[3 * b + 1], cz = at[3 * b + 2];
    const int z0 = cz - r[2] > 0 ? cz - r[2] : 0, z1 = cz + r[2] < n[2] - 1 ? cz + r[2] : n[2] - 1;
    const int y0 = cy - r[1] > 0 ? cy - r[1] : 0, y1 = cy + r[1] < n[1] - 1 ? cy + r[1] : n[1] - 1;
    const int x0 = cx - r[0] > 0 ? cx - r[0] : 0, x1 = cx + r[0] < n[0] - 1 ? cx + r[0] : n[0] - 1;
    for (int z = z0; z <= z1; ++z)
      for (int y = y0; y <= y1; ++y) {
        const double* gr = g.data() + (size_t)sx * ((y - cy + r[1]) + (size_t)sy * (z - cz + r[2]));
        float* row = out + (long long)n[0] * (y + (long long)n[1] * z);
        for (int x = x0; x <= x1; ++x) {
          const float term = (float)(w[b] * gr[x - cx + r[0]]);
          row[x] = row[x] + term;
        }
      }
  }
  return ZEB_OK;
}
