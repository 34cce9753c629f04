// Error reporting shared by the C-ABI entry points: a per-thread message that zeb_error() hands
// back, argument checks that fail with a message rather than launching, and a launch check.
#pragma once
#include <cuda_runtime.h>
#include <stdio.h>

#include "../../include/zebsdsolve_b200.h"
#include "common.cuh"

namespace zeb {
void set_error(const char* fmt, ...);
long long test_stall_ns();  // zeb_set_test_stall's value (0: off)
// how long a wait of the tensor-core kernels may take (1 s, far above any legitimate wait inside
// one CTA), and the waits for a CTA's own copies and MMAs in flight once it has given up
constexpr long long kWaitNs = 1000000000LL;
constexpr long long kDrainNs = 1000000000LL;
}

#define ZEB_REQUIRE(cond, code, ...) \
  do {                               \
    if (!(cond)) {                   \
      ::zeb::set_error(__VA_ARGS__); \
      return (code);                 \
    }                                \
  } while (0)

static inline int zeb_launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ::zeb::set_error("%s: %s", what, cudaGetErrorString(e));
    return ZEB_ECUDA;
  }
  return ZEB_OK;
}

// pixels of an h × w pattern inside the frame's circular mask (all of them without one), on the host
static inline int zeb_mask_count(const zeb_frame_t* fr) {
  int cnt = 0;
  for (int r = 0; r < fr->h; ++r)
    for (int c = 0; c < fr->w; ++c) {
      const float dr = (float)r - fr->mask[0], dc = (float)c - fr->mask[1];
      if (::zeb::zeb_in_circle(dr, dc, fr->mask[2])) ++cnt;
    }
  return cnt;
}
