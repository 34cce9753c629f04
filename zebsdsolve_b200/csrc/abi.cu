// The library's own C-ABI plumbing: version and the per-thread error message.
#include <stdarg.h>
#include <string.h>

#include "abi_util.cuh"

namespace zeb {
static thread_local char g_error[1024];
static long long g_test_stall_ns = 0;  // zeb_set_test_stall: 0 off

long long test_stall_ns() { return __atomic_load_n(&g_test_stall_ns, __ATOMIC_RELAXED); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}
}  // namespace zeb

extern "C" size_t zeb_error(char* buf, size_t cap) {
  size_t n = strlen(zeb::g_error);
  if (buf && cap > 0) {
    size_t k = n < cap - 1 ? n : cap - 1;
    memcpy(buf, zeb::g_error, k);
    buf[k] = 0;
  }
  zeb::g_error[0] = 0;
  return n;
}

extern "C" const char* zeb_version(void) { return "0.2.8"; }

// The wait limit of the tensor-core kernels' failure test: while ns > 0, every tcgen05 kernel
// launched makes its MMA thread wait first on an mbarrier that nothing arrives at, and gives each
// of its waits ns nanoseconds (the waits for its own copies in flight keep 1 s).
extern "C" int zeb_set_test_stall(long long ns) {
  ZEB_REQUIRE(ns >= 0 && ns <= 10000000000LL, ZEB_EARG, "set_test_stall: %lld ns", ns);
  __atomic_store_n(&zeb::g_test_stall_ns, ns, __ATOMIC_RELAXED);
  return ZEB_OK;
}
