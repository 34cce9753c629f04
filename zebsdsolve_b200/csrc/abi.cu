// The library's own C-ABI plumbing: version and the per-thread error message.
#include <stdarg.h>
#include <string.h>

#include "abi_util.cuh"

namespace zeb {
static thread_local char g_error[1024];

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
