// C ABI runtime pieces: per-thread error messages, launch accounting, version.
#include <stdarg.h>
#include "common.cuh"

namespace dpb {

static thread_local char g_err[1024] = "";
static std::atomic<uint64_t> g_launches{0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

}  // namespace dpb

extern "C" const char* dp_last_error(void) { return dpb::g_err; }
extern "C" int dp_version(void) { return 1; }
extern "C" uint64_t dp_launch_count(void) { return dpb::g_launches.load(std::memory_order_relaxed); }
