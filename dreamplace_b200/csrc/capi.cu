// C ABI runtime pieces: per-thread error messages, launch accounting, version.
#include <stdarg.h>
#include <mutex>
#include <set>
#include <utility>

#include "reduce.cuh"

namespace dpb {

static thread_local char g_err[1024] = "";
static std::atomic<uint64_t> g_launches{0};
static const int* g_trial_gate = nullptr;

const int* trial_gate() { return g_trial_gate; }

__global__ void trial_gate_kernel(int* gate, const double* accept_prev) {
  grid_dep_sync();
  *gate = accept_prev ? (*accept_prev == 0.0 ? 1 : 0) : 0;
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

static std::mutex g_smem_mu;
static std::set<std::pair<const void*, int>> g_smem_opted;
bool smem_opt_in_done(const void* kernel, int device) {
  std::lock_guard<std::mutex> lock(g_smem_mu);
  return g_smem_opted.count({kernel, device}) != 0;
}
void smem_opt_in_mark(const void* kernel, int device) {
  std::lock_guard<std::mutex> lock(g_smem_mu);
  g_smem_opted.insert({kernel, device});
}

__global__ void finish_sum_kernel(double* buf, int count, float* out_f32) {
  grid_dep_sync();
  double r = finish_sum(buf + 1, count);
  if (threadIdx.x == 0) {
    buf[0] = r;
    if (out_f32) *out_f32 = (float)r;
  }
}

int launch_finish_sum(double* buf, int count, float* out_f32, cudaStream_t s) {
  launch_kernel(finish_sum_kernel, 1, kReduceThreads, 0, s, buf, count, out_f32);
  return check_launch("finish_sum");
}

// two independent fixed-order reductions of `count` partials in one launch
__global__ void finish_sum2_kernel(double* a, double* b, int count) {
  grid_dep_sync();
  double ra = finish_sum(a + 1, count);
  double rb = finish_sum(b + 1, count);
  if (threadIdx.x == 0) {
    a[0] = ra;
    b[0] = rb;
  }
}

int launch_finish_sum2(double* a, double* b, int count, cudaStream_t s) {
  launch_kernel(finish_sum2_kernel, 1, kReduceThreads, 0, s, a, b, count);
  return check_launch("finish_sum2");
}

}  // namespace dpb

extern "C" const char* dp_last_error(void) { return dpb::g_err; }
extern "C" int dp_set_trial_gate(const int* gate) {
  dpb::g_trial_gate = gate;
  return DP_OK;
}
extern "C" int dp_trial_gate(int* gate, const double* accept_prev, dp_stream_t stream) {
  DP_REQUIRE(gate, "dp_trial_gate: null gate");
  dpb::launch_kernel(dpb::trial_gate_kernel, 1, 1, 0, dpb::as_stream(stream), gate, accept_prev);
  return dpb::check_launch("dp_trial_gate");
}
extern "C" int dp_version(void) { return 1; }
extern "C" uint64_t dp_launch_count(void) { return dpb::g_launches.load(std::memory_order_relaxed); }

extern "C" int dp_zero(void* ptr, size_t bytes, dp_stream_t stream) {
  DP_REQUIRE(ptr || bytes == 0, "dp_zero: null pointer");
  if (bytes == 0) return DP_OK;
  cudaError_t e = cudaMemsetAsync(ptr, 0, bytes, dpb::as_stream(stream));
  if (e != cudaSuccess) {
    dpb::set_error("dp_zero: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  return DP_OK;
}
