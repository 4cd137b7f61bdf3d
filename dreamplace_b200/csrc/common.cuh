// Shared helpers for the dreamplace_b200 C ABI implementation (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <float.h>
#include <math.h>
#include <string.h>
#include <stdio.h>
#include <atomic>
#include <string>
#include <utility>

#include "dreamplace_b200.h"

namespace dpb {

constexpr int kNumSMs = 148;  // B200

void set_error(const char* fmt, ...);
void count_launch(int n = 1);

// Trial gate (dp_set_trial_gate): the device word that the heavy kernels of a
// GP trial receive while a gate is installed on the host; such a kernel returns
// at once when the word is non-zero (a trial enqueued ahead whose predecessor
// was rejected, to be enqueued again).  nullptr when no gate is installed.
const int* trial_gate();
__device__ __forceinline__ bool gate_closed(const int* gate) { return gate != nullptr && *gate != 0; }

inline cudaStream_t as_stream(dp_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: CUDA launch failed: %s", what, cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  count_launch();
  return DP_OK;
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Programmatic dependent launch.  Every kernel of this library is launched
// with programmatic stream serialisation allowed, and starts with
// grid_dep_sync(): it waits there until the kernels before it in the stream
// have completed and their writes are visible (griddepcontrol.wait), then lets
// the next kernel be scheduled (griddepcontrol.launch_dependents).  The next
// kernel's launch and block scheduling thus overlap this kernel's run instead
// of following its last block; no kernel reads data before its wait.  A kernel
// launched without the attribute (or after a copy or memset) waits as usual.
__device__ __forceinline__ void grid_dep_sync() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline void launch_kernel(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                          Args&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // a failed launch is reported by the caller's check_launch (cudaGetLastError)
  (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Raises a kernel's dynamic shared-memory limit once per device: the
// attribute applies to the device current when it is set, so a process that
// launches on several GPUs sets it on each.  Thread-safe; returns DP_OK or
// DP_ERR_CUDA (message set).
// whether a kernel's shared-memory limit was already raised on a device, and
// the record that it was (capi.cu; thread-safe)
bool smem_opt_in_done(const void* kernel, int device);
void smem_opt_in_mark(const void* kernel, int device);
template <typename Kernel>
int opt_in_smem(Kernel kernel, int bytes, const char* who) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("%s: cudaGetDevice: %s", who, cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  const void* key = reinterpret_cast<const void*>(kernel);
  if (smem_opt_in_done(key, dev)) return DP_OK;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) {
    set_error("%s: cudaFuncSetAttribute: %s", who, cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  smem_opt_in_mark(key, dev);
  return DP_OK;
}

// grid size for a grid-stride elementwise kernel: a multiple of the SM count
inline int grid_for(long long n, int threads, int per_sm = 8) {
  long long blocks = (n + threads - 1) / threads;
  long long cap = (long long)kNumSMs * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

#define DP_REQUIRE(cond, ...)            \
  do {                                   \
    if (!(cond)) {                       \
      ::dpb::set_error(__VA_ARGS__);     \
      return DP_ERR_INVALID_ARGUMENT;    \
    }                                    \
  } while (0)

// Round-to-nearest float arithmetic that nvcc may not contract into FMA; used
// wherever the CPU reference's operation order must be reproduced bit for bit.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// triangle_density_function of electric_potential/src/density_function.h:12-17:
//   bin_xl = xl + k*bin_size; min(x+size, bin_xl+bin_size) - max(x, bin_xl)
__device__ __forceinline__ float triangle_overlap(float x, float size, float xl, int k, float bs) {
  float bin_xl = fadd(xl, fmul((float)k, bs));
  return fsub(fminf(fadd(x, size), fadd(bin_xl, bs)), fmaxf(x, bin_xl));
}

// exact_density_function of electric_potential/src/density_function.h:19-36
__device__ __forceinline__ float exact_overlap(float x, float size, float bin_center, float bs,
                                               float l, float h, bool fixed_flag) {
  float half = bs / 2;
  float bin_xl = fsub(bin_center, half);
  float bin_xh = fadd(bin_center, half);
  if (!fixed_flag) {
    if (bin_xl <= l) bin_xl = fminf(bin_xl, x);
    if (bin_xh >= h) bin_xh = fmaxf(bin_xh, fadd(x, size));
  }
  return fmaxf(0.0f, fsub(fminf(fadd(x, size), bin_xh), fmaxf(x, bin_xl)));
}

// Bin range of a stretched cell: C int() truncation toward zero, as the
// reference does (electric_potential/src/electric_density_map.cpp:254-266).
__device__ __forceinline__ void triangle_bin_range(float x, float size, float lo, float inv_bs,
                                                   int nbins, int& b0, int& b1) {
  int l = (int)fmul(fsub(x, lo), inv_bs);
  int h = (int)fmul(fsub(fadd(x, size), lo), inv_bs) + 1;
  b0 = max(l, 0);
  b1 = min(h, nbins);
}

// fixed-point conversion of one bin contribution: float * 2^f, truncated to a
// signed 64-bit integer (the CPU reference's `long sv = v * scale_factor`)
__device__ __forceinline__ long long to_fixed(float v, float scale) {
  return (long long)fmul(v, scale);
}

}  // namespace dpb
