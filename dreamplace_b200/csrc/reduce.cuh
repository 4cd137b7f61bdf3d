// Fixed-order fp64 reductions: each block writes its partial sum to
// partials[blockIdx.x]; a one-block finisher adds the partials in a fixed
// tree order.  Totals are therefore bit-reproducible run to run (the
// deterministic mode's requirement), unlike fp64 atomicAdd.  Callers pass
// DP_REDUCE_DOUBLES doubles: [0] receives the total, [1..] are the partials.
#pragma once
#include "common.cuh"

namespace dpb {

constexpr int kReduceThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// blockDim.x must be kReduceThreads
__device__ __forceinline__ void block_partial(double a, double* partials) {
  __shared__ double sa[kReduceThreads / 32];
  a = warp_sum(a);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sa[w] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kReduceThreads / 32; ++i) t += sa[i];
    partials[blockIdx.x] = t;
  }
  __syncthreads();
}

// every thread returns the same total: strided per-thread sums, an xor
// butterfly per warp (identical in every lane), then the warp totals in warp
// order; a fixed order, two block barriers
__device__ __forceinline__ double finish_sum(const double* partials, int count) {
  __shared__ double sh[kReduceThreads / 32];
  double v = 0.0;
  for (int i = threadIdx.x; i < count; i += kReduceThreads) v += partials[i];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
#pragma unroll
  for (int w = 0; w < kReduceThreads / 32; ++w) r += sh[w];
  __syncthreads();
  return r;
}

// <<<1, kReduceThreads>>>: buf[0] = sum(buf[1 .. 1+count)); out_f32 (optional) = (float)buf[0]
__global__ void finish_sum_kernel(double* buf, int count, float* out_f32);

int launch_finish_sum(double* buf, int count, float* out_f32, cudaStream_t s);
int launch_finish_sum2(double* a, double* b, int count, cudaStream_t s);

// the largest grid a reduction may use (partials must fit in DP_REDUCE_DOUBLES - 1)
constexpr int kMaxReduceBlocks = DP_REDUCE_DOUBLES - 1;

}  // namespace dpb
