// tcgen05 tensor-core GEMMs for the Poisson solve (TF32, BF16, split-BF16).
//
// C[m,n] = sum_k A[m,k] * B[n,k], A and B K-contiguous in global memory.
// One CTA computes a 128 x BN tile (BN = 64 or 128): TMA (128-byte swizzle, no multicast)
// stages A and B k-blocks into a STAGES-deep shared-memory ring, one thread
// issues tcgen05.mma (M=128, N=BN) into a TMEM accumulator, and all eight
// warps read the accumulator back with tcgen05.ld for the fused epilogue
// (transposed operand store with bf16 hi/lo split, spectral scaling, fp32
// field store, or the energy dot product; epilogue.cuh).
//
// Split-BF16 stages A_hi, A_lo, B_hi and B_lo of one k-block together and
// issues A_hi*B_hi, A_hi*B_lo and A_lo*B_hi on them into the same accumulator
// (the lo*lo term is below fp32 rounding), so every operand tile crosses L2
// once per k-block instead of once per product.
//
// Every wait on an mbarrier is bounded by a clock budget; on expiry the
// kernel records an error code in g_tc_status, drains what it issued and
// returns, so a broken launch reports instead of hanging the GPU.
#include <cuda.h>
#include <cstdlib>
#include "epilogue.cuh"

namespace dpb {

__device__ int g_tc_status = 0;
// bound of every mbarrier wait, in SM clock cycles (dp_tc_set_wait_budget)
__device__ long long g_tc_wait_budget = 4000000000ll;  // ~2 s at 2 GHz
// test hook (dp_tc_set_skip_loads): the producer issues no copy, so the MMA
// warp's bounded wait on the first stage runs out and the kernel reports it
__device__ int g_tc_skip_loads = 0;

constexpr int TC_BM = 128;
constexpr int TC_THREADS = 256;  // 8 warps: producer, MMA issuer, and all 8 in the epilogue

struct TcBatch {
  CUtensorMap a_hi[3];
  CUtensorMap a_lo[3];
  CUtensorMap b_hi[3];
  CUtensorMap b_lo[3];
  EpiParams epi[3];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; returns false (and records `code`) when the budget runs out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long start = clock64();
  const long long budget = g_tc_wait_budget;
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - start > budget) {
      atomicCAS(&g_tc_status, 0, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_addr(dst)), "l"(map), "r"(smem_addr(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <bool kTF32>
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  if (kTF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor: K-major operand tile in the 128-byte
// swizzle layout TMA writes (rows of 128 B, 8-row atoms of 1024 B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address, bits [0,14)
  d |= (uint64_t)1 << 16;                     // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;           // stride byte offset: 8-row group pitch
  d |= (uint64_t)1 << 46;                     // descriptor version (tcgen05)
  d |= (uint64_t)2 << 61;                     // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D fp32, A/B bf16 (1) or tf32 (2), both K-major, M=128, N=BN.
template <bool kTF32, int BN>
__host__ __device__ constexpr uint32_t make_idesc() {
  return (1u << 4)                                   // D format fp32
         | ((kTF32 ? 2u : 1u) << 7)                  // A format
         | ((kTF32 ? 2u : 1u) << 10)                 // B format
         | ((uint32_t)(BN >> 3) << 17)               // N >> 3
         | ((uint32_t)(TC_BM >> 4) << 24);           // M >> 4
}

template <int PREC, int BN, int STAGES>
struct TcConfig {
  static constexpr bool kTF32 = PREC == DP_PREC_TF32;
  static constexpr bool kSplit = PREC == DP_PREC_SPLIT_BF16;
  static constexpr int kElem = kTF32 ? 4 : 2;
  static constexpr int kBK = 128 / kElem;                 // elements per 128-byte row
  static constexpr int kMmaK = 32 / kElem;                // K per tcgen05.mma
  static constexpr int kMmaPerBlock = kBK / kMmaK;        // = 4
  static constexpr int kABytes = TC_BM * 128;
  static constexpr int kBBytes = BN * 128;
  // stage layout: A_hi | B_hi (| A_lo | B_lo for split-BF16)
  static constexpr int kStageBytes = (kSplit ? 2 : 1) * (kABytes + kBBytes);
  static constexpr int kSmemBytes = STAGES * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
  // the epilogue stages the 128 x BN accumulator (padded rows) in the ring
  static_assert(STAGES * kStageBytes >= (BN + 4) * TC_BM * 4 && STAGES * kStageBytes >= (TC_BM + 4) * BN * 4,
                "operand ring too small for the epilogue staging tile");
};

template <int PREC, int BN, int STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm_kernel(const __grid_constant__ TcBatch batch, int M,
                                                                 int N, int K, const int* __restrict__ gate) {
  grid_dep_sync();
  // a closed trial gate (dp_set_trial_gate): every thread of every CTA returns
  // before any barrier, TMEM allocation or copy is set up
  if (gate_closed(gate)) return;
  using Cfg = TcConfig<PREC, BN, STAGES>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* tiles = smem;
  uint64_t* full_bar = (uint64_t*)(smem + STAGES * Cfg::kStageBytes);
  uint64_t* empty_bar = full_bar + STAGES;
  uint64_t* acc_bar = empty_bar + STAGES;
  uint32_t* tmem_slot = (uint32_t*)(acc_bar + 1);

  const int z = blockIdx.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;
  const int total_kb = (K + Cfg::kBK - 1) / Cfg::kBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&batch.a_hi[z]) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&batch.b_hi[z]) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    const int skip = g_tc_skip_loads;
    for (int kb = 0; kb < total_kb && !skip; ++kb) {
      int s = kb % STAGES, round = kb / STAGES;
      if (round > 0 && !mbar_wait(&empty_bar[s], (round - 1) & 1, 1)) break;
      const int kx = kb * Cfg::kBK;
      uint8_t* sa = tiles + s * Cfg::kStageBytes;
      uint8_t* sb = sa + Cfg::kABytes;
      mbar_expect_tx(&full_bar[s], Cfg::kStageBytes);
      tma_load_2d(sa, &batch.a_hi[z], &full_bar[s], kx, m0);
      tma_load_2d(sb, &batch.b_hi[z], &full_bar[s], kx, n0);
      if (Cfg::kSplit) {
        tma_load_2d(sb + Cfg::kBBytes, &batch.a_lo[z], &full_bar[s], kx, m0);
        tma_load_2d(sb + Cfg::kBBytes + Cfg::kABytes, &batch.b_lo[z], &full_bar[s], kx, n0);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    constexpr uint32_t idesc = make_idesc<Cfg::kTF32, BN>();
    for (int kb = 0; kb < total_kb; ++kb) {
      int s = kb % STAGES, round = kb / STAGES;
      if (!mbar_wait(&full_bar[s], round & 1, 2)) break;
      tc_fence_after();
      uint32_t sa = smem_addr(tiles + s * Cfg::kStageBytes);
      uint32_t sb = sa + Cfg::kABytes;
      const uint64_t adesc = sw128_desc(sa), bdesc = sw128_desc(sb);
      const uint64_t alo = sw128_desc(sb + Cfg::kBBytes), blo = sw128_desc(sb + Cfg::kBBytes + Cfg::kABytes);
#pragma unroll
      for (int kk = 0; kk < Cfg::kMmaPerBlock; ++kk) {
        // advance the start address by 32 bytes per K step inside the swizzle row
        const uint64_t dk = (uint64_t)(kk * 2);
        tc_mma<Cfg::kTF32>(tmem_base, adesc + dk, bdesc + dk, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
        if (Cfg::kSplit) {
          tc_mma<Cfg::kTF32>(tmem_base, adesc + dk, blo + dk, idesc, 1u);
          tc_mma<Cfg::kTF32>(tmem_base, alo + dk, bdesc + dk, idesc, 1u);
        }
      }
      tc_commit(&empty_bar[s]);  // frees the stage once these MMAs retire
    }
    tc_commit(acc_bar);  // accumulator complete (also on the error path: drains issued MMAs)
  }
  __syncwarp();

  // ---- epilogue ----
  // The accumulator is staged through shared memory (the operand ring is
  // drained once the accumulator is complete) in the orientation of the output
  // rows, then every thread applies the epilogue to 8 consecutive elements of
  // one output row, so each warp store covers whole row segments instead of
  // one element of 32 different rows.
  const EpiParams& P = batch.epi[z];
  const bool acc_ok = mbar_wait(acc_bar, 0, 3);
  double e = 0.0;
  if (__syncthreads_and(acc_ok)) {
    tc_fence_after();
    const bool trans = P.kind == DP_EPI_STORE_T;
    float* stage = reinterpret_cast<float*>(tiles);
    constexpr int kRowPitch = BN + 4;     // stage[m][n] for row-major outputs
    constexpr int kColPitch = TC_BM + 4;  // stage[n][m] for STORE_T
    // a warp reads the TMEM lane quarter (warp % 4) it may access, and half of
    // the columns (warp / 4)
    const int quarter = warp & 3, half = warp >> 2;
    const int r_acc = quarter * 32 + lane;  // accumulator row = TMEM lane
    const uint32_t row_addr = tmem_base + ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
    for (int c = half * (BN / 2); c < (half + 1) * (BN / 2); c += 16) {
      float v[16];
      tmem_ld16(row_addr + (uint32_t)c, v);
      if (trans) {
#pragma unroll
        for (int j = 0; j < 16; ++j) stage[(c + j) * kColPitch + r_acc] = v[j];
      } else {
        float4* d = reinterpret_cast<float4*>(stage + r_acc * kRowPitch + c);
#pragma unroll
        for (int q = 0; q < 4; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
    }
    __syncthreads();
    const int cols = trans ? TC_BM : BN;
    const int pitch = trans ? kColPitch : kRowPitch;
    const int segs = cols / 8;
#pragma unroll 1
    for (int i = threadIdx.x; i < (trans ? BN : TC_BM) * segs; i += TC_THREADS) {
      const int r = i / segs, c0 = (i % segs) * 8;
      float v[8];
      const float4* src = reinterpret_cast<const float4*>(stage + r * pitch + c0);
      const float4 a = src[0], b4 = src[1];
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b4.x; v[5] = b4.y; v[6] = b4.z; v[7] = b4.w;
      if (trans) {
        if (n0 + r < N) epi_store_t8(P, n0 + r, m0 + c0, v);
      } else {
        if (m0 + r < M) e += epi_row8(P, m0 + r, n0 + c0, v);
      }
    }
  }
  if (P.energy) {  // ENERGY, or SPECTRAL with the spectral-domain energy
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (lane == 0 && e != 0.0) atomicAdd(P.energy, e);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(BN) : "memory");
  }
}

// ---------------------------------------------------------------- host side

typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                     const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode_fn() {
  static PFN_encodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encodeTiled)p;
  }
  return fn;
}

// rows x K matrix, K contiguous, leading dimension ld (elements), box = box_rows x (128 bytes)
static int encode_operand(CUtensorMap* map, const void* ptr, int rows, int K, int ld, int elem_bytes,
                          int box_rows) {
  PFN_encodeTiled enc = get_encode_fn();
  DP_REQUIRE(enc, "dp_transform_gemm: cuTensorMapEncodeTiled unavailable");
  DP_REQUIRE(((uintptr_t)ptr & 15) == 0, "dp_transform_gemm: operand base must be 16-byte aligned");
  DP_REQUIRE(((long long)ld * elem_bytes) % 16 == 0, "dp_transform_gemm: operand row pitch must be a multiple of 16 bytes");
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * elem_bytes};
  cuuint32_t box[2] = {(cuuint32_t)(128 / elem_bytes), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                   const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  DP_REQUIRE(r == CUDA_SUCCESS, "dp_transform_gemm: cuTensorMapEncodeTiled failed (%d)", (int)r);
  return DP_OK;
}

template <int PREC, int BN, int STAGES>
static int run_tc(int M, int N, int K, const dp_gemm_problem* probs, int count, cudaStream_t s) {
  using Cfg = TcConfig<PREC, BN, STAGES>;
  static TcBatch batch;  // host staging; copied into the launch's parameter buffer
  memset(&batch, 0, sizeof(batch));
  for (int i = 0; i < count; ++i) {
    const dp_gemm_problem& q = probs[i];
    int rc = encode_operand(&batch.a_hi[i], q.a_hi, M, K, q.lda, Cfg::kElem, TC_BM);
    if (!rc) rc = encode_operand(&batch.b_hi[i], q.b_hi, N, K, q.ldb, Cfg::kElem, BN);
    if (!rc && Cfg::kSplit) rc = encode_operand(&batch.a_lo[i], q.a_lo, M, K, q.lda, Cfg::kElem, TC_BM);
    if (!rc && Cfg::kSplit) rc = encode_operand(&batch.b_lo[i], q.b_lo, N, K, q.ldb, Cfg::kElem, BN);
    if (rc) return rc;
    batch.epi[i] = make_epi(q, PREC, M, N);
  }
  auto kern = tc_gemm_kernel<PREC, BN, STAGES>;
  int rc_smem = opt_in_smem(kern, Cfg::kSmemBytes, "dp_transform_gemm");
  if (rc_smem) return rc_smem;
  dim3 grid(ceil_div(N, BN), ceil_div(M, TC_BM), count);
  launch_kernel(kern, grid, TC_THREADS, Cfg::kSmemBytes, s, batch, M, N, K, trial_gate());
  return check_launch("dp_transform_gemm(tcgen05)");
}

// Output tile width: a single transform runs 128 x 64 tiles (at 1024 x 1024
// that is 128 CTAs, where 128 x 128 tiles leave 84 of the 148 SMs idle); a
// batch of three runs 128 x 128 tiles (192 CTAs in two waves beat 384 in
// three).  DP_TC_TILE_N=64 or 128 forces one width.
static int tile_n(int count) {
  static int forced = [] {
    const char* e = getenv("DP_TC_TILE_N");
    return e ? atoi(e) : 0;
  }();
  if (forced == 64 || forced == 128) return forced;
  return count == 1 ? 64 : 128;
}

int launch_tc_gemm(int precision, int M, int N, int K, const dp_gemm_problem* probs, int count, cudaStream_t s) {
  const bool wide = tile_n(count) == 128;
  switch (precision) {
    // one CTA per SM; the TMA ring fills ~192 KB of shared memory: 32 KB or
    // 24 KB stages, or 64 KB / 48 KB stages holding the hi and lo planes of
    // both operands for split-BF16
    case DP_PREC_TF32:
      return wide ? run_tc<DP_PREC_TF32, 128, 6>(M, N, K, probs, count, s)
                  : run_tc<DP_PREC_TF32, 64, 8>(M, N, K, probs, count, s);
    case DP_PREC_BF16:
      return wide ? run_tc<DP_PREC_BF16, 128, 6>(M, N, K, probs, count, s)
                  : run_tc<DP_PREC_BF16, 64, 8>(M, N, K, probs, count, s);
    case DP_PREC_SPLIT_BF16:
      return wide ? run_tc<DP_PREC_SPLIT_BF16, 128, 3>(M, N, K, probs, count, s)
                  : run_tc<DP_PREC_SPLIT_BF16, 64, 4>(M, N, K, probs, count, s);
  }
  set_error("dp_transform_gemm: unsupported precision %d", precision);
  return DP_ERR_UNSUPPORTED;
}

}  // namespace dpb

// Reads and clears the device-side status word of the tensor-core kernels
// (0 = no bounded wait expired).  Synchronises the device.
extern "C" int dp_tc_status(int* status_out) {
  DP_REQUIRE(status_out, "dp_tc_status: null output");
  int zero = 0;
  cudaError_t e = cudaMemcpyFromSymbol(status_out, dpb::g_tc_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(dpb::g_tc_status, &zero, sizeof(int));
  if (e != cudaSuccess) {
    dpb::set_error("dp_tc_status: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  return DP_OK;
}

extern "C" int dp_tc_set_wait_budget(long long cycles) {
  DP_REQUIRE(cycles > 0, "dp_tc_set_wait_budget: the budget must be positive");
  cudaError_t e = cudaMemcpyToSymbol(dpb::g_tc_wait_budget, &cycles, sizeof(long long));
  if (e != cudaSuccess) {
    dpb::set_error("dp_tc_set_wait_budget: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  return DP_OK;
}

extern "C" int dp_tc_set_skip_loads(int skip) {
  const int v = skip ? 1 : 0;
  cudaError_t e = cudaMemcpyToSymbol(dpb::g_tc_skip_loads, &v, sizeof(int));
  if (e != cudaSuccess) {
    dpb::set_error("dp_tc_set_skip_loads: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  return DP_OK;
}
