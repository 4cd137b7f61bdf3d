// The 2-D DCT family as dense GEMMs: C[m,n] = sum_k A[m,k] * B[n,k].
//
// The reference computes DCT2 / IDCT2 / IDCT_IDXST / IDXST_IDCT through a
// real FFT with pre/post twiddle kernels (dct/src/dct2_fft2_cuda_kernel.cu).
// Here each 2-D transform is two GEMMs against precomputed cosine / sine
// matrices (dct2_fft2(x) = 4/(MN) C_M x C_N^T, idct2(y) = 4 C^_M y C^_N^T,
// idct_idxst(y) = 4 C^_M y S^_N^T, idxst_idct(y) = 4 S^_M y C^_N^T), so the
// whole Poisson solve is matrix products that map onto tcgen05.
//
// This file holds the fp32 SIMT kernel (the plain form, DP_PREC_FP32), the
// operand preparation kernel and the precision dispatcher; the tensor-core
// kernels are in gemm_tc.cu.
#include "epilogue.cuh"

namespace dpb {

int launch_tc_gemm(int precision, int M, int N, int K, const dp_gemm_problem* probs, int count,
                   cudaStream_t stream);

struct SimtProblem {
  const float* A;
  const float* B;
  int lda, ldb;
  EpiParams epi;
};
struct SimtBatch {
  SimtProblem p[3];
};

// 128 x 64 output tile, K step 16, 256 threads, 8 x 4 outputs per thread,
// shared-memory double buffering with register prefetch.
constexpr int SBM = 128, SBN = 64, SBK = 16;

__global__ void __launch_bounds__(256) simt_gemm_kernel(SimtBatch batch, int M, int N, int K,
                                                        const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  const SimtProblem& P = batch.p[blockIdx.z];
  __shared__ float As[2][SBK][SBM + 4];
  __shared__ float Bs[2][SBK][SBN + 4];
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * SBM, n0 = blockIdx.x * SBN;
  const int tx = tid & 15, ty = tid >> 4;  // 16 x 16 thread grid
  // loaders: A tile 128 rows x 16 k = 512 float4 (2 per thread); B tile 64 x 16 = 256 float4
  const int a_row0 = tid >> 2, a_kq = (tid & 3) * 4;  // rows a_row0 and a_row0+64
  const int b_row = tid >> 2, b_kq = (tid & 3) * 4;
  float acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;

  auto load_a = [&](int kt, int r) -> float4 {
    int m = m0 + a_row0 + r * 64, k = kt + a_kq;
    if (m < M && k + 3 < K) return *reinterpret_cast<const float4*>(P.A + (size_t)m * P.lda + k);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m < M) {
      if (k < K) v.x = P.A[(size_t)m * P.lda + k];
      if (k + 1 < K) v.y = P.A[(size_t)m * P.lda + k + 1];
      if (k + 2 < K) v.z = P.A[(size_t)m * P.lda + k + 2];
      if (k + 3 < K) v.w = P.A[(size_t)m * P.lda + k + 3];
    }
    return v;
  };
  auto load_b = [&](int kt) -> float4 {
    int n = n0 + b_row, k = kt + b_kq;
    if (n < N && k + 3 < K) return *reinterpret_cast<const float4*>(P.B + (size_t)n * P.ldb + k);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (n < N) {
      if (k < K) v.x = P.B[(size_t)n * P.ldb + k];
      if (k + 1 < K) v.y = P.B[(size_t)n * P.ldb + k + 1];
      if (k + 2 < K) v.z = P.B[(size_t)n * P.ldb + k + 2];
      if (k + 3 < K) v.w = P.B[(size_t)n * P.ldb + k + 3];
    }
    return v;
  };
  auto store_tiles = [&](int buf, float4 a0, float4 a1, float4 b0) {
    As[buf][a_kq + 0][a_row0] = a0.x;
    As[buf][a_kq + 1][a_row0] = a0.y;
    As[buf][a_kq + 2][a_row0] = a0.z;
    As[buf][a_kq + 3][a_row0] = a0.w;
    As[buf][a_kq + 0][a_row0 + 64] = a1.x;
    As[buf][a_kq + 1][a_row0 + 64] = a1.y;
    As[buf][a_kq + 2][a_row0 + 64] = a1.z;
    As[buf][a_kq + 3][a_row0 + 64] = a1.w;
    Bs[buf][b_kq + 0][b_row] = b0.x;
    Bs[buf][b_kq + 1][b_row] = b0.y;
    Bs[buf][b_kq + 2][b_row] = b0.z;
    Bs[buf][b_kq + 3][b_row] = b0.w;
  };

  int ktiles = (K + SBK - 1) / SBK;
  {
    float4 a0 = load_a(0, 0), a1 = load_a(0, 1), b0 = load_b(0);
    store_tiles(0, a0, a1, b0);
  }
  __syncthreads();
  for (int t = 0; t < ktiles; ++t) {
    int buf = t & 1;
    float4 na0, na1, nb0;
    bool more = t + 1 < ktiles;
    if (more) {
      na0 = load_a((t + 1) * SBK, 0);
      na1 = load_a((t + 1) * SBK, 1);
      nb0 = load_b((t + 1) * SBK);
    }
#pragma unroll
    for (int kk = 0; kk < SBK; ++kk) {
      float a[8], b[4];
      float4 av0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
      float4 av1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
      float4 bv = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
      a[0] = av0.x; a[1] = av0.y; a[2] = av0.z; a[3] = av0.w;
      a[4] = av1.x; a[5] = av1.y; a[6] = av1.z; a[7] = av1.w;
      b[0] = bv.x; b[1] = bv.y; b[2] = bv.z; b[3] = bv.w;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (more) store_tiles(buf ^ 1, na0, na1, nb0);
    __syncthreads();
  }
  // epilogue: rows ty*4 + {0..3} and 64 + ty*4 + {0..3}; cols tx*4 + {0..3}
  double e = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int n = n0 + tx * 4 + j;
      if (n < N) e += epi_apply(P.epi, m, n, acc[i][j]);
    }
  }
  if (P.epi.energy) {  // ENERGY, or SPECTRAL with the spectral-domain energy
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    __shared__ double red[8];
    if ((tid & 31) == 0) red[tid >> 5] = e;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int w = 0; w < 8; ++w) s += red[w];
      atomicAdd(P.epi.energy, s);
    }
  }
}

template <int FMT>
__global__ void prepare_operand_kernel(const float* __restrict__ x, size_t n, float scale,
                                       float* __restrict__ f32, __nv_bfloat16* __restrict__ hi,
                                       __nv_bfloat16* __restrict__ lo, const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float v = __fmul_rn(x[i], scale);
    store_operand(FMT, v, i, f32, hi, lo);
  }
}

}  // namespace dpb

using namespace dpb;

extern "C" int dp_transform_gemm(int precision, int M, int N, int K, const dp_gemm_problem* probs,
                                 int count, dp_stream_t stream) {
  DP_REQUIRE(probs && count >= 1 && count <= 3, "dp_transform_gemm: count must be 1..3");
  DP_REQUIRE(M > 0 && N > 0 && K > 0, "dp_transform_gemm: bad sizes %d x %d x %d", M, N, K);
  DP_REQUIRE(precision >= DP_PREC_FP32 && precision <= DP_PREC_SPLIT_BF16, "dp_transform_gemm: bad precision %d", precision);
  for (int i = 0; i < count; ++i) {
    int rc = validate_problem(probs[i], precision, M, N, K);
    if (rc) return rc;
  }
  cudaStream_t s = as_stream(stream);
  if (precision != DP_PREC_FP32) return launch_tc_gemm(precision, M, N, K, probs, count, s);
  SimtBatch b;
  memset(&b, 0, sizeof(b));
  for (int i = 0; i < count; ++i) {
    b.p[i].A = (const float*)probs[i].a_hi;
    b.p[i].B = (const float*)probs[i].b_hi;
    b.p[i].lda = probs[i].lda;
    b.p[i].ldb = probs[i].ldb;
    b.p[i].epi = make_epi(probs[i], precision, M, N);
    DP_REQUIRE(((uintptr_t)probs[i].a_hi & 15) == 0 && ((uintptr_t)probs[i].b_hi & 15) == 0 &&
                   (probs[i].lda % 4) == 0 && (probs[i].ldb % 4) == 0,
               "dp_transform_gemm: fp32 operands need 16-byte aligned rows");
  }
  dim3 grid(ceil_div(N, SBN), ceil_div(M, SBM), count);
  launch_kernel(simt_gemm_kernel, grid, 256, 0, s, b, M, N, K, trial_gate());
  return check_launch("dp_transform_gemm(fp32)");
}

extern "C" int dp_prepare_operand(int precision, const float* x, size_t n, float scale, float* out_f32,
                                  void* out_hi, void* out_lo, dp_stream_t stream) {
  DP_REQUIRE(x, "dp_prepare_operand: null input");
  int fmt = operand_fmt(precision);
  DP_REQUIRE(fmt == kFmtF32 ? out_f32 != nullptr : out_hi != nullptr, "dp_prepare_operand: output missing");
  DP_REQUIRE(fmt != kFmtSplit || out_lo, "dp_prepare_operand: split output needs out_lo");
  if (n == 0) return DP_OK;
  cudaStream_t s = as_stream(stream);
  int g = grid_for((long long)n, 256, 8);
  if (fmt == kFmtF32)
    launch_kernel(prepare_operand_kernel<kFmtF32>, g, 256, 0, s, x, n, scale, out_f32, nullptr, nullptr, trial_gate());
  else if (fmt == kFmtBF16)
    launch_kernel(prepare_operand_kernel<kFmtBF16>, g, 256, 0, s, x, n, scale, nullptr, (__nv_bfloat16*)out_hi, nullptr,
                                                       trial_gate());
  else
    launch_kernel(prepare_operand_kernel<kFmtSplit>, g, 256, 0, s, x, n, scale, nullptr, (__nv_bfloat16*)out_hi,
                                                        (__nv_bfloat16*)out_lo, trial_gate());
  return check_launch("dp_prepare_operand");
}

namespace dpb {
__global__ void spectral_table_kernel(EpiParams p, float* out) {
  grid_dep_sync();
  const size_t mn = (size_t)p.M * p.N;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < mn; t += (size_t)gridDim.x * blockDim.x) {
    float wx, wy, wi;
    spectral_weights(p, (int)(t / p.N), (int)(t % p.N), wx, wy, wi);
    out[t] = wx;
    out[mn + t] = wy;
    out[2 * mn + t] = wi;
  }
}
}  // namespace dpb

extern "C" int dp_spectral_weights(int M, int N, float wv_scale, float* out, dp_stream_t stream) {
  DP_REQUIRE(M > 0 && N > 0 && out, "dp_spectral_weights: bad arguments");
  dp_gemm_problem q;
  memset(&q, 0, sizeof(q));
  q.epilogue = DP_EPI_SPECTRAL;
  q.wv_scale = wv_scale;
  EpiParams e = make_epi(q, DP_PREC_FP32, M, N);
  launch_kernel(spectral_table_kernel, grid_for((long long)M * N, 256, 8), 256, 0, as_stream(stream), e, out);
  return check_launch("dp_spectral_weights");
}
