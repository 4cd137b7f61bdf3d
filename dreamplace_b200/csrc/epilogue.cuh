// Epilogues of the Poisson-solve GEMMs, shared by the SIMT (fp32) and the
// tcgen05 (tf32 / bf16 / split-bf16) kernels.  Each epilogue consumes one
// output element value v = alpha * C[m,n] at (m, n).
#pragma once
#include "common.cuh"

namespace dpb {

// operand storage formats of a GEMM input / intermediate
enum OperandFmt { kFmtF32 = 0, kFmtBF16 = 1, kFmtSplit = 2 };

inline int operand_fmt(int precision) {
  switch (precision) {
    case DP_PREC_BF16: return kFmtBF16;
    case DP_PREC_SPLIT_BF16: return kFmtSplit;
    default: return kFmtF32;
  }
}

struct EpiParams {
  int kind;  // DP_EPI_*
  float alpha;
  int ldc;
  int fmt;  // OperandFmt of operand-typed outputs (STORE_T, SPECTRAL)
  int M, N;
  float* out_f32;
  __nv_bfloat16* out_hi;
  __nv_bfloat16* out_lo;
  float* sp_f32[3];
  __nv_bfloat16* sp_hi[3];
  __nv_bfloat16* sp_lo[3];
  float wv_scale;
  float two_pi_over_m, two_pi_over_n;
  const float* spec_w;  // optional precomputed spectral tables [3*M*N]
  const float* rho;
  double* energy;
};

__device__ __forceinline__ void store_operand(int fmt, float v, size_t idx, float* f32,
                                              __nv_bfloat16* hi, __nv_bfloat16* lo) {
  if (fmt == kFmtF32) {
    f32[idx] = v;
  } else {
    __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[idx] = h;
    if (fmt == kFmtSplit) lo[idx] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

// Spectral weights as the reference builds them in fp32
// (electric_potential/electric_potential.py:504-519):
//   wu = u*(2pi/M); wv = v*(2pi/N)*(bsx/bsy); d = wu^2 + wv^2 (1 at [0,0]);
//   inv = 1/d (0 at [0,0]); wx = wu*inv*0.5; wy = wv*inv*0.5
__device__ __forceinline__ void spectral_weights(const EpiParams& p, int u, int v, float& wx,
                                                 float& wy, float& winv) {
  float wu = __fmul_rn((float)u, p.two_pi_over_m);
  float wv = __fmul_rn(__fmul_rn((float)v, p.two_pi_over_n), p.wv_scale);
  float d = __fadd_rn(__fmul_rn(wu, wu), __fmul_rn(wv, wv));
  if (u == 0 && v == 0) d = 1.0f;
  float inv = __fdiv_rn(1.0f, d);
  if (u == 0 && v == 0) inv = 0.0f;
  winv = inv;
  wx = __fmul_rn(__fmul_rn(wu, inv), 0.5f);
  wy = __fmul_rn(__fmul_rn(wv, inv), 0.5f);
}

// Energy term of one spectral coefficient a = v at (u, v_idx):
//   sum_xy rho * IDCT2(a * winv) = M N sum_uv w_u w_v winv_uv a_uv^2,
// w_0 = 1/2, w_k = 1 otherwise (the DCT-II / DCT-III pair of the transforms),
// so the potential map is never formed.
__device__ __forceinline__ double spectral_energy(const EpiParams& p, int u, int vi, float a, float winv) {
  const double w = (u == 0 ? 0.5 : 1.0) * (vi == 0 ? 0.5 : 1.0);
  return (double)p.M * (double)p.N * w * (double)winv * (double)a * (double)a;
}

// Applies the epilogue to one element.  Returns the contribution to the
// energy dot product (ENERGY) or 0.
__device__ __forceinline__ double epi_apply(const EpiParams& p, int m, int n, float acc) {
  float v = __fmul_rn(acc, p.alpha);
  switch (p.kind) {
    case DP_EPI_STORE:
      p.out_f32[(size_t)m * p.ldc + n] = v;
      return 0.0;
    case DP_EPI_STORE_T:
      store_operand(p.fmt, v, (size_t)n * p.ldc + m, p.out_f32, p.out_hi, p.out_lo);
      return 0.0;
    case DP_EPI_SPECTRAL: {
      float wx, wy, winv;
      size_t idx = (size_t)m * p.ldc + n;
      if (p.spec_w) {
        size_t t = (size_t)m * p.N + n, mn = (size_t)p.M * p.N;
        wx = p.spec_w[t];
        wy = p.spec_w[mn + t];
        winv = p.spec_w[2 * mn + t];
      } else {
        spectral_weights(p, m, n, wx, wy, winv);
      }
      store_operand(p.fmt, __fmul_rn(v, wx), idx, p.sp_f32[0], p.sp_hi[0], p.sp_lo[0]);
      store_operand(p.fmt, __fmul_rn(v, wy), idx, p.sp_f32[1], p.sp_hi[1], p.sp_lo[1]);
      if (p.sp_f32[2] || p.sp_hi[2])
        store_operand(p.fmt, __fmul_rn(v, winv), idx, p.sp_f32[2], p.sp_hi[2], p.sp_lo[2]);
      return p.energy ? spectral_energy(p, m, n, v, winv) : 0.0;
    }
    case DP_EPI_ENERGY: {
      size_t idx = (size_t)m * p.ldc + n;
      if (p.out_f32) p.out_f32[idx] = v;
      return (double)__fmul_rn(v, p.rho[idx]);
    }
  }
  return 0.0;
}

// Host: builds the device-side epilogue parameters from a public problem.
inline EpiParams make_epi(const dp_gemm_problem& q, int precision, int M, int N) {
  EpiParams e;
  memset(&e, 0, sizeof(e));
  e.kind = q.epilogue;
  e.alpha = q.alpha;
  e.ldc = q.ldc;
  e.fmt = operand_fmt(precision);
  e.M = M;
  e.N = N;
  e.out_f32 = q.out_f32;
  e.out_hi = (__nv_bfloat16*)q.out_hi;
  e.out_lo = (__nv_bfloat16*)q.out_lo;
  for (int i = 0; i < 3; ++i) {
    e.sp_f32[i] = q.spec_out_f32[i];
    e.sp_hi[i] = (__nv_bfloat16*)q.spec_out_hi[i];
    e.sp_lo[i] = (__nv_bfloat16*)q.spec_out_lo[i];
  }
  e.wv_scale = q.wv_scale;
  e.two_pi_over_m = (float)(2.0 * M_PI / M);
  e.two_pi_over_n = (float)(2.0 * M_PI / N);
  e.rho = q.rho;
  e.energy = q.energy_f64;
  e.spec_w = q.spec_weights;
  return e;
}

// ---- 8 consecutive elements of one output row (staged epilogue of the
// tcgen05 kernel).  Same per-element arithmetic as epi_apply; vector memory
// operations where the addresses are 16-byte aligned, scalar otherwise.
__device__ __forceinline__ bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

__device__ __forceinline__ void store_operand8(int fmt, const float* v, size_t idx, float* f32,
                                               __nv_bfloat16* hi, __nv_bfloat16* lo) {
  if (fmt == kFmtF32) {
    float* d = f32 + idx;
    if (aligned16(d)) {
      reinterpret_cast<float4*>(d)[0] = make_float4(v[0], v[1], v[2], v[3]);
      reinterpret_cast<float4*>(d)[1] = make_float4(v[4], v[5], v[6], v[7]);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) d[j] = v[j];
    }
    return;
  }
  __align__(16) __nv_bfloat16 h[8];
  __align__(16) __nv_bfloat16 l[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    h[j] = __float2bfloat16_rn(v[j]);
    l[j] = __float2bfloat16_rn(v[j] - __bfloat162float(h[j]));
  }
  __nv_bfloat16* dh = hi + idx;
  if (aligned16(dh)) {
    *reinterpret_cast<uint4*>(dh) = *reinterpret_cast<const uint4*>(h);
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) dh[j] = h[j];
  }
  if (fmt == kFmtSplit) {
    __nv_bfloat16* dl = lo + idx;
    if (aligned16(dl)) {
      *reinterpret_cast<uint4*>(dl) = *reinterpret_cast<const uint4*>(l);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) dl[j] = l[j];
    }
  }
}

__device__ __forceinline__ void load8(const float* src, float* v) {
  if (aligned16(src)) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(src));
    const float4 b = __ldg(reinterpret_cast<const float4*>(src) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = __ldg(src + j);
  }
}

// row-major kinds (STORE, SPECTRAL, ENERGY): elements (m, n0 .. n0+7)
__device__ __forceinline__ double epi_row8(const EpiParams& p, int m, int n0, const float* acc) {
  if (n0 + 8 > p.N) {
    double e = 0.0;
    for (int j = 0; j < 8 && n0 + j < p.N; ++j) e += epi_apply(p, m, n0 + j, acc[j]);
    return e;
  }
  float v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = __fmul_rn(acc[j], p.alpha);
  const size_t idx = (size_t)m * p.ldc + n0;
  switch (p.kind) {
    case DP_EPI_STORE:
      store_operand8(kFmtF32, v, idx, p.out_f32, nullptr, nullptr);
      return 0.0;
    case DP_EPI_SPECTRAL: {
      float wx[8], wy[8], wi[8];
      if (p.spec_w) {
        const size_t t = (size_t)m * p.N + n0, mn = (size_t)p.M * p.N;
        load8(p.spec_w + t, wx);
        load8(p.spec_w + mn + t, wy);
        load8(p.spec_w + 2 * mn + t, wi);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) spectral_weights(p, m, n0 + j, wx[j], wy[j], wi[j]);
      }
      float o[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = __fmul_rn(v[j], wx[j]);
      store_operand8(p.fmt, o, idx, p.sp_f32[0], p.sp_hi[0], p.sp_lo[0]);
#pragma unroll
      for (int j = 0; j < 8; ++j) o[j] = __fmul_rn(v[j], wy[j]);
      store_operand8(p.fmt, o, idx, p.sp_f32[1], p.sp_hi[1], p.sp_lo[1]);
      if (p.sp_f32[2] || p.sp_hi[2]) {
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = __fmul_rn(v[j], wi[j]);
        store_operand8(p.fmt, o, idx, p.sp_f32[2], p.sp_hi[2], p.sp_lo[2]);
      }
      double e = 0.0;
      if (p.energy) {
#pragma unroll
        for (int j = 0; j < 8; ++j) e += spectral_energy(p, m, n0 + j, v[j], wi[j]);
      }
      return e;
    }
    case DP_EPI_ENERGY: {
      float r[8];
      load8(p.rho + idx, r);
      double e = 0.0;
#pragma unroll
      for (int j = 0; j < 8; ++j) e += (double)__fmul_rn(v[j], r[j]);
      if (p.out_f32) store_operand8(kFmtF32, v, idx, p.out_f32, nullptr, nullptr);
      return e;
    }
  }
  return 0.0;
}

// STORE_T: elements (m0 .. m0+7, n), written to [n*ldc + m]
__device__ __forceinline__ void epi_store_t8(const EpiParams& p, int n, int m0, const float* acc) {
  if (m0 + 8 > p.M) {
    for (int j = 0; j < 8 && m0 + j < p.M; ++j) epi_apply(p, m0 + j, n, acc[j]);
    return;
  }
  float v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = __fmul_rn(acc[j], p.alpha);
  store_operand8(p.fmt, v, (size_t)n * p.ldc + m0, p.out_f32, p.out_hi, p.out_lo);
}

inline int validate_problem(const dp_gemm_problem& q, int precision, int M, int N, int K) {
  DP_REQUIRE(q.a_hi && q.b_hi, "dp_transform_gemm: null operand");
  DP_REQUIRE(precision != DP_PREC_SPLIT_BF16 || (q.a_lo && q.b_lo),
             "dp_transform_gemm: split-bf16 needs lo operands");
  DP_REQUIRE(q.lda >= K && q.ldb >= K, "dp_transform_gemm: leading dimension smaller than K");
  int fmt = operand_fmt(precision);
  switch (q.epilogue) {
    case DP_EPI_STORE:
      DP_REQUIRE(q.out_f32 && q.ldc >= N, "dp_transform_gemm: STORE needs out_f32 and ldc >= N");
      break;
    case DP_EPI_STORE_T:
      DP_REQUIRE(q.ldc >= M, "dp_transform_gemm: STORE_T needs ldc >= M");
      DP_REQUIRE(fmt == kFmtF32 ? q.out_f32 != nullptr : q.out_hi != nullptr,
                 "dp_transform_gemm: STORE_T output missing");
      DP_REQUIRE(fmt != kFmtSplit || q.out_lo, "dp_transform_gemm: STORE_T split output needs out_lo");
      break;
    case DP_EPI_SPECTRAL:
      DP_REQUIRE(q.ldc >= N, "dp_transform_gemm: SPECTRAL needs ldc >= N");
      for (int i = 0; i < 2; ++i) {
        DP_REQUIRE(fmt == kFmtF32 ? q.spec_out_f32[i] != nullptr : q.spec_out_hi[i] != nullptr,
                   "dp_transform_gemm: SPECTRAL output %d missing", i);
        DP_REQUIRE(fmt != kFmtSplit || q.spec_out_lo[i], "dp_transform_gemm: SPECTRAL lo output %d missing", i);
      }
      DP_REQUIRE(fmt != kFmtSplit || !q.spec_out_hi[2] || q.spec_out_lo[2],
                 "dp_transform_gemm: SPECTRAL lo output 2 missing");
      break;
    case DP_EPI_ENERGY:
      DP_REQUIRE(q.rho && q.energy_f64 && q.ldc >= N, "dp_transform_gemm: ENERGY needs rho and energy_f64");
      break;
    default:
      DP_REQUIRE(false, "dp_transform_gemm: unknown epilogue %d", q.epilogue);
  }
  return DP_OK;
}

}  // namespace dpb
