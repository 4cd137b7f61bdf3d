// Fused kernels of one global-placement iteration (the engine path).
//
// The reference composes an iteration from separate ops: pin_pos -> WA ->
// (autograd) WA backward -> pin_pos backward, HPWL through pin_pos, and the
// Nesterov update as a dozen tensor expressions
// (dreamplace/NesterovAcceleratedGradientOptimizer.py:65-166,
// dreamplace/PlaceObj.py:37-132).  Here:
//
//  * pins are visited in "slot" order (the flat_netpin order): per slot the
//    owning node and the pin offsets are stored contiguously, so the WA and
//    HPWL kernels gather node positions (resident in L2) instead of reading a
//    materialised pin-position array;
//  * WA backward and the pin -> node sum are one gather over a node -> slot
//    CSR, in the reference's per-node pin order, so the node gradient equals
//    pin_pos backward of the reference's per-pin gradient bit for bit;
//  * the Nesterov trial point, the move-boundary clamp, the preconditioner
//    and both step-size norms (fp64) are two streaming passes over the
//    position / gradient vectors, and a one-thread kernel finishes the step
//    size, the backtracking test and the momentum scalars on the device.
#include <vector>
#include <climits>
#include "reduce.cuh"

namespace dpb {

// two-value block partial: partials[blockIdx.x], partials[gridDim.x + blockIdx.x]
__device__ __forceinline__ void block_partial2(double a, double b, double* partials) {
  __shared__ double sa[kReduceThreads / 32], sb[kReduceThreads / 32];
  a = warp_sum(a);
  b = warp_sum(b);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int i = 0; i < kReduceThreads / 32; ++i) { ta += sa[i]; tb += sb[i]; }
    partials[blockIdx.x] = ta;
    partials[gridDim.x + blockIdx.x] = tb;
  }
}

// ---------------------------------------------------------------- Nesterov
// Device scalars of the optimizer (one array of doubles):
enum {
  NS_ALPHA = 0,      // alpha_k (step size, updated by every trial)
  NS_A = 1,          // a_k
  NS_A_NEXT = 2,     // a_{k+1}
  NS_COEF = 3,       // (a_k - 1) / a_{k+1}
  NS_ACC_DV = 4,     // sum (v_{k+1} - v_k)^2 accumulator
  NS_ACC_DG = 5,     // sum (g_{k+1} - g_k)^2 accumulator
  NS_ALPHA_NEW = 6,  // alpha_{k+1}
  NS_ACCEPT = 7,     // 1.0 when alpha_{k+1} > 0.95 alpha_k
  NS_COUNT = 8
};

// u' = v - alpha g; v' = u' + coef (u' - u); v' clamped into the die for
// movable and filler nodes (move_boundary semantics); one thread per node
// also writes the interleaved copy xy' used by the gather kernels.
__global__ void nesterov_trial_kernel(const float* __restrict__ v, const float* __restrict__ g,
                                      const float* __restrict__ u, float* __restrict__ u_new,
                                      float* __restrict__ v_new, float2* __restrict__ xy_new,
                                      const double* __restrict__ st, const float* __restrict__ sx,
                                      const float* __restrict__ sy, float xl, float yl, float xh, float yh,
                                      int num_nodes, int num_movable, int num_filler,
                                      const int* __restrict__ inv_order, float2* __restrict__ xy_o,
                                      const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  const float alpha = (float)st[NS_ALPHA];
  const float coef = (float)st[NS_COEF];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nodes; i += gridDim.x * blockDim.x) {
    const int j = i + num_nodes;
    const float ux = fsub(v[i], fmul(alpha, g[i]));
    const float uy = fsub(v[j], fmul(alpha, g[j]));
    float vx = fadd(ux, fmul(coef, fsub(ux, u[i])));
    float vy = fadd(uy, fmul(coef, fsub(uy, u[j])));
    if (i < num_movable || i >= num_nodes - num_filler) {
      vx = fminf(fmaxf(vx, xl), fsub(xh, sx[i]));
      vy = fminf(fmaxf(vy, yl), fsub(yh, sy[i]));
    }
    u_new[i] = ux;
    u_new[j] = uy;
    v_new[i] = vx;
    v_new[j] = vy;
    if (xy_new) xy_new[i] = make_float2(vx, vy);
    // the scattered cells' positions also land in visiting order
    if (xy_o && (i < num_movable || i >= num_nodes - num_filler)) xy_o[inv_order[i]] = make_float2(vx, vy);
  }
}

__global__ void pack_xy_kernel(const float* __restrict__ v, float2* __restrict__ xy, int num_nodes) {
  grid_dep_sync();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nodes; i += gridDim.x * blockDim.x)
    xy[i] = make_float2(v[i], v[i + num_nodes]);
}

// g' /= max(1, pws + lambda*area) in place, and per-block fp64 sums of
// (v' - v)^2 and (g' - g)^2 (finished by nesterov_finish_kernel).
__global__ void __launch_bounds__(256) precondition_norms_kernel(
    float* __restrict__ g_new, const float* __restrict__ g, const float* __restrict__ v_new,
    const float* __restrict__ v, const float* __restrict__ pws, const float* __restrict__ area,
    const float* __restrict__ lam_p, int num_nodes, double* __restrict__ partials) {
  grid_dep_sync();
  const float lam = *lam_p;
  const int n2 = 2 * num_nodes;
  double dv = 0.0, dg = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    {
      int node = i < num_nodes ? i : i - num_nodes;
      float p = fmaxf(fadd(pws[node], fmul(lam, area[node])), 1.0f);
      float gn = __fdiv_rn(g_new[i], p);
      g_new[i] = gn;
      double a = (double)v_new[i] - (double)v[i];
      double b = (double)gn - (double)g[i];
      dv += a * a;
      dg += b * b;
    }
  }
  block_partial2(dv, dg, partials);
}

// g'[i] = (wirelength pin sum of node i, nodes < num_movable) + (force of node i,
// movable and filler nodes, read from order space through inv_order); then
// g' /= max(1, pws + lambda*area), and the fp64 step-size norms as above.
// One warp per tile of 32 consecutive nodes; the warps of a block work on
// independent tiles, so no block barrier sits inside the loop.  The tile's
// movable pins form one contiguous node-CSR range, gathered kAsmWarpPins at a
// time (8 independent gathers per lane, through grad_index) into the warp's
// shared buffer; each lane then folds its own node's staged pins in pin order,
// so the sums are those of the sequential per-node loop.
constexpr int kAsmThreads = 256;
constexpr int kAsmWarpPins = 128;

__global__ void __launch_bounds__(kAsmThreads, 4) assemble_precondition_kernel(
    const float2* __restrict__ gnode, const int* __restrict__ node_start, const float* __restrict__ wl_scale_p,
    const float2* __restrict__ force_o, const int* __restrict__ inv_order, int num_movable, int num_filler,
    const float* __restrict__ pws, const float* __restrict__ area, const float* __restrict__ lam_p, int num_nodes,
    const float* __restrict__ v_new, const float* __restrict__ v, const float* __restrict__ g,
    float* __restrict__ g_new, double* __restrict__ partials, const int* __restrict__ grad_index,
    const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  __shared__ float2 s_q[kAsmThreads / 32][kAsmWarpPins];
  const float lam = *lam_p;
  const float ws = *wl_scale_p;
  const int lane = threadIdx.x & 31;
  float2* q_s = s_q[threadIdx.x >> 5];
  const int warp = (blockIdx.x * kAsmThreads + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kAsmThreads) >> 5;
  double dv = 0.0, dg = 0.0;
  // the tile's pin offsets are loaded one tile ahead
  int nx0 = 0, nx1 = 0;
  {
    const int i = warp * 32 + lane;
    if (warp * 32 < num_movable && i < num_movable) {  // node_start holds an entry past the last movable node
      nx0 = __ldg(node_start + i);
      nx1 = __ldg(node_start + i + 1);
    }
  }
  for (int n0 = warp * 32; n0 < num_nodes; n0 += nwarps * 32) {  // warp-uniform
    const int i = n0 + lane;
    const bool valid = i < num_nodes;
    const int my0 = nx0, my1 = nx1;
    {
      const int inext = n0 + nwarps * 32 + lane;
      nx0 = nx1 = 0;
      if (inext < num_movable) {
        nx0 = __ldg(node_start + inext);
        nx1 = __ldg(node_start + inext + 1);
      }
    }
    // the node's own loads first: independent of the pin gather below
    float2 f = make_float2(0.f, 0.f);
    float pw = 0.f, ar = 0.f, vnx = 0.f, vny = 0.f, vx = 0.f, vy = 0.f, gx0 = 0.f, gy0 = 0.f;
    if (valid) {
      if (i < num_movable || i >= num_nodes - num_filler) f = force_o[__ldg(inv_order + i)];
      pw = __ldg(pws + i);
      ar = __ldg(area + i);
      vnx = __ldcs(v_new + i);
      vny = __ldcs(v_new + i + num_nodes);
      vx = __ldcs(v + i);
      vy = __ldcs(v + i + num_nodes);
      gx0 = __ldcs(g + i);
      gy0 = __ldcs(g + i + num_nodes);
    }
    float sx = 0.f, sy = 0.f;
    const int m_cnt = min(num_movable - n0, 32);  // movable nodes of the tile (warp-uniform)
    if (m_cnt > 0) {
      const int p0 = __shfl_sync(0xffffffffu, my0, 0);
      const int p1 = __shfl_sync(0xffffffffu, my1, m_cnt - 1);
      for (int c0 = p0; c0 < p1; c0 += kAsmWarpPins) {
        float2 q[kAsmWarpPins / 32];
#pragma unroll
        for (int j = 0; j < kAsmWarpPins / 32; ++j) {
          const int k = c0 + 32 * j + lane;
          q[j] = make_float2(0.f, 0.f);
          if (k < p1) q[j] = grad_index ? gnode[__ldcs(grad_index + k)] : __ldcs(gnode + k);
        }
#pragma unroll
        for (int j = 0; j < kAsmWarpPins / 32; ++j) q_s[32 * j + lane] = q[j];
        __syncwarp();
        const int ka = max(my0, c0), kb = min(my1, c0 + kAsmWarpPins);
        for (int k = ka; k < kb; ++k) {
          const float2 w = q_s[k - c0];
          sx = fadd(sx, fmul(w.x, ws));
          sy = fadd(sy, fmul(w.y, ws));
        }
        __syncwarp();  // q_s is refilled by the next chunk or tile
      }
    }
    if (valid) {
      const float p = fmaxf(fadd(pw, fmul(lam, ar)), 1.0f);
      const float gx = __fdiv_rn(fadd(sx, f.x), p);
      const float gy = __fdiv_rn(fadd(sy, f.y), p);
      __stcs(g_new + i, gx);
      __stcs(g_new + i + num_nodes, gy);
      const double a1 = (double)vnx - (double)vx, a2 = (double)vny - (double)vy;
      const double b1 = (double)gx - (double)gx0, b2 = (double)gy - (double)gy0;
      dv += a1 * a1 + a2 * a2;
      dg += b1 * b1 + b2 * b2;
    }
  }
  block_partial2(dv, dg, partials);
}

__global__ void nesterov_finish_kernel(double* st, const double* partials, int count) {
  grid_dep_sync();
  double dv = finish_sum(partials, count);
  double dg = finish_sum(partials + count, count);
  if (threadIdx.x != 0) return;
  st[NS_ACC_DV] = dv;
  st[NS_ACC_DG] = dg;
  double an = sqrt(dv / dg);
  double accept = an > 0.95 * st[NS_ALPHA] ? 1.0 : 0.0;
  st[NS_ALPHA_NEW] = an;
  st[NS_ACCEPT] = accept;
  st[NS_ALPHA] = an;  // the reference copies alpha_{k+1} into alpha_k after every trial
}

__global__ void nesterov_init_kernel(double* st, double alpha) {
  grid_dep_sync();
  st[NS_ALPHA] = alpha;
  st[NS_A] = 1.0;
  double an = (1.0 + sqrt(5.0)) / 2.0;
  st[NS_A_NEXT] = an;
  st[NS_COEF] = 0.0;
  for (int i = NS_ACC_DV; i < NS_COUNT; ++i) st[i] = 0.0;
}

// objective = wl + lambda_eff * D' with D' = D (1 + c D) under the quadratic
// penalty (c > 0) and lambda_eff = density_factor * density_weight; the density
// gradient's scale (d objective / d D) goes to grad_scale for the force kernel
// (dreamplace/PlaceObj.py:293-320).
__global__ void objective_finish_kernel(const double* wl, const double* energy, const float* density_weight,
                                        const float* factor_quad, double* obj, float* grad_scale) {
  grid_dep_sync();
  const float density_factor = factor_quad[0], quad_c = factor_quad[1];
  double lam = (double)density_factor * (double)density_weight[0];
  double d = energy[0];
  double dp = quad_c > 0.f ? d * (1.0 + (double)quad_c * d) : d;
  if (obj) obj[0] = wl[0] + lam * dp;
  double dd = quad_c > 0.f ? 1.0 + 2.0 * (double)quad_c * d : 1.0;
  if (grad_scale) grad_scale[0] = (float)(lam * dd);
}

// the metrics a trial's host read-back needs, gathered into one 8-double row:
// HPWL and (overflow, max density) of v_k, the accept flag and step size of
// the trial, its objective, wirelength and energy
__global__ void trial_metrics_kernel(const double* hpwl, const double* overflow2, const double* state,
                                     const double* obj, const double* wl, const double* energy, double* out) {
  grid_dep_sync();
  out[0] = hpwl[0];
  out[1] = overflow2[0];
  out[2] = overflow2[1];
  out[3] = state[NS_ACCEPT];
  out[4] = state[NS_ALPHA];
  out[5] = obj[0];
  out[6] = wl[0];
  out[7] = energy[0];
}

}  // namespace dpb

using namespace dpb;

extern "C" int dp_trial_metrics(const double* hpwl, const double* overflow2, const double* state, const double* obj,
                                const double* wl, const double* energy, double* out8, dp_stream_t stream) {
  DP_REQUIRE(hpwl && overflow2 && state && obj && wl && energy && out8, "dp_trial_metrics: null pointer");
  launch_kernel(trial_metrics_kernel, 1, 1, 0, as_stream(stream), hpwl, overflow2, state, obj, wl, energy, out8);
  return check_launch("dp_trial_metrics");
}

extern "C" int dp_objective_finish(const double* wl, const double* energy, const float* density_weight,
                                   const float* factor_quad, double* obj, float* grad_scale, dp_stream_t stream) {
  DP_REQUIRE(energy && density_weight && factor_quad && (obj || grad_scale) && (!obj || wl),
             "dp_objective_finish: null pointer");
  launch_kernel(objective_finish_kernel, 1, 1, 0, as_stream(stream), wl, energy, density_weight, factor_quad, obj, grad_scale);
  return check_launch("dp_objective_finish");
}

extern "C" int dp_nesterov_init(double* state, double alpha, dp_stream_t stream) {
  DP_REQUIRE(state, "dp_nesterov_init: null state");
  launch_kernel(nesterov_init_kernel, 1, 1, 0, as_stream(stream), state, alpha);
  return check_launch("dp_nesterov_init");
}

extern "C" int dp_nesterov_trial(const float* v, const float* g, const float* u, float* u_new, float* v_new,
                                 float* xy_new, const double* state, const float* sx, const float* sy, float xl,
                                 float yl, float xh, float yh, int num_nodes, int num_movable, int num_filler,
                                 const int* inv_order, float* xy_order, dp_stream_t stream) {
  DP_REQUIRE(v && g && u && u_new && v_new && state && sx && sy, "dp_nesterov_trial: null pointer");
  DP_REQUIRE(((uintptr_t)xy_new & 7) == 0 && ((uintptr_t)xy_order & 7) == 0,
             "dp_nesterov_trial: xy_new / xy_order must be 8-byte aligned");
  DP_REQUIRE(!xy_order || inv_order, "dp_nesterov_trial: xy_order needs inv_order");
  if (num_nodes == 0) return DP_OK;
  launch_kernel(nesterov_trial_kernel, grid_for(num_nodes, 256, 8), 256, 0, as_stream(stream), 
      v, g, u, u_new, v_new, reinterpret_cast<float2*>(xy_new), state, sx, sy, xl, yl, xh, yh, num_nodes, num_movable,
      num_filler, inv_order, reinterpret_cast<float2*>(xy_order), trial_gate());
  return check_launch("dp_nesterov_trial");
}

extern "C" int dp_pack_xy(const float* pos, int num_nodes, float* xy, dp_stream_t stream) {
  DP_REQUIRE(pos && xy && ((uintptr_t)xy & 7) == 0, "dp_pack_xy: bad arguments");
  if (num_nodes == 0) return DP_OK;
  launch_kernel(pack_xy_kernel, grid_for(num_nodes, 256, 8), 256, 0, as_stream(stream), pos, reinterpret_cast<float2*>(xy),
                                                                            num_nodes);
  return check_launch("dp_pack_xy");
}

extern "C" int dp_precondition_step_size(float* g_new, const float* g, const float* v_new, const float* v,
                                         const float* pws, const float* area, const float* lambda_, int num_nodes,
                                         double* state, dp_stream_t stream) {
  DP_REQUIRE(g_new && g && v_new && v && pws && area && lambda_ && state, "dp_precondition_step_size: null pointer");
  cudaStream_t s = as_stream(stream);
  int blocks = grid_for(2ll * num_nodes, 256, 4);
  if (2 * blocks > 2 * DP_REDUCE_DOUBLES) blocks = DP_REDUCE_DOUBLES;
  double* partials = state + DP_NESTEROV_STATE_DOUBLES;
  launch_kernel(precondition_norms_kernel, blocks, 256, 0, s, g_new, g, v_new, v, pws, area, lambda_, num_nodes, partials);
  int rc = check_launch("dp_precondition_step_size");
  if (rc) return rc;
  launch_kernel(nesterov_finish_kernel, 1, 256, 0, s, state, partials, blocks);
  return check_launch("dp_precondition_step_size finish");
}

// What the GP loop does on the host between iteration k and k+1, on the
// device, so that iteration k+1 can be enqueued before the host has read
// iteration k's metrics:
//  * Nesterov: the scalars of iteration k (after its last trial) are copied
//    to iteration k+1's state and advanced (a_k <- a_{k+1}, coef);
//  * density weight (RePlAce HPWL mode, dreamplace/PlaceObj.py:833-851): with
//    f = k + 1 iterations done, for f > 1
//      mu = upper * max(0.9999^f, 0.98)                         if hpwl_k < hpwl_{k-1}
//      mu = upper * min(max(upper^(-(hpwl_k - hpwl_{k-1}) / ref_hpwl), lower), upper)  otherwise
//    lambda <- lambda * (float)mu;
//  * gamma (dreamplace/PlaceObj.py:901-915): gamma = base_gamma *
//    10^((ovf_k / total_area - 0.1) * 20 / 9 - 1), rounded to float, and its
//    reciprocal (the WA kernel's scalar).
// sched = {k, hpwl_{k-1}}; weights = {lambda, gamma, 1 / gamma}.
__global__ void iteration_head_kernel(const double* __restrict__ st_prev, double* __restrict__ st_new,
                                      const double* __restrict__ sched_prev, double* __restrict__ sched_new,
                                      const double* __restrict__ hpwl_k, const double* __restrict__ ovf_k,
                                      const float* __restrict__ w_prev, float* __restrict__ w_new, double base_gamma,
                                      double total_area, double ref_hpwl, double lower, double upper, int* gate) {
  grid_dep_sync();
  // the previous trial was rejected: this iteration was enqueued ahead and is
  // void; its gated kernels return at once
  if (gate) *gate = st_prev[NS_ACCEPT] == 0.0 ? 1 : 0;
  for (int i = 0; i < DP_NESTEROV_STATE_DOUBLES; ++i) st_new[i] = st_prev[i];
  const double a = st_new[NS_A_NEXT];
  st_new[NS_A] = a;
  const double an = (1.0 + sqrt(4.0 * a * a + 1.0)) / 2.0;
  st_new[NS_A_NEXT] = an;
  st_new[NS_COEF] = (a - 1.0) / an;
  const double f = sched_prev[0] + 1.0;
  const double hp = hpwl_k[0];
  float lam = w_prev[0];
  if (f > 1.0) {
    const double delta = hp - sched_prev[1];
    double mu;
    if (delta < 0.0)
      mu = upper * fmax(pow(0.9999, f), 0.98);
    else
      mu = upper * fmin(fmax(pow(upper, -delta / ref_hpwl), lower), upper);
    lam = fmul(lam, (float)mu);
  }
  sched_new[0] = f;
  sched_new[1] = hp;
  const double t = (ovf_k[0] / total_area - 0.1) * 20.0 / 9.0 - 1.0;
  const float gamma = (float)(base_gamma * pow(10.0, t));
  w_new[0] = lam;
  w_new[1] = gamma;
  w_new[2] = __fdiv_rn(1.0f, gamma);
}

extern "C" int dp_iteration_head(const double* state_prev, double* state_new, const double* sched_prev,
                                 double* sched_new, const double* hpwl_k, const double* overflow_k,
                                 const float* weights_prev, float* weights_new, double base_gamma, double total_area,
                                 double ref_hpwl, double lower, double upper, int* gate, dp_stream_t stream) {
  DP_REQUIRE(state_prev && state_new && sched_prev && sched_new && hpwl_k && overflow_k && weights_prev &&
                 weights_new,
             "dp_iteration_head: null pointer argument");
  DP_REQUIRE(state_prev != state_new && sched_prev != sched_new && weights_prev != weights_new,
             "dp_iteration_head: the previous and the new iteration need separate buffers");
  DP_REQUIRE(total_area > 0.0 && ref_hpwl > 0.0, "dp_iteration_head: total_area and ref_hpwl must be positive");
  launch_kernel(iteration_head_kernel, 1, 1, 0, as_stream(stream), state_prev, state_new, sched_prev, sched_new, hpwl_k,
                                                        overflow_k, weights_prev, weights_new, base_gamma,
                                                        total_area, ref_hpwl, lower, upper, gate);
  return check_launch("dp_iteration_head");
}

// ============================================================== warp reductions, pin sums
namespace dpb {

// max (kind 0), min (kind 1) or sum (kind 2) over the warp's 32 lanes, in every lane
__device__ __forceinline__ float warp_all(float v, int kind) {
  for (int o = 16; o > 0; o >>= 1) {
    float u = __shfl_xor_sync(0xffffffffu, v, o);
    v = kind == 0 ? fmaxf(v, u) : kind == 1 ? fminf(v, u) : fadd(v, u);
  }
  return v;
}

// node grad (+)= grad_pos[0] * sum of its pins' (weighted) gradients, which
// sit contiguously in node-CSR order; nodes >= num_movable get 0
__global__ void node_sum_kernel(const float2* __restrict__ gnode, const int* __restrict__ node_start,
                                const float* __restrict__ grad_p, int num_movable, int num_nodes, int accumulate,
                                float* __restrict__ out_x, float* __restrict__ out_y) {
  grid_dep_sync();
  const float g = *grad_p;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nodes; i += gridDim.x * blockDim.x) {
    float sx = 0.f, sy = 0.f;
    if (i < num_movable) {
      const int k1 = node_start[i + 1];
      for (int k = node_start[i]; k < k1; ++k) {
        const float2 v = __ldcs(gnode + k);
        sx = fadd(sx, fmul(v.x, g));
        sy = fadd(sy, fmul(v.y, g));
      }
    }
    if (accumulate) {
      out_x[i] = fadd(sx, out_x[i]);
      out_y[i] = fadd(sy, out_y[i]);
    } else {
      out_x[i] = sx;
      out_y[i] = sy;
    }
  }
}

}  // namespace dpb

extern "C" int dp_node_pin_sum(const float* grad_node_order, int num_slots, const int* node_start,
                               const float* grad_pos, int num_movable, int num_nodes, int accumulate, float* grad_out,
                               dp_stream_t stream) {
  DP_REQUIRE(grad_node_order && node_start && grad_pos && grad_out, "dp_node_pin_sum: null pointer argument");
  if (num_nodes == 0) return DP_OK;
  DP_REQUIRE(((uintptr_t)grad_node_order & 7) == 0, "dp_node_pin_sum: grad_node_order must be 8-byte aligned");
  launch_kernel(dpb::node_sum_kernel, dpb::grid_for(num_nodes, 256, 8), 256, 0, dpb::as_stream(stream), 
      reinterpret_cast<const float2*>(grad_node_order), node_start, grad_pos, num_movable, num_nodes, accumulate,
      grad_out, grad_out + num_nodes);
  return dpb::check_launch("dp_node_pin_sum");
}

extern "C" int dp_assemble_precondition_step(const float* grad_node_order, const int* node_start,
                                             const float* wl_scale, const float* force_o, const int* inv_order,
                                             int num_movable, int num_filler, const float* pws, const float* area,
                                             const float* lambda_, int num_nodes, const float* v_new, const float* v,
                                             const float* g, float* g_new, double* state, const int* grad_index,
                                             dp_stream_t stream) {
  using namespace dpb;
  DP_REQUIRE(grad_node_order && node_start && wl_scale && force_o && inv_order && pws && area && lambda_ && v_new &&
                 v && g && g_new && state,
             "dp_assemble_precondition_step: null pointer argument");
  DP_REQUIRE(num_nodes > 0 && num_movable >= 0 && num_filler >= 0 && num_movable + num_filler <= num_nodes,
             "dp_assemble_precondition_step: bad node counts");
  cudaStream_t s = as_stream(stream);
  int blocks = grid_for(num_nodes, kAsmThreads, 4);
  if (blocks > DP_REDUCE_DOUBLES) blocks = DP_REDUCE_DOUBLES;
  double* partials = state + DP_NESTEROV_STATE_DOUBLES;
  launch_kernel(assemble_precondition_kernel, blocks, kAsmThreads, 0, s, 
      reinterpret_cast<const float2*>(grad_node_order), node_start, wl_scale, reinterpret_cast<const float2*>(force_o),
      inv_order, num_movable, num_filler, pws, area, lambda_, num_nodes, v_new, v, g, g_new, partials, grad_index,
      trial_gate());
  int rc = check_launch("dp_assemble_precondition_step");
  if (rc) return rc;
  launch_kernel(nesterov_finish_kernel, 1, 256, 0, s, state, partials, blocks);
  return check_launch("dp_assemble_precondition_step finish");
}

// ============================================================== lane-per-net WA / HPWL
// Nets of degree d <= kLaneDeg are grouped 32 at a time by degree (host
// planner dp_plan_net_lanes); one warp takes a group, one lane a whole net.
// The group's pins are stored transposed (pin j of lane l at base + 32 j + l),
// so every pin load of the warp is one coalesced access.  A lane holds its
// net's pins in registers and runs the reference's per-net loops in pin order
// (so the sums are formed in the CPU op's order), and the per-net terms (the
// fp64 a terms, the divisions) are issued once per 32 nets instead of once
// per chunk of ~10 nets.  Nets of degree 9..32 go four of one degree to a
// group, eight lanes each (pins in registers, segment reductions); a larger
// net is a group of its own, handled by the whole warp with strided loops and
// warp reductions.
namespace dpb {

constexpr int kLaneDeg = 8;
// nets of degree kLaneDeg < d <= kSubDeg: four nets of one degree per group,
// kSubLanes lanes per net (each lane up to kSubDeg / kSubLanes pins)
constexpr int kSubDeg = 32;
constexpr int kSubLanes = 8;
constexpr int kSubPins = kSubDeg / kSubLanes;

struct LaneArgs {
  const float2* xy;        // interleaved node positions, or nullptr: planar pin positions below
  const float* px;         // pin x (planar form: ln_node holds pin ids, no offsets)
  const float* py;
  const int* group_deg;
  const int* group_base;
  const int* group_net;
  int num_groups;
  const int* ln_node;
  const float* ln_offx;
  const float* ln_offy;
  const int* ln_csr;
  const float* net_weights;
  const unsigned char* net_mask;
  const unsigned char* hpwl_mask;
  const float* inv_gamma;  // device scalar (read once per thread)
  float2* gnode;
};

// position of lane slot p: node position + pin offset, or (planar form) the
// pin's own position
template <bool kPins>
__device__ __forceinline__ float2 lane_xy(const LaneArgs& A, int p) {
  const int node = __ldcs(A.ln_node + p);
  if (kPins) return make_float2(A.px[node], A.py[node]);
  const float2 q = A.xy[node];
  return make_float2(fadd(__ldcs(A.ln_offx + p), q.x), fadd(__ldcs(A.ln_offy + p), q.y));
}

// where the gradient of lane slot p goes: its pin's node-CSR position, or p
// itself (lane-slot order, gathered by the assembly through grad_index)
__device__ __forceinline__ int grad_slot(const LaneArgs& A, int p) { return A.ln_csr ? __ldcs(A.ln_csr + p) : p; }

// Quotients of the WA sums.  Every exponential sum e is >= 1 (the extreme pin
// of a net contributes exp(0) = 1), so 1/e comes from one rcp.approx (within
// one ulp; no denormal or special operand can occur) and x / e from
// q = x * (1/e) with one FMA-residual correction (Markstein, IBM J. Res. Dev.
// 34(1), 1990): the residual x - q e is exact in one fma, and
// q + (x - q e) / e is the correctly rounded quotient -- the value of the
// reference's fp32 division -- in all but near-tie cases.
__device__ __forceinline__ float sum_rcp(float e) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e));
  return r;
}

__device__ __forceinline__ float sum_quot(float x, float e, float r) {
  const float q = fmul(x, r);
  return __fmaf_rn(__fmaf_rn(-q, e, x), r, q);
}

// a = (1 - b xe) / e.  The reference forms 1 - b xe in double (the literal
// 1.0 promotes it; weighted_average_wirelength_merged.cpp) and rounds the
// double quotient to float.  Here 1 - p (p = b xe rounded to float) is carried
// exactly as the float pair s + t (Knuth's TwoSum, TAOCP vol. 2, 4.2.2) and
// (s + t) / e is corrected as in sum_quot: the same float in all but near-tie
// cases, with no fp64 arithmetic.
__device__ __forceinline__ float wa_a_term(float b, float xe, float e, float r) {
  const float p = fmul(b, xe);
  const float s = fsub(1.f, p);
  const float bb = fsub(s, 1.f);
  const float t = fadd(fsub(1.f, fsub(s, bb)), fsub(-p, bb));
  const float q = fmul(s, r);
  return __fmaf_rn(fadd(__fmaf_rn(-q, e, s), t), r, q);
}

// b = ig / e and a = (1 - b xe) / e of one direction of a net
__device__ __forceinline__ void wa_terms(float ig, float e, float xe, float& b, float& a) {
  const float r = sum_rcp(e);
  b = sum_quot(ig, e, r);
  a = wa_a_term(b, xe, e, r);
}

// the WA value of a net from its eight sums
__device__ __forceinline__ float wa_value(float xe_p, float e_p, float xe_n, float e_n, float ye_p, float f_p,
                                          float ye_n, float f_n) {
  return fsub(fadd(fsub(sum_quot(xe_p, e_p, sum_rcp(e_p)), sum_quot(xe_n, e_n, sum_rcp(e_n))),
                   sum_quot(ye_p, f_p, sum_rcp(f_p))),
              sum_quot(ye_n, f_n, sum_rcp(f_n)));
}

template <int D, bool kGrad, bool kPins>
__device__ __forceinline__ void lane_net(const LaneArgs& A, float ig, int base, int lane, int net, bool hpwl,
                                         double& contrib, double& hcontrib) {
  float x[D], y[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const float2 q = lane_xy<kPins>(A, base + 32 * j + lane);
    x[j] = q.x;
    y[j] = q.y;
  }
  float x_max = x[0], x_min = x[0], y_max = y[0], y_min = y[0];
#pragma unroll
  for (int j = 1; j < D; ++j) {
    x_max = fmaxf(x_max, x[j]);
    x_min = fminf(x_min, x[j]);
    y_max = fmaxf(y_max, y[j]);
    y_min = fminf(y_min, y[j]);
  }
  const float w = A.net_weights ? A.net_weights[net] : 1.0f;
  if (!kGrad) {  // HPWL pass: net_mask is the HPWL mask
    if (A.net_mask[net]) {
      float h = fsub(fadd(fsub(x_max, x_min), y_max), y_min);
      if (A.net_weights) h = fmul(h, w);
      contrib += (double)h;
    }
    return;
  }
  if (hpwl && A.hpwl_mask[net]) {
    float h = fsub(fadd(fsub(x_max, x_min), y_max), y_min);
    if (A.net_weights) h = fmul(h, w);
    hcontrib += (double)h;
  }
  if (!A.net_mask[net]) {
#pragma unroll
    for (int j = 0; j < D; ++j) __stcs(A.gnode + grad_slot(A, base + 32 * j + lane), make_float2(0.f, 0.f));
    return;
  }
  // up to 4 pins the exponentials stay in registers for the gradient pass;
  // larger nets recompute them there (keeps the kernel's register count, and
  // with it the occupancy, at the small-net level)
  constexpr bool kKeep = D <= 4;
  constexpr int K = kKeep ? D : 1;
  float ex[K], enx[K], ey[K], eny[K];
  float e_p = 0.f, e_n = 0.f, xe_p = 0.f, xe_n = 0.f, f_p = 0.f, f_n = 0.f, ye_p = 0.f, ye_n = 0.f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const float a1 = expf(fmul(fsub(x[j], x_max), ig));
    const float a2 = expf(fmul(fsub(x_min, x[j]), ig));
    const float a3 = expf(fmul(fsub(y[j], y_max), ig));
    const float a4 = expf(fmul(fsub(y_min, y[j]), ig));
    if (kKeep) {
      ex[kKeep ? j : 0] = a1;
      enx[kKeep ? j : 0] = a2;
      ey[kKeep ? j : 0] = a3;
      eny[kKeep ? j : 0] = a4;
    }
    e_p = fadd(e_p, a1);
    e_n = fadd(e_n, a2);
    xe_p = fadd(xe_p, fmul(x[j], a1));
    xe_n = fadd(xe_n, fmul(x[j], a2));
    f_p = fadd(f_p, a3);
    f_n = fadd(f_n, a4);
    ye_p = fadd(ye_p, fmul(y[j], a3));
    ye_n = fadd(ye_n, fmul(y[j], a4));
  }
  const float wl = wa_value(xe_p, e_p, xe_n, e_n, ye_p, f_p, ye_n, f_n);
  contrib += (double)(A.net_weights ? fmul(wl, w) : wl);
  float b_x, a_x, b_nx, a_nx, b_y, a_y, b_ny, a_ny;
  wa_terms(ig, e_p, xe_p, b_x, a_x);
  wa_terms(-ig, e_n, xe_n, b_nx, a_nx);
  wa_terms(ig, f_p, ye_p, b_y, a_y);
  wa_terms(-ig, f_n, ye_n, b_ny, a_ny);
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const float a1 = kKeep ? ex[kKeep ? j : 0] : expf(fmul(fsub(x[j], x_max), ig));
    const float a2 = kKeep ? enx[kKeep ? j : 0] : expf(fmul(fsub(x_min, x[j]), ig));
    const float a3 = kKeep ? ey[kKeep ? j : 0] : expf(fmul(fsub(y[j], y_max), ig));
    const float a4 = kKeep ? eny[kKeep ? j : 0] : expf(fmul(fsub(y_min, y[j]), ig));
    float gx = fsub(fmul(fadd(a_x, fmul(b_x, x[j])), a1), fmul(fadd(a_nx, fmul(b_nx, x[j])), a2));
    float gy = fsub(fmul(fadd(a_y, fmul(b_y, y[j])), a3), fmul(fadd(a_ny, fmul(b_ny, y[j])), a4));
    if (A.net_weights) {
      gx = fmul(gx, w);
      gy = fmul(gy, w);
    }
    __stcs(A.gnode + grad_slot(A, base + 32 * j + lane), make_float2(gx, gy));
  }
}

// reduction over the kSubLanes lanes of one net (aligned lane segment)
__device__ __forceinline__ float sub_all(float v, int kind) {
#pragma unroll
  for (int o = kSubLanes / 2; o > 0; o >>= 1) {
    const float u = __shfl_xor_sync(0xffffffffu, v, o);
    v = kind == 0 ? fmaxf(v, u) : kind == 1 ? fminf(v, u) : fadd(v, u);
  }
  return v;
}

// a net of degree kLaneDeg < deg <= kSubDeg on kSubLanes lanes (four nets per
// warp, net -1 on padding segments): its pins are contiguous from base, lane
// s of the segment holds pins s, s + kSubLanes, ... in registers; maxima,
// minima and the exponential sums are reduced across the segment.  Every lane
// of the warp takes part in the shuffles.
template <bool kGrad, bool kPins>
__device__ void sub_net(const LaneArgs& A, float ig, int base, int deg, int lane, int net, bool hpwl,
                        double& contrib, double& hcontrib) {
  const int sl = lane & (kSubLanes - 1);
  const bool live = net >= 0;
  float x[kSubPins], y[kSubPins];
  float x_max = -FLT_MAX, x_min = FLT_MAX, y_max = -FLT_MAX, y_min = FLT_MAX;
#pragma unroll
  for (int t = 0; t < kSubPins; ++t) {
    const int j = sl + kSubLanes * t;
    x[t] = y[t] = 0.f;
    if (live && j < deg) {
      const float2 q = lane_xy<kPins>(A, base + j);
      x[t] = q.x;
      y[t] = q.y;
      x_max = fmaxf(x_max, q.x);
      x_min = fminf(x_min, q.x);
      y_max = fmaxf(y_max, q.y);
      y_min = fminf(y_min, q.y);
    }
  }
  x_max = sub_all(x_max, 0);
  x_min = sub_all(x_min, 1);
  y_max = sub_all(y_max, 0);
  y_min = sub_all(y_min, 1);
  // no early exit before the last shuffle: every lane runs the same sequence
  const float w = live && A.net_weights ? A.net_weights[net] : 1.0f;
  if (!kGrad) {
    if (live && sl == 0 && A.net_mask[net]) {
      float h = fsub(fadd(fsub(x_max, x_min), y_max), y_min);
      if (A.net_weights) h = fmul(h, w);
      contrib += (double)h;
    }
    return;
  }
  if (live && hpwl && sl == 0 && A.hpwl_mask[net]) {
    float h = fsub(fadd(fsub(x_max, x_min), y_max), y_min);
    if (A.net_weights) h = fmul(h, w);
    hcontrib += (double)h;
  }
  const bool on = live && A.net_mask[net];
  float e_p = 0.f, e_n = 0.f, xe_p = 0.f, xe_n = 0.f, f_p = 0.f, f_n = 0.f, ye_p = 0.f, ye_n = 0.f;
  if (on) {
#pragma unroll
    for (int t = 0; t < kSubPins; ++t) {
      if (sl + kSubLanes * t < deg) {
        const float a1 = expf(fmul(fsub(x[t], x_max), ig));
        const float a2 = expf(fmul(fsub(x_min, x[t]), ig));
        const float a3 = expf(fmul(fsub(y[t], y_max), ig));
        const float a4 = expf(fmul(fsub(y_min, y[t]), ig));
        e_p = fadd(e_p, a1);
        e_n = fadd(e_n, a2);
        xe_p = fadd(xe_p, fmul(x[t], a1));
        xe_n = fadd(xe_n, fmul(x[t], a2));
        f_p = fadd(f_p, a3);
        f_n = fadd(f_n, a4);
        ye_p = fadd(ye_p, fmul(y[t], a3));
        ye_n = fadd(ye_n, fmul(y[t], a4));
      }
    }
  }
  e_p = sub_all(e_p, 2); e_n = sub_all(e_n, 2); xe_p = sub_all(xe_p, 2); xe_n = sub_all(xe_n, 2);
  f_p = sub_all(f_p, 2); f_n = sub_all(f_n, 2); ye_p = sub_all(ye_p, 2); ye_n = sub_all(ye_n, 2);
  if (!live) return;
  if (!on) {
#pragma unroll
    for (int t = 0; t < kSubPins; ++t)
      if (sl + kSubLanes * t < deg) __stcs(A.gnode + grad_slot(A, base + sl + kSubLanes * t), make_float2(0.f, 0.f));
    return;
  }
  if (sl == 0) {
    const float wl = wa_value(xe_p, e_p, xe_n, e_n, ye_p, f_p, ye_n, f_n);
    contrib += (double)(A.net_weights ? fmul(wl, w) : wl);
  }
  float b_x, a_x, b_nx, a_nx, b_y, a_y, b_ny, a_ny;
  wa_terms(ig, e_p, xe_p, b_x, a_x);
  wa_terms(-ig, e_n, xe_n, b_nx, a_nx);
  wa_terms(ig, f_p, ye_p, b_y, a_y);
  wa_terms(-ig, f_n, ye_n, b_ny, a_ny);
#pragma unroll
  for (int t = 0; t < kSubPins; ++t) {
    const int j = sl + kSubLanes * t;
    if (j < deg) {
      const float a1 = expf(fmul(fsub(x[t], x_max), ig)), a2 = expf(fmul(fsub(x_min, x[t]), ig));
      const float a3 = expf(fmul(fsub(y[t], y_max), ig)), a4 = expf(fmul(fsub(y_min, y[t]), ig));
      float gx = fsub(fmul(fadd(a_x, fmul(b_x, x[t])), a1), fmul(fadd(a_nx, fmul(b_nx, x[t])), a2));
      float gy = fsub(fmul(fadd(a_y, fmul(b_y, y[t])), a3), fmul(fadd(a_ny, fmul(b_ny, y[t])), a4));
      if (A.net_weights) {
        gx = fmul(gx, w);
        gy = fmul(gy, w);
      }
      __stcs(A.gnode + grad_slot(A, base + j), make_float2(gx, gy));
    }
  }
}

// a net of degree > kSubDeg: pins base .. base + deg (contiguous), whole warp
template <bool kGrad, bool kPins>
__device__ void warp_net(const LaneArgs& A, float ig, int base, int deg, int lane, int net, bool hpwl,
                         double& contrib, double& hcontrib) {
  float x_max = -FLT_MAX, x_min = FLT_MAX, y_max = -FLT_MAX, y_min = FLT_MAX;
  for (int j = lane; j < deg; j += 32) {
    const float2 q = lane_xy<kPins>(A, base + j);
    const float xx = q.x, yy = q.y;
    x_max = fmaxf(x_max, xx);
    x_min = fminf(x_min, xx);
    y_max = fmaxf(y_max, yy);
    y_min = fminf(y_min, yy);
  }
  x_max = warp_all(x_max, 0);
  x_min = warp_all(x_min, 1);
  y_max = warp_all(y_max, 0);
  y_min = warp_all(y_min, 1);
  const float w = A.net_weights ? A.net_weights[net] : 1.0f;
  if (!kGrad) {
    if (lane == 0 && A.net_mask[net]) {
      float h = fsub(fadd(fsub(x_max, x_min), y_max), y_min);
      if (A.net_weights) h = fmul(h, w);
      contrib += (double)h;
    }
    return;
  }
  if (hpwl && lane == 0 && A.hpwl_mask[net]) {
    float h = fsub(fadd(fsub(x_max, x_min), y_max), y_min);
    if (A.net_weights) h = fmul(h, w);
    hcontrib += (double)h;
  }
  const bool on = A.net_mask[net];
  float xe_p = 0.f, xe_n = 0.f, e_p = 0.f, e_n = 0.f, ye_p = 0.f, ye_n = 0.f, f_p = 0.f, f_n = 0.f;
  if (on) {
    for (int j = lane; j < deg; j += 32) {
      const float2 q = lane_xy<kPins>(A, base + j);
      const float xx = q.x, yy = q.y;
      const float a1 = expf(fmul(fsub(xx, x_max), ig)), a2 = expf(fmul(fsub(x_min, xx), ig));
      const float a3 = expf(fmul(fsub(yy, y_max), ig)), a4 = expf(fmul(fsub(y_min, yy), ig));
      xe_p = fadd(xe_p, fmul(xx, a1));
      xe_n = fadd(xe_n, fmul(xx, a2));
      e_p = fadd(e_p, a1);
      e_n = fadd(e_n, a2);
      ye_p = fadd(ye_p, fmul(yy, a3));
      ye_n = fadd(ye_n, fmul(yy, a4));
      f_p = fadd(f_p, a3);
      f_n = fadd(f_n, a4);
    }
    xe_p = warp_all(xe_p, 2); xe_n = warp_all(xe_n, 2); e_p = warp_all(e_p, 2); e_n = warp_all(e_n, 2);
    ye_p = warp_all(ye_p, 2); ye_n = warp_all(ye_n, 2); f_p = warp_all(f_p, 2); f_n = warp_all(f_n, 2);
    if (lane == 0) {
      const float wl = wa_value(xe_p, e_p, xe_n, e_n, ye_p, f_p, ye_n, f_n);
      contrib += (double)(A.net_weights ? fmul(wl, w) : wl);
    }
  }
  float b_x = 0.f, a_x = 0.f, b_nx = 0.f, a_nx = 0.f, b_y = 0.f, a_y = 0.f, b_ny = 0.f, a_ny = 0.f;
  if (on) {
    wa_terms(ig, e_p, xe_p, b_x, a_x);
    wa_terms(-ig, e_n, xe_n, b_nx, a_nx);
    wa_terms(ig, f_p, ye_p, b_y, a_y);
    wa_terms(-ig, f_n, ye_n, b_ny, a_ny);
  }
  for (int j = lane; j < deg; j += 32) {
    float gx = 0.f, gy = 0.f;
    if (on) {
      const float2 q = lane_xy<kPins>(A, base + j);
      const float xx = q.x, yy = q.y;
      const float a1 = expf(fmul(fsub(xx, x_max), ig)), a2 = expf(fmul(fsub(x_min, xx), ig));
      const float a3 = expf(fmul(fsub(yy, y_max), ig)), a4 = expf(fmul(fsub(y_min, yy), ig));
      gx = fsub(fmul(fadd(a_x, fmul(b_x, xx)), a1), fmul(fadd(a_nx, fmul(b_nx, xx)), a2));
      gy = fsub(fmul(fadd(a_y, fmul(b_y, yy)), a3), fmul(fadd(a_ny, fmul(b_ny, yy)), a4));
      if (A.net_weights) {
        gx = fmul(gx, w);
        gy = fmul(gy, w);
      }
    }
    A.gnode[grad_slot(A, base + j)] = make_float2(gx, gy);
  }
}

// 4 blocks of 256 per SM: the 64-register cap spills a few words of the
// 5..8-pin paths to L1, and still measures faster than 3 blocks without spills
template <bool kGrad, bool kPins>
__global__ void __launch_bounds__(256, 4) wa_lane_kernel(LaneArgs A, double* __restrict__ partials,
                                                      double* __restrict__ hpwl_partials,
                                                      const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool hpwl = kGrad && hpwl_partials != nullptr;
  const float ig = kGrad ? *A.inv_gamma : 0.f;
  double contrib = 0.0, hcontrib = 0.0;
  for (int g = warp; g < A.num_groups; g += nwarps) {
    const int deg = A.group_deg[g], base = A.group_base[g];
    if (deg > kSubDeg) {
      warp_net<kGrad, kPins>(A, ig, base, deg, lane, A.group_net[32 * g], hpwl, contrib, hcontrib);
      continue;
    }
    if (deg > kLaneDeg) {
      const int s = lane / kSubLanes;
      sub_net<kGrad, kPins>(A, ig, base + s * deg, deg, lane, A.group_net[32 * g + s], hpwl, contrib, hcontrib);
      continue;
    }
    const int net = A.group_net[32 * g + lane];
    if (net < 0) continue;  // padding lane of the last group of a degree
    switch (deg) {
      case 1: lane_net<1, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 2: lane_net<2, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 3: lane_net<3, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 4: lane_net<4, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 5: lane_net<5, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 6: lane_net<6, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 7: lane_net<7, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      case 8: lane_net<8, kGrad, kPins>(A, ig, base, lane, net, hpwl, contrib, hcontrib); break;
      default: break;
    }
  }
  block_partial(contrib, partials);
  if (hpwl) block_partial(hcontrib, hpwl_partials);
}

}  // namespace dpb

extern "C" int dp_plan_net_lanes(const int* netpin_start_host, int num_nets, const int* net_order_host,
                                 int* num_groups, int* num_lane_slots, int* group_deg, int* group_base,
                                 int* group_net, int* lane_slot) {
  using namespace dpb;
  DP_REQUIRE(netpin_start_host && num_groups && num_lane_slots && num_nets >= 0, "dp_plan_net_lanes: bad arguments");
  if (net_order_host) {  // must be a permutation: every net planned exactly once
    std::vector<unsigned char> seen(num_nets, 0);
    for (int t = 0; t < num_nets; ++t) {
      const int e = net_order_host[t];
      DP_REQUIRE(e >= 0 && e < num_nets && !seen[e], "dp_plan_net_lanes: net_order is not a permutation");
      seen[e] = 1;
    }
  }
  const bool fill = group_deg && group_base && group_net && lane_slot;
  int g = 0;
  long long base = 0;
  for (int d = 1; d <= kLaneDeg; ++d) {
    int in_group = 0;
    for (int t = 0; t < num_nets; ++t) {
      const int e = net_order_host ? net_order_host[t] : t;
      const int s0 = netpin_start_host[e];
      if (netpin_start_host[e + 1] - s0 != d) continue;
      if (in_group == 0) {
        if (fill) {
          group_deg[g] = d;
          group_base[g] = (int)base;
          for (int l = 0; l < 32; ++l) group_net[32 * g + l] = -1;
          for (int i = 0; i < 32 * d; ++i) lane_slot[base + i] = -1;
        }
      }
      if (fill) {
        group_net[32 * g + in_group] = e;
        for (int j = 0; j < d; ++j) lane_slot[base + 32 * j + in_group] = s0 + j;
      }
      if (++in_group == 32) {
        in_group = 0;
        ++g;
        base += 32 * d;
      }
    }
    if (in_group) {
      ++g;
      base += 32 * d;
    }
  }
  // degrees kLaneDeg + 1 .. kSubDeg: 32 / kSubLanes nets of one degree per
  // group, net s's pins contiguous from group_base + s * d
  constexpr int kSubNets = 32 / kSubLanes;
  for (int d = kLaneDeg + 1; d <= kSubDeg; ++d) {
    int in_group = 0;
    for (int t = 0; t < num_nets; ++t) {
      const int e = net_order_host ? net_order_host[t] : t;
      const int s0 = netpin_start_host[e];
      if (netpin_start_host[e + 1] - s0 != d) continue;
      if (in_group == 0 && fill) {
        group_deg[g] = d;
        group_base[g] = (int)base;
        for (int l = 0; l < 32; ++l) group_net[32 * g + l] = -1;
        for (int i = 0; i < kSubNets * d; ++i) lane_slot[base + i] = -1;
      }
      if (fill) {
        group_net[32 * g + in_group] = e;
        for (int j = 0; j < d; ++j) lane_slot[base + in_group * d + j] = s0 + j;
      }
      if (++in_group == kSubNets) {
        in_group = 0;
        ++g;
        base += kSubNets * d;
      }
    }
    if (in_group) {
      ++g;
      base += kSubNets * d;
    }
  }
  for (int t = 0; t < num_nets; ++t) {
    const int e = net_order_host ? net_order_host[t] : t;
    const int s0 = netpin_start_host[e], d = netpin_start_host[e + 1] - s0;
    if (d <= kSubDeg) continue;
    if (fill) {
      group_deg[g] = d;
      group_base[g] = (int)base;
      group_net[32 * g] = e;
      for (int l = 1; l < 32; ++l) group_net[32 * g + l] = -1;
      for (int j = 0; j < d; ++j) lane_slot[base + j] = s0 + j;
    }
    ++g;
    base += d;
  }
  DP_REQUIRE(base < (1ll << 31), "dp_plan_net_lanes: too many pins");
  *num_groups = g;
  *num_lane_slots = (int)base;
  return DP_OK;
}

static int launch_lanes(bool grad, const dpb::LaneArgs& A, double* out_f64, double* hpwl_f64, cudaStream_t s) {
  using namespace dpb;
  // one wave: the launch bounds keep 4 blocks of 256 resident per SM, and the
  // warps stride over the groups, so a larger grid only adds a partial last
  // wave (at 1279 blocks, a third wave of 95)
  int blocks = A.num_groups > 0 ? ceil_div((long long)A.num_groups * 32, 256) : 1;
  if (blocks > kNumSMs * 4) blocks = kNumSMs * 4;
  if (blocks > kMaxReduceBlocks) blocks = kMaxReduceBlocks;
  if (grad && A.px)
    launch_kernel(wa_lane_kernel<true, true>, blocks, 256, 0, s, A, out_f64 + 1, nullptr, trial_gate());
  else if (grad)
    launch_kernel(wa_lane_kernel<true, false>, blocks, 256, 0, s, A, out_f64 + 1, hpwl_f64 ? hpwl_f64 + 1 : nullptr,
                                                       trial_gate());
  else
    launch_kernel(wa_lane_kernel<false, false>, blocks, 256, 0, s, A, out_f64 + 1, nullptr, trial_gate());
  int rc = check_launch(grad ? "dp_wa_lanes_forward" : "dp_hpwl_lanes");
  if (rc) return rc;
  // the WA total and the HPWL (same fixed-order reduction each) in one launch
  if (grad && hpwl_f64) return launch_finish_sum2(out_f64, hpwl_f64, blocks, s);
  return launch_finish_sum(out_f64, blocks, nullptr, s);
}

static dpb::LaneArgs lane_args(const float* xy, const int* group_deg, const int* group_base, const int* group_net,
                               int num_groups, const int* ln_node, const float* ln_offx, const float* ln_offy,
                               const int* ln_csr, const float* net_weights, const unsigned char* net_mask,
                               const unsigned char* hpwl_mask, const float* inv_gamma, float* grad_node_order) {
  dpb::LaneArgs A;
  A.xy = reinterpret_cast<const float2*>(xy);
  A.px = A.py = nullptr;
  A.group_deg = group_deg;
  A.group_base = group_base;
  A.group_net = group_net;
  A.num_groups = num_groups;
  A.ln_node = ln_node;
  A.ln_offx = ln_offx;
  A.ln_offy = ln_offy;
  A.ln_csr = ln_csr;
  A.net_weights = net_weights;
  A.net_mask = net_mask;
  A.hpwl_mask = hpwl_mask;
  A.inv_gamma = inv_gamma;
  A.gnode = reinterpret_cast<float2*>(grad_node_order);
  return A;
}

extern "C" int dp_wa_lanes_forward(const float* xy, const int* group_deg, const int* group_base, const int* group_net,
                                   int num_groups, const int* ln_node, const float* ln_offx, const float* ln_offy,
                                   const int* ln_csr, const float* net_weights, const unsigned char* net_mask,
                                   const float* inv_gamma, double* wl_f64, float* grad_node_order,
                                   const unsigned char* hpwl_mask, double* hpwl_f64, dp_stream_t stream) {
  DP_REQUIRE(xy && group_deg && group_base && group_net && ln_node && ln_offx && ln_offy && net_mask && inv_gamma &&
                 wl_f64 && grad_node_order,
             "dp_wa_lanes_forward: null pointer argument");
  DP_REQUIRE(((uintptr_t)xy & 7) == 0 && ((uintptr_t)grad_node_order & 7) == 0,
             "dp_wa_lanes_forward: xy and grad_node_order must be 8-byte aligned");
  DP_REQUIRE(!hpwl_f64 || hpwl_mask, "dp_wa_lanes_forward: hpwl_f64 needs hpwl_mask");
  DP_REQUIRE(num_groups >= 0, "dp_wa_lanes_forward: bad group count");
  const dpb::LaneArgs A = lane_args(xy, group_deg, group_base, group_net, num_groups, ln_node, ln_offx, ln_offy,
                                    ln_csr, net_weights, net_mask, hpwl_mask, inv_gamma, grad_node_order);
  return launch_lanes(true, A, wl_f64, hpwl_f64, dpb::as_stream(stream));
}

extern "C" int dp_hpwl_lanes(const float* xy, const int* group_deg, const int* group_base, const int* group_net,
                             int num_groups, const int* ln_node, const float* ln_offx, const float* ln_offy,
                             const float* net_weights, const unsigned char* net_mask, double* out_f64,
                             dp_stream_t stream) {
  DP_REQUIRE(xy && group_deg && group_base && group_net && ln_node && ln_offx && ln_offy && net_mask && out_f64,
             "dp_hpwl_lanes: null pointer argument");
  DP_REQUIRE(((uintptr_t)xy & 7) == 0, "dp_hpwl_lanes: xy must be 8-byte aligned");
  DP_REQUIRE(num_groups >= 0, "dp_hpwl_lanes: bad group count");
  const dpb::LaneArgs A = lane_args(xy, group_deg, group_base, group_net, num_groups, ln_node, ln_offx, ln_offy,
                                    nullptr, net_weights, net_mask, nullptr, nullptr, nullptr);
  return launch_lanes(false, A, out_f64, nullptr, dpb::as_stream(stream));
}

// ---------------------------------------------------------------- WA on pin positions
// The lane-per-net WA of dp_wa_lanes_forward reading the pins' own positions
// (planar [x(P) | y(P)], the layout of the reference op's input), for the
// drop-in WeightedAverageWirelength: the lane slots hold pin ids.
extern "C" int dp_wa_pins_forward(const float* pin_pos, int num_pins, const int* group_deg, const int* group_base,
                                  const int* group_net, int num_groups, const int* ln_pin, const float* net_weights,
                                  const unsigned char* net_mask, const float* inv_gamma, double* wl_f64,
                                  float* grad_lane, dp_stream_t stream) {
  DP_REQUIRE(pin_pos && group_deg && group_base && group_net && ln_pin && net_mask && inv_gamma && wl_f64 && grad_lane,
             "dp_wa_pins_forward: null pointer argument");
  DP_REQUIRE(num_pins >= 0 && num_groups >= 0, "dp_wa_pins_forward: bad sizes");
  DP_REQUIRE(((uintptr_t)grad_lane & 7) == 0, "dp_wa_pins_forward: grad_lane must be 8-byte aligned");
  dpb::LaneArgs A = lane_args(nullptr, group_deg, group_base, group_net, num_groups, ln_pin, nullptr, nullptr, nullptr,
                              net_weights, net_mask, nullptr, inv_gamma, grad_lane);
  A.px = pin_pos;
  A.py = pin_pos + num_pins;
  return launch_lanes(true, A, wl_f64, nullptr, dpb::as_stream(stream));
}

namespace dpb {
// grad_pin_pos[p] = grad_out * grad_lane[lane_of_pin[p]] (x then y), 0 where pin_mask
__global__ void wa_pins_backward_kernel(const float2* __restrict__ grad_lane, const int* __restrict__ lane_of_pin,
                                        const unsigned char* __restrict__ pin_mask, const float* __restrict__ grad_out,
                                        int num_pins, float* __restrict__ gx, float* __restrict__ gy) {
  grid_dep_sync();
  const float g = grad_out[0];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < num_pins; p += gridDim.x * blockDim.x) {
    float x = 0.f, y = 0.f;
    if (!(pin_mask && pin_mask[p])) {
      const float2 v = __ldg(grad_lane + __ldg(lane_of_pin + p));
      x = fmul(v.x, g);
      y = fmul(v.y, g);
    }
    __stcs(gx + p, x);
    __stcs(gy + p, y);
  }
}
}  // namespace dpb

extern "C" int dp_wa_pins_backward(const float* grad_lane, const int* lane_of_pin, const unsigned char* pin_mask,
                                   const float* grad_out, int num_pins, float* grad_pin_pos, dp_stream_t stream) {
  using namespace dpb;
  DP_REQUIRE(grad_lane && lane_of_pin && grad_out && grad_pin_pos, "dp_wa_pins_backward: null pointer argument");
  DP_REQUIRE(((uintptr_t)grad_lane & 7) == 0, "dp_wa_pins_backward: grad_lane must be 8-byte aligned");
  if (num_pins == 0) return DP_OK;
  launch_kernel(wa_pins_backward_kernel, grid_for(num_pins, 256, 8), 256, 0, as_stream(stream), 
      reinterpret_cast<const float2*>(grad_lane), lane_of_pin, pin_mask, grad_out, num_pins, grad_pin_pos,
      grad_pin_pos + num_pins);
  return check_launch("dp_wa_pins_backward");
}
