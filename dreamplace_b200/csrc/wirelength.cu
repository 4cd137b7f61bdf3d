// Wirelength-side kernels: WA merged forward/backward, pin positions,
// HPWL, move-boundary and pin-weight sums.
//
// Reference semantics (paths relative to dreamplace/ops):
//   weighted_average_wirelength/src/weighted_average_wirelength_merged.cpp:31-231
//   weighted_average_wirelength/src/integrate_net_weights_cuda_kernel.cu:17-48
//   weighted_average_wirelength/weighted_average_wirelength.py:160-213
//   pin_pos/src/pin_pos.cpp (forward gather, node-by-node backward)
//   hpwl/src/hpwl.cpp, move_boundary/src/move_boundary.cpp, pin_weight_sum/src/pws.cpp
//
// The WA forward keeps the CPU op's per-net arithmetic (x and y in one pass,
// a = (1.0 - b*S1)/S0 in double as the C++ expression promotes it, no FMA
// contraction); only exp() differs (CUDA expf, <= 2 ulp).  Totals are
// accumulated in fp64.
#include "reduce.cuh"

namespace dpb {

__device__ __forceinline__ float wa_exp(float a) { return expf(a); }

__global__ void __launch_bounds__(256) wa_merged_forward_kernel(
    const float* __restrict__ px, const float* __restrict__ py, const int* __restrict__ flat_netpin,
    const int* __restrict__ netpin_start, int num_nets, const float* __restrict__ net_weights,
    const unsigned char* __restrict__ net_mask, const float* __restrict__ inv_gamma_p,
    float* __restrict__ partial_wl, double* __restrict__ partials, float* __restrict__ gx,
    float* __restrict__ gy) {
  grid_dep_sync();
  const float inv_gamma = *inv_gamma_p;
  double contrib = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nets; i += gridDim.x * blockDim.x) {
    {
      int b = netpin_start[i], e = netpin_start[i + 1];
      if (net_mask[i]) {
        float x_max = -FLT_MAX, x_min = FLT_MAX, y_max = -FLT_MAX, y_min = FLT_MAX;
        for (int j = b; j < e; ++j) {
          int p = flat_netpin[j];
          float xx = px[p], yy = py[p];
          x_max = fmaxf(xx, x_max);
          x_min = fminf(xx, x_min);
          y_max = fmaxf(yy, y_max);
          y_min = fminf(yy, y_min);
        }
        float xe_p = 0.f, xe_n = 0.f, e_p = 0.f, e_n = 0.f;
        float ye_p = 0.f, ye_n = 0.f, f_p = 0.f, f_n = 0.f;
        for (int j = b; j < e; ++j) {
          int p = flat_netpin[j];
          float xx = px[p], yy = py[p];
          float ex = wa_exp(fmul(fsub(xx, x_max), inv_gamma));
          float enx = wa_exp(fmul(fsub(x_min, xx), inv_gamma));
          xe_p = fadd(xe_p, fmul(xx, ex));
          xe_n = fadd(xe_n, fmul(xx, enx));
          e_p = fadd(e_p, ex);
          e_n = fadd(e_n, enx);
          float ey = wa_exp(fmul(fsub(yy, y_max), inv_gamma));
          float eny = wa_exp(fmul(fsub(y_min, yy), inv_gamma));
          ye_p = fadd(ye_p, fmul(yy, ey));
          ye_n = fadd(ye_n, fmul(yy, eny));
          f_p = fadd(f_p, ey);
          f_n = fadd(f_n, eny);
        }
        float wl = fsub(fadd(fsub(__fdiv_rn(xe_p, e_p), __fdiv_rn(xe_n, e_n)), __fdiv_rn(ye_p, f_p)),
                        __fdiv_rn(ye_n, f_n));
        float w = net_weights ? net_weights[i] : 1.0f;
        float pw = net_weights ? fmul(wl, w) : wl;
        if (partial_wl) partial_wl[i] = pw;
        contrib += (double)pw;
        float b_x = __fdiv_rn(inv_gamma, e_p);
        float a_x = (float)((1.0 - (double)fmul(b_x, xe_p)) / (double)e_p);
        float b_nx = __fdiv_rn(-inv_gamma, e_n);
        float a_nx = (float)((1.0 - (double)fmul(b_nx, xe_n)) / (double)e_n);
        float b_y = __fdiv_rn(inv_gamma, f_p);
        float a_y = (float)((1.0 - (double)fmul(b_y, ye_p)) / (double)f_p);
        float b_ny = __fdiv_rn(-inv_gamma, f_n);
        float a_ny = (float)((1.0 - (double)fmul(b_ny, ye_n)) / (double)f_n);
        for (int j = b; j < e; ++j) {
          int p = flat_netpin[j];
          float xx = px[p], yy = py[p];
          float ex = wa_exp(fmul(fsub(xx, x_max), inv_gamma));
          float enx = wa_exp(fmul(fsub(x_min, xx), inv_gamma));
          gx[p] = fsub(fmul(fadd(a_x, fmul(b_x, xx)), ex), fmul(fadd(a_nx, fmul(b_nx, xx)), enx));
          float ey = wa_exp(fmul(fsub(yy, y_max), inv_gamma));
          float eny = wa_exp(fmul(fsub(y_min, yy), inv_gamma));
          gy[p] = fsub(fmul(fadd(a_y, fmul(b_y, yy)), ey), fmul(fadd(a_ny, fmul(b_ny, yy)), eny));
        }
      } else {
        if (partial_wl) partial_wl[i] = 0.f;
        for (int j = b; j < e; ++j) {
          int p = flat_netpin[j];
          gx[p] = 0.f;
          gy[p] = 0.f;
        }
      }
    }
  }
  block_partial(contrib, partials);
}


__global__ void wa_merged_backward_kernel(const float* __restrict__ grad_pos,
                                          const int* __restrict__ pin2net,
                                          const float* __restrict__ net_weights,
                                          const unsigned char* __restrict__ net_mask,
                                          const unsigned char* __restrict__ pin_mask, int num_pins,
                                          float* __restrict__ gx, float* __restrict__ gy) {
  grid_dep_sync();
  const float g = grad_pos[0];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < num_pins; p += gridDim.x * blockDim.x) {
    float vx = fmul(gx[p], g), vy = fmul(gy[p], g);
    if (net_weights) {
      int net = pin2net[p];
      if (net >= 0 && net_mask[net]) {
        float w = net_weights[net];
        vx = fmul(vx, w);
        vy = fmul(vy, w);
      }
    }
    if (pin_mask && pin_mask[p]) {
      vx = 0.f;
      vy = 0.f;
    }
    gx[p] = vx;
    gy[p] = vy;
  }
}

__global__ void pin_pos_forward_kernel(const float* __restrict__ x, const float* __restrict__ y,
                                       const float* __restrict__ offx, const float* __restrict__ offy,
                                       const int* __restrict__ pin2node, int num_pins,
                                       float* __restrict__ pin_x, float* __restrict__ pin_y) {
  grid_dep_sync();
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < num_pins; p += gridDim.x * blockDim.x) {
    int n = pin2node[p];
    pin_x[p] = fadd(offx[p], x[n]);
    pin_y[p] = fadd(offy[p], y[n]);
  }
}

__global__ void pin_pos_backward_kernel(const float* __restrict__ gpx, const float* __restrict__ gpy,
                                        const int* __restrict__ flat_node2pin,
                                        const int* __restrict__ node_start, int num_physical,
                                        int num_nodes, float* __restrict__ gx, float* __restrict__ gy) {
  grid_dep_sync();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nodes; i += gridDim.x * blockDim.x) {
    float sx = 0.f, sy = 0.f;
    if (i < num_physical) {
      int b = node_start[i], e = node_start[i + 1];
      for (int j = b; j < e; ++j) {
        int p = flat_node2pin[j];
        sx = fadd(sx, gpx[p]);
        sy = fadd(sy, gpy[p]);
      }
    }
    gx[i] = sx;
    gy[i] = sy;
  }
}

__global__ void __launch_bounds__(256) hpwl_kernel(const float* __restrict__ px, const float* __restrict__ py,
                                                   const int* __restrict__ flat_netpin,
                                                   const int* __restrict__ netpin_start, int num_nets,
                                                   const float* __restrict__ net_weights,
                                                   const unsigned char* __restrict__ net_mask,
                                                   double* __restrict__ partials) {
  grid_dep_sync();
  double c = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nets; i += gridDim.x * blockDim.x) {
    if (net_mask[i]) {
      float max_x = -FLT_MAX, min_x = FLT_MAX, max_y = -FLT_MAX, min_y = FLT_MAX;
      for (int j = netpin_start[i]; j < netpin_start[i + 1]; ++j) {
        int p = flat_netpin[j];
        float xx = px[p], yy = py[p];
        min_x = fminf(min_x, xx);
        max_x = fmaxf(max_x, xx);
        min_y = fminf(min_y, yy);
        max_y = fmaxf(max_y, yy);
      }
      float h = fsub(fadd(fsub(max_x, min_x), max_y), min_y);
      if (net_weights) h = fmul(h, net_weights[i]);
      c += (double)h;
    }
  }
  block_partial(c, partials);
}

__global__ void move_boundary_kernel(float* __restrict__ x, float* __restrict__ y,
                                     const float* __restrict__ sx, const float* __restrict__ sy,
                                     float xl, float yl, float xh, float yh, int num_nodes,
                                     int num_movable, int num_filler) {
  grid_dep_sync();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nodes; i += gridDim.x * blockDim.x) {
    if (i < num_movable || i >= num_nodes - num_filler) {
      float vx = fmaxf(x[i], xl);
      vx = fminf(vx, fsub(xh, sx[i]));
      float vy = fmaxf(y[i], yl);
      vy = fminf(vy, fsub(yh, sy[i]));
      x[i] = vx;
      y[i] = vy;
    }
  }
}

__global__ void pws_kernel(const float* __restrict__ w, const int* __restrict__ flat_nodepin,
                           const int* __restrict__ node_start, const int* __restrict__ pin2net,
                           int num_physical, int num_nodes, float* __restrict__ out) {
  grid_dep_sync();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_nodes; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    if (i < num_physical)
      for (int j = node_start[i]; j < node_start[i + 1]; ++j) s = fadd(s, w[pin2net[flat_nodepin[j]]]);
    out[i] = s;
  }
}

}  // namespace dpb

using namespace dpb;

extern "C" int dp_wa_merged_forward(const float* pin_pos, int num_pins, const int* flat_netpin,
                                    const int* netpin_start, int num_nets, const float* net_weights,
                                    const unsigned char* net_mask, const float* inv_gamma,
                                    float* partial_wl, double* wl_f64, float* wl_out,
                                    float* grad_intermediate, dp_stream_t stream) {
  DP_REQUIRE(pin_pos && flat_netpin && netpin_start && net_mask && inv_gamma && wl_f64 && grad_intermediate,
             "dp_wa_merged_forward: null pointer argument");
  DP_REQUIRE(num_pins >= 0 && num_nets >= 0, "dp_wa_merged_forward: negative sizes");
  cudaStream_t s = as_stream(stream);
  int blocks = num_nets > 0 ? grid_for(num_nets, 256, 8) : 1;
  if (blocks > kMaxReduceBlocks) blocks = kMaxReduceBlocks;
  launch_kernel(wa_merged_forward_kernel, blocks, 256, 0, s, pin_pos, pin_pos + num_pins, flat_netpin, netpin_start, num_nets,
                                                 net_weights, net_mask, inv_gamma, partial_wl, wl_f64 + 1,
                                                 grad_intermediate, grad_intermediate + num_pins);
  int rc = check_launch("dp_wa_merged_forward");
  if (rc) return rc;
  return launch_finish_sum(wl_f64, blocks, wl_out, s);
}

extern "C" int dp_wa_merged_backward(const float* grad_pos, const int* pin2net_map,
                                     const float* net_weights, const unsigned char* net_mask,
                                     const unsigned char* pin_mask, int num_pins,
                                     float* grad_intermediate, dp_stream_t stream) {
  DP_REQUIRE(grad_pos && grad_intermediate, "dp_wa_merged_backward: null pointer argument");
  DP_REQUIRE(!net_weights || (pin2net_map && net_mask), "dp_wa_merged_backward: net weights need pin2net_map and net_mask");
  if (num_pins == 0) return DP_OK;
  cudaStream_t s = as_stream(stream);
  launch_kernel(wa_merged_backward_kernel, grid_for(num_pins, 256, 8), 256, 0, s, 
      grad_pos, pin2net_map, net_weights, net_mask, pin_mask, num_pins, grad_intermediate,
      grad_intermediate + num_pins);
  return check_launch("dp_wa_merged_backward");
}

extern "C" int dp_pin_pos_forward(const float* pos, int num_nodes, const float* offx,
                                  const float* offy, const int* pin2node, int num_pins,
                                  float* pin_pos, dp_stream_t stream) {
  DP_REQUIRE(pos && offx && offy && pin2node && pin_pos, "dp_pin_pos_forward: null pointer argument");
  if (num_pins == 0) return DP_OK;
  launch_kernel(pin_pos_forward_kernel, grid_for(num_pins, 256, 8), 256, 0, as_stream(stream), 
      pos, pos + num_nodes, offx, offy, pin2node, num_pins, pin_pos, pin_pos + num_pins);
  return check_launch("dp_pin_pos_forward");
}

extern "C" int dp_pin_pos_backward(const float* grad_pin, int num_pins, const int* flat_node2pin,
                                   const int* node_start, int num_physical, int num_nodes,
                                   float* grad_pos, dp_stream_t stream) {
  DP_REQUIRE(grad_pin && flat_node2pin && node_start && grad_pos, "dp_pin_pos_backward: null pointer argument");
  DP_REQUIRE(num_physical <= num_nodes, "dp_pin_pos_backward: num_physical_nodes > num_nodes");
  if (num_nodes == 0) return DP_OK;
  launch_kernel(pin_pos_backward_kernel, grid_for(num_nodes, 256, 8), 256, 0, as_stream(stream), 
      grad_pin, grad_pin + num_pins, flat_node2pin, node_start, num_physical, num_nodes, grad_pos,
      grad_pos + num_nodes);
  return check_launch("dp_pin_pos_backward");
}

extern "C" int dp_hpwl(const float* pin_pos, int num_pins, const int* flat_netpin,
                       const int* netpin_start, int num_nets, const float* net_weights,
                       const unsigned char* net_mask, double* out_f64, float* out_f32,
                       dp_stream_t stream) {
  DP_REQUIRE(pin_pos && flat_netpin && netpin_start && net_mask && out_f64, "dp_hpwl: null pointer argument");
  cudaStream_t s = as_stream(stream);
  int blocks = num_nets > 0 ? grid_for(num_nets, 256, 8) : 1;
  if (blocks > kMaxReduceBlocks) blocks = kMaxReduceBlocks;
  launch_kernel(hpwl_kernel, blocks, 256, 0, s, pin_pos, pin_pos + num_pins, flat_netpin, netpin_start, num_nets, net_weights,
                                    net_mask, out_f64 + 1);
  int rc = check_launch("dp_hpwl");
  if (rc) return rc;
  return launch_finish_sum(out_f64, blocks, out_f32, s);
}

extern "C" int dp_move_boundary(float* pos, int num_nodes, const float* sx, const float* sy, float xl,
                                float yl, float xh, float yh, int nm, int nf, dp_stream_t stream) {
  DP_REQUIRE(pos && sx && sy, "dp_move_boundary: null pointer argument");
  if (num_nodes == 0) return DP_OK;
  launch_kernel(move_boundary_kernel, grid_for(num_nodes, 256, 8), 256, 0, as_stream(stream), 
      pos, pos + num_nodes, sx, sy, xl, yl, xh, yh, num_nodes, nm, nf);
  return check_launch("dp_move_boundary");
}

extern "C" int dp_pin_weight_sum(const float* w, const int* flat_nodepin, const int* node_start,
                                 const int* pin2net, int num_physical, int num_nodes, float* out,
                                 dp_stream_t stream) {
  DP_REQUIRE(w && flat_nodepin && node_start && pin2net && out, "dp_pin_weight_sum: null pointer argument");
  if (num_nodes == 0) return DP_OK;
  launch_kernel(pws_kernel, grid_for(num_nodes, 256, 8), 256, 0, as_stream(stream), w, flat_nodepin, node_start,
                                                                        pin2net, num_physical, num_nodes, out);
  return check_launch("dp_pin_weight_sum");
}
