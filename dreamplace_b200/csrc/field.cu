// Field gather: the electric force on every movable and filler cell, the
// hand-written adjoint of the density scatter (electric_potential.py:219-275).
//
// Per cell the sum runs in the CPU reference's order
// (electric_potential/src/electric_force.cpp:114-166): k-major over the
// stretched cell's x bins, h-minor over y bins, area = px*py, gx += area*Ex,
// then gx *= ratio, then * grad_pos, all with round-to-nearest and no FMA
// contraction, so the result equals the CPU op bit for bit given the same
// field maps.  One thread per cell; the two 4 MB field maps stay resident in
// L2 across the gather.
#include "common.cuh"

namespace dpb {

__global__ void __launch_bounds__(256) electric_force_kernel(
    const float* __restrict__ grad_pos, int nbx, int nby, const float* __restrict__ ex,
    const float* __restrict__ ey, const float* __restrict__ x, const float* __restrict__ y,
    const float* __restrict__ sx_c, const float* __restrict__ sy_c, const float* __restrict__ ox,
    const float* __restrict__ oy, const float* __restrict__ ratio, float xl, float yl, float bsx,
    float bsy, float ibx, float iby, int num_movable, int filler_begin, int total,
    const int* __restrict__ sorted, float scale, float* __restrict__ gx_out,
    float* __restrict__ gy_out) {
  grid_dep_sync();
  const float g = grad_pos[0];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    int i = idx < num_movable ? (sorted ? sorted[idx] : idx) : filler_begin + (idx - num_movable);
    float sx = sx_c[i], sy = sy_c[i];
    float nx = fadd(x[i], ox[i]);
    float ny = fadd(y[i], oy[i]);
    int k0, k1, h0, h1;
    triangle_bin_range(nx, sx, xl, ibx, nbx, k0, k1);
    triangle_bin_range(ny, sy, yl, iby, nby, h0, h1);
    float gx = 0.f, gy = 0.f;
    for (int k = k0; k < k1; ++k) {
      float px = triangle_overlap(nx, sx, xl, k, bsx);
      const float* exr = ex + (size_t)k * nby;
      const float* eyr = ey + (size_t)k * nby;
      for (int h = h0; h < h1; ++h) {
        float py = triangle_overlap(ny, sy, yl, h, bsy);
        float area = fmul(px, py);
        gx = fadd(gx, fmul(area, __ldg(exr + h)));
        gy = fadd(gy, fmul(area, __ldg(eyr + h)));
      }
    }
    float r = ratio[i];
    gx = fmul(fmul(fmul(gx, r), g), scale);
    gy = fmul(fmul(fmul(gy, r), g), scale);
    gx_out[i] = gx;
    gy_out[i] = gy;
  }
}

__global__ void zero_range_kernel(float* a, int begin, int end, float* b) {
  grid_dep_sync();
  for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    a[i] = 0.f;
    b[i] = 0.f;
  }
}

constexpr int kForceWin = 3;  // almost every stretched cell covers at most 3 x 3 bins

// Field gather over cells in visiting order (engine path): attributes from the
// per-cell records, positions from xy_o (both in visiting order, or xy_o in
// node order read through `order`); the force pair is written in order
// space, force_o[idx] = scale * grad * ratio * sum(px py E), for the gradient
// assembly kernel to pick up per node.
__global__ void __launch_bounds__(256) electric_force_records_kernel(
    const float* __restrict__ grad_pos, int nbx, int nby, const float* __restrict__ ex, const float* __restrict__ ey,
    const float2* __restrict__ xy_o, const int* __restrict__ order, const float4* __restrict__ rec4,
    const float* __restrict__ ratio_o, int count, float xl, float yl, float bsx, float bsy, float ibx, float iby,
    float scale, float2* __restrict__ force_o, const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  const float g = grad_pos[0];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    const float4 r4 = __ldcs(rec4 + idx);
    const float2 p = order ? __ldg(xy_o + __ldg(order + idx)) : __ldg(xy_o + idx);
    const float sx = r4.x, sy = r4.y;
    const float nx = fadd(p.x, r4.z);
    const float ny = fadd(p.y, r4.w);
    int k0, k1, h0, h1;
    triangle_bin_range(nx, sx, xl, ibx, nbx, k0, k1);
    triangle_bin_range(ny, sy, yl, iby, nby, h0, h1);
    const int nk = k1 - k0, nh = h1 - h0;
    float gx = 0.f, gy = 0.f;
    if (nk <= kForceWin && nh <= kForceWin) {
      // py computed once per y bin; the sum keeps the k-major, h-minor order
      float py[kForceWin];
#pragma unroll
      for (int hh = 0; hh < kForceWin; ++hh) py[hh] = hh < nh ? triangle_overlap(ny, sy, yl, h0 + hh, bsy) : 0.f;
#pragma unroll
      for (int kk = 0; kk < kForceWin; ++kk) {
        if (kk < nk) {
          const float px = triangle_overlap(nx, sx, xl, k0 + kk, bsx);
          const float* exr = ex + (size_t)(k0 + kk) * nby + h0;
          const float* eyr = ey + (size_t)(k0 + kk) * nby + h0;
#pragma unroll
          for (int hh = 0; hh < kForceWin; ++hh) {
            if (hh < nh) {
              const float area = fmul(px, py[hh]);
              gx = fadd(gx, fmul(area, __ldg(exr + hh)));
              gy = fadd(gy, fmul(area, __ldg(eyr + hh)));
            }
          }
        }
      }
    } else {
      for (int k = k0; k < k1; ++k) {
        const float px = triangle_overlap(nx, sx, xl, k, bsx);
        const float* exr = ex + (size_t)k * nby;
        const float* eyr = ey + (size_t)k * nby;
        for (int h = h0; h < h1; ++h) {
          const float py = triangle_overlap(ny, sy, yl, h, bsy);
          const float area = fmul(px, py);
          gx = fadd(gx, fmul(area, __ldg(exr + h)));
          gy = fadd(gy, fmul(area, __ldg(eyr + h)));
        }
      }
    }
    const float r = __ldcs(ratio_o + idx);
    force_o[idx] = make_float2(fmul(fmul(fmul(gx, r), g), scale), fmul(fmul(fmul(gy, r), g), scale));
  }
}

}  // namespace dpb

using namespace dpb;

extern "C" int dp_electric_force_ordered(const float* grad_pos, int nbx, int nby, const float* ex, const float* ey,
                                         const float* xy_o, const int* order, const float* rec4,
                                         const float* ratio_o,
                                         int count, float xl, float yl, float bsx, float bsy, float ibx, float iby,
                                         float scale, float* force_o, dp_stream_t stream) {
  DP_REQUIRE(grad_pos && ex && ey && xy_o && rec4 && ratio_o && force_o,
             "dp_electric_force_ordered: null pointer argument");
  DP_REQUIRE(((uintptr_t)xy_o & 7) == 0 && ((uintptr_t)rec4 & 15) == 0 && ((uintptr_t)force_o & 7) == 0,
             "dp_electric_force_ordered: misaligned xy_o / rec4 / force_o");
  if (count == 0) return DP_OK;
  launch_kernel(electric_force_records_kernel, grid_for(count, 256, 16), 256, 0, as_stream(stream), 
      grad_pos, nbx, nby, ex, ey, reinterpret_cast<const float2*>(xy_o), order, reinterpret_cast<const float4*>(rec4),
      ratio_o, count, xl, yl, bsx, bsy, ibx, iby, scale, reinterpret_cast<float2*>(force_o), trial_gate());
  return check_launch("dp_electric_force_ordered");
}

extern "C" int dp_electric_force(const float* grad_pos, int nbx, int nby, const float* ex,
                                 const float* ey, const float* pos, int num_nodes, const float* sx,
                                 const float* sy, const float* ox, const float* oy,
                                 const float* ratio, float xl, float yl, float xh, float yh,
                                 float bsx, float bsy, float ibx, float iby, int nm, int nf,
                                 const int* sorted, float scale, float* out, dp_stream_t stream) {
  DP_REQUIRE(grad_pos && ex && ey && pos && sx && sy && ox && oy && ratio && out,
             "dp_electric_force: null pointer argument");
  DP_REQUIRE(nm >= 0 && nf >= 0 && nm + nf <= num_nodes, "dp_electric_force: bad node counts");
  DP_REQUIRE(nbx > 0 && nby > 0, "dp_electric_force: bad bin grid");
  cudaStream_t s = as_stream(stream);
  float* gx = out;
  float* gy = out + num_nodes;
  int fixed_begin = nm, fixed_end = num_nodes - nf;
  if (fixed_end > fixed_begin) {
    launch_kernel(zero_range_kernel, grid_for(fixed_end - fixed_begin, 256), 256, 0, s, gx, fixed_begin, fixed_end, gy);
    int rc = check_launch("dp_electric_force zero");
    if (rc) return rc;
  }
  int total = nm + nf;
  if (total == 0) return DP_OK;
  launch_kernel(electric_force_kernel, grid_for(total, 256, 16), 256, 0, s, 
      grad_pos, nbx, nby, ex, ey, pos, pos + num_nodes, sx, sy, ox, oy, ratio, xl, yl, bsx, bsy, ibx,
      iby, nm, num_nodes - nf, total, sorted, scale, gx, gy);
  return check_launch("dp_electric_force");
}

namespace dpb {
// out[node] = v.x, out[n + node] = v.y for node = order[idx]: values kept in
// visiting order put back in node order
__global__ void scatter_pairs_kernel(const float2* __restrict__ vals_o, const int* __restrict__ order, int count,
                                     int num_nodes, float* __restrict__ out) {
  grid_dep_sync();
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    const int i = __ldg(order + idx);
    const float2 v = __ldcs(vals_o + idx);
    out[i] = v.x;
    out[num_nodes + i] = v.y;
  }
}
}  // namespace dpb

extern "C" int dp_scatter_pairs_to_nodes(const float* vals_o, const int* order, int count, int num_nodes, float* out,
                                         dp_stream_t stream) {
  DP_REQUIRE(vals_o && order && out, "dp_scatter_pairs_to_nodes: null pointer argument");
  DP_REQUIRE(count >= 0 && count <= num_nodes, "dp_scatter_pairs_to_nodes: bad counts");
  DP_REQUIRE(((uintptr_t)vals_o & 7) == 0, "dp_scatter_pairs_to_nodes: vals_o must be 8-byte aligned");
  cudaStream_t s = as_stream(stream);
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * 2 * (size_t)num_nodes, s);
  if (e != cudaSuccess) {
    set_error("dp_scatter_pairs_to_nodes: cudaMemsetAsync: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  if (count == 0) return DP_OK;
  launch_kernel(scatter_pairs_kernel, grid_for(count, 256, 8), 256, 0, s, reinterpret_cast<const float2*>(vals_o), order, count,
                                                               num_nodes, out);
  return check_launch("dp_scatter_pairs_to_nodes");
}
