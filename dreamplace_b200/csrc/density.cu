// Density scatter kernels: triangle (stretched-cell) model in fp32 and in
// 64-bit fixed point, the exact-overlap maps, and the overflow reduction.
//
// Semantics follow the reference CPU ops (paths relative to dreamplace/ops):
//   electric_potential/src/electric_density_map.cpp:100-152, 216-268
//   electric_potential/src/electric_density_map.cpp:155-213, 270-309
//   electric_potential/src/density_function.h:12-36
//   utility/src/atomic_ops.h:43-54 (fixed-point add and final conversion)
//   density_map/src/density_map.cpp (exact DensityMap)
//   electric_potential/electric_overflow.py:260-278 (overflow / max density)
//
// Layout: one thread per scattered cell; cells are addressed through
// sorted_node_map (movable, ascending width, so neighbouring threads have
// similar loop trip counts) followed by the filler range.  A warp whose lanes
// hit the same bin combines their contributions with a match/reduce before
// one atomic, which removes most same-address serialisation when cells are
// clustered (the GP starts with every movable cell at the die centre).
#include <climits>
#include <cstdlib>
#include <mutex>
#include <cuda.h>
#include <type_traits>
#include <cub/block/block_radix_sort.cuh>
#include "reduce.cuh"

namespace dpb {

struct TriangleArgs {
  const float* x; const float* y;
  const float* sx; const float* sy; const float* ox; const float* oy; const float* ratio;
  float xl, yl, bsx, bsy, inv_bsx, inv_bsy;
  int num_bins_x, num_bins_y;
  int num_movable, num_filler, filler_begin;
  const int* sorted_node_map;
};

__device__ __forceinline__ int scatter_node_index(const TriangleArgs& a, int idx) {
  if (idx < a.num_movable) return a.sorted_node_map ? a.sorted_node_map[idx] : idx;
  return a.filler_begin + (idx - a.num_movable);
}

// Adds v to map[bin] after combining the lanes of the warp that target the
// same bin: one atomic per distinct bin instead of one per lane.
template <typename T, typename U>
__device__ __forceinline__ void combined_add(U* map, int bin, T v, unsigned active) {
  unsigned peers = __match_any_sync(active, bin);
  int leader = __ffs(peers) - 1;
  unsigned rest = peers & (peers - 1);  // peers without the leader
  T sum = v;
  while (rest) {  // identical trip sequence on every lane of the group
    int src = __ffs(rest) - 1;
    rest &= rest - 1;
    sum += __shfl_sync(peers, v, src);
  }
  if ((int)(threadIdx.x & 31) == leader) atomicAdd(map + bin, (U)sum);
}

// Each lane walks its cell's bins in k-major, h-minor order.  All lanes of the
// warp iterate together up to the warp's largest trip count so that
// __match_any_sync sees every lane that is still issuing an update.
template <bool kFixed>
__global__ void __launch_bounds__(256) triangle_scatter_kernel(TriangleArgs a, int total,
                                                               float fx_scale, float* map_f32,
                                                               unsigned long long* map_fx) {
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < total; base += stride) {
    int idx = base + threadIdx.x;
    bool valid = idx < total;
    int kx0 = 0, kx1 = 0, hy0 = 0, hy1 = 0;
    float nx = 0.f, ny = 0.f, sx = 0.f, sy = 0.f, r = 0.f;
    if (valid) {
      int i = scatter_node_index(a, idx);
      sx = a.sx[i];
      sy = a.sy[i];
      nx = fadd(a.x[i], a.ox[i]);
      ny = fadd(a.y[i], a.oy[i]);
      r = a.ratio[i];
      triangle_bin_range(nx, sx, a.xl, a.inv_bsx, a.num_bins_x, kx0, kx1);
      triangle_bin_range(ny, sy, a.yl, a.inv_bsy, a.num_bins_y, hy0, hy1);
    }
    int nkx = max(kx1 - kx0, 0), nhy = max(hy1 - hy0, 0);
    int trips = nkx * nhy;
    // warp-uniform loop bound
    int max_trips = trips;
    for (int o = 16; o > 0; o >>= 1) max_trips = max(max_trips, __shfl_xor_sync(0xffffffffu, max_trips, o));
    float px_r = 0.f;
    int cur_k = -1;
    for (int t = 0; t < max_trips; ++t) {
      bool live = t < trips;
      unsigned active = __ballot_sync(0xffffffffu, live);
      if (live) {
        int k = kx0 + t / nhy;
        int h = hy0 + t % nhy;
        if (k != cur_k) {
          float px = triangle_overlap(nx, sx, a.xl, k, a.bsx);
          px_r = fmul(px, r);
          cur_k = k;
        }
        float py = triangle_overlap(ny, sy, a.yl, h, a.bsy);
        float area = fmul(px_r, py);
        int bin = k * a.num_bins_y + h;
        if (kFixed) {
          combined_add<long long, unsigned long long>(map_fx, bin, to_fixed(area, fx_scale), active);
        } else {
          combined_add<float, float>(map_f32, bin, area, active);
        }
      }
    }
  }
}

// ---------------------------------------------------------------- window scatter
// Cells are visited in the caller's order (a spatial order refreshed every few
// iterations, grouping cells whose stretched footprint starts in the same
// bin), read from per-cell records (stretched width, height, offsets,
// ratio) and positions stored in the same order (written there by the
// Nesterov trial kernel), so every read of the scatter is contiguous.
//
// A stretched cell is at least sqrt(2) bins wide, and a standard cell covers
// at most kWin x kWin bins.  Each lane computes its cell's kWin px and kWin py
// overlaps once and forms the kWin x kWin window of bin contributions in
// registers (fp32, or int64 fixed point converted per contribution as the CPU
// op does).  A lane keeps one running window while its successive cells start
// at the same bin.  At the end, a run of lanes whose windows start at the same
// bin is summed with a segmented shuffle reduction (only as many steps as the
// longest run needs), and the run's first lane adds the window to the block's
// shared-memory tile over its bin bounding box (or to global memory when the
// box does not fit).  The tile is flushed with one global atomic per touched
// bin.  Cells wider than the window take a plain per-bin loop.  In the
// clustered start of GP, tens of thousands of cells share a bin, so one warp
// issues kWin*kWin adds for its 128 cells; when cells are spread each cell
// flushes its own window and adds only its own bins.  The fixed-point map is
// independent of the summation order, so the deterministic result does not
// depend on the visiting order or the tiling.
constexpr int kWin = 3;
constexpr int kWsThreads = 256;
constexpr int kWsCellsPerLane = 4;
constexpr int kWsWarpCells = 32 * kWsCellsPerLane;
constexpr int kWsCells = kWsThreads * kWsCellsPerLane;
constexpr int kWsSmemBytes = 24 * 1024;

template <typename Acc>
__device__ __forceinline__ void add_to(Acc* tile, float* map_f32, unsigned long long* map_fx, bool use_tile, int slot,
                                       int bin, Acc v) {
  if (use_tile) {
    atomicAdd(tile + slot, v);
  } else if (sizeof(Acc) == 8) {
    atomicAdd(map_fx + bin, (unsigned long long)v);
  } else {
    atomicAdd(map_f32 + bin, (float)v);
  }
}

// adds the non-zero entries of a window starting at bin (k0, h0)
template <typename Acc>
__device__ __forceinline__ void flush_window(const Acc (&w)[kWin][kWin], int k0, int h0, int bk0, int bh0, int H,
                                             int nby, bool use_tile, Acc* tile, float* map_f32,
                                             unsigned long long* map_fx) {
#pragma unroll
  for (int kk = 0; kk < kWin; ++kk)
#pragma unroll
    for (int hh = 0; hh < kWin; ++hh)
      if (w[kk][hh] != (Acc)0) {
        const int k = k0 + kk, h = h0 + hh;
        add_to<Acc>(tile, map_f32, map_fx, use_tile, (k - bk0) * H + (h - bh0), k * nby + h, w[kk][hh]);
      }
}

// Cells [b0, b1) of the visiting order (blocked-sorted when sort0, added to
// map0) and [b1, b2) (sorted when sort1, added to map1) in one launch: the
// first ceil((b1 - b0) / kWsCells) blocks take the first range, so the
// second range's blocks fill the first's last wave.
struct WsRanges {
  int b0, b1, b2;
  int sort0, sort1;
  float* map0_f32;
  float* map1_f32;
  unsigned long long* map0_fx;
  unsigned long long* map1_fx;
};

template <bool kFixed, int kRadixBits>
__global__ void __launch_bounds__(kWsThreads, kFixed ? 2 : 4) window_scatter_kernel(TriangleArgs a, WsRanges rg,
                                                                        const float2* __restrict__ xy_o,
                                                                        const int* __restrict__ order,
                                                                        const float4* __restrict__ rec4,
                                                                        const float* __restrict__ ratio_o,
                                                                        float fx_scale,
                                                                        const int* __restrict__ gate) {
  if (gate_closed(gate)) return;
  const int nb0 = (rg.b1 - rg.b0 + kWsCells - 1) / kWsCells;
  const bool second = (int)blockIdx.x >= nb0;
  const int begin = second ? rg.b1 : rg.b0;
  const int count = second ? rg.b2 : rg.b1;  // end of this block's range
  const int sort_cells = second ? rg.sort1 : rg.sort0;
  float* const map_f32 = second ? rg.map1_f32 : rg.map0_f32;
  unsigned long long* const map_fx = second ? rg.map1_fx : rg.map0_fx;
  const int bid = second ? (int)blockIdx.x - nb0 : (int)blockIdx.x;
  extern __shared__ __align__(16) unsigned char tile_raw[];
  using Acc = typename std::conditional<kFixed, unsigned long long, float>::type;
  Acc* tile = reinterpret_cast<Acc*>(tile_raw);
  constexpr int kCap = kWsSmemBytes / sizeof(Acc);
  __shared__ int red[4][kWsThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // each warp takes kWsWarpCells consecutive cells, each lane kWsCellsPerLane
  // consecutive ones, so cells of one window start bin (sorted together) meet
  // in one lane's running window and then in neighbouring lanes
  const int wbase = begin + bid * kWsCells + warp * kWsWarpCells;
  float nx[kWsCellsPerLane], ny[kWsCellsPerLane], sxs[kWsCellsPerLane], sys[kWsCellsPerLane], rr[kWsCellsPerLane];
  int bk0 = INT_MAX, bk1 = INT_MIN, bh0 = INT_MAX, bh1 = INT_MIN;
  unsigned live = 0;
#pragma unroll
  for (int c = 0; c < kWsCellsPerLane; ++c) {
    const int idx = wbase + lane * kWsCellsPerLane + c;
    nx[c] = ny[c] = sxs[c] = sys[c] = rr[c] = 0.f;
    if (idx < count) {
      const float4 r4 = __ldg(rec4 + idx);
      // positions in visiting order, or in node order read through the order
      const float2 p = order ? __ldg(xy_o + __ldg(order + idx)) : __ldg(xy_o + idx);
      sxs[c] = r4.x;
      sys[c] = r4.y;
      nx[c] = fadd(p.x, r4.z);
      ny[c] = fadd(p.y, r4.w);
      rr[c] = __ldg(ratio_o + idx);
      int k0, k1, h0, h1;
      triangle_bin_range(nx[c], sxs[c], a.xl, a.inv_bsx, a.num_bins_x, k0, k1);
      triangle_bin_range(ny[c], sys[c], a.yl, a.inv_bsy, a.num_bins_y, h0, h1);
      if (k1 > k0 && h1 > h0) {
        live |= 1u << c;
        bk0 = min(bk0, k0);
        bk1 = max(bk1, k1);
        bh0 = min(bh0, h0);
        bh1 = max(bh1, h1);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    bk0 = min(bk0, __shfl_xor_sync(0xffffffffu, bk0, o));
    bk1 = max(bk1, __shfl_xor_sync(0xffffffffu, bk1, o));
    bh0 = min(bh0, __shfl_xor_sync(0xffffffffu, bh0, o));
    bh1 = max(bh1, __shfl_xor_sync(0xffffffffu, bh1, o));
  }
  if (lane == 0) {
    red[0][warp] = bk0;
    red[1][warp] = bk1;
    red[2][warp] = bh0;
    red[3][warp] = bh1;
  }
  __syncthreads();
  bk0 = INT_MAX; bk1 = INT_MIN; bh0 = INT_MAX; bh1 = INT_MIN;
#pragma unroll
  for (int i = 0; i < kWsThreads / 32; ++i) {
    bk0 = min(bk0, red[0][i]);
    bk1 = max(bk1, red[1][i]);
    bh0 = min(bh0, red[2][i]);
    bh1 = max(bh1, red[3][i]);
  }
  if (bk1 <= bk0) return;  // nothing to scatter (uniform across the block)
  const int H = bh1 - bh0;
  const long long box = (long long)(bk1 - bk0) * H;
  if (sort_cells && box < (1 << 16)) {
    // Block-local order: the visiting order is refreshed only every few
    // iterations, while cells keep moving; sorting the block's cells by the
    // bin where their window starts (relative to the block's bounding box)
    // restores the runs that the lane windows and the warp reduction rely on.
    using BlockSort = cub::BlockRadixSort<unsigned, kWsThreads, kWsCellsPerLane, int, kRadixBits>;
    __shared__ typename BlockSort::TempStorage sort_tmp;
    __shared__ float s_cell[5][kWsCells];
    unsigned keys[kWsCellsPerLane];
    int vals[kWsCellsPerLane];
#pragma unroll
    for (int c = 0; c < kWsCellsPerLane; ++c) {
      const int li = warp * kWsWarpCells + lane * kWsCellsPerLane + c;
      keys[c] = (unsigned)box;  // empty cells sort last
      if (live & (1u << c)) {
        int k0, k1, h0, h1;
        triangle_bin_range(nx[c], sxs[c], a.xl, a.inv_bsx, a.num_bins_x, k0, k1);
        triangle_bin_range(ny[c], sys[c], a.yl, a.inv_bsy, a.num_bins_y, h0, h1);
        keys[c] = (unsigned)((k0 - bk0) * H + (h0 - bh0));
      }
      vals[c] = li;
      s_cell[0][li] = nx[c];
      s_cell[1][li] = ny[c];
      s_cell[2][li] = sxs[c];
      s_cell[3][li] = sys[c];
      s_cell[4][li] = rr[c];
    }
    BlockSort(sort_tmp).Sort(keys, vals, 0, 32 - __clz((unsigned)box));
    __syncthreads();
    live = 0;
#pragma unroll
    for (int c = 0; c < kWsCellsPerLane; ++c) {
      const int li = vals[c];
      nx[c] = s_cell[0][li];
      ny[c] = s_cell[1][li];
      sxs[c] = s_cell[2][li];
      sys[c] = s_cell[3][li];
      rr[c] = s_cell[4][li];
      if (keys[c] < (unsigned)box) live |= 1u << c;
    }
  }
  const bool use_tile = box <= kCap;
  if (use_tile) {
    for (int t = threadIdx.x; t < (int)box; t += kWsThreads) tile[t] = (Acc)0;
    __syncthreads();
  }
  const int nby = a.num_bins_y;
  unsigned wide = 0;
  // Running window of this lane: consecutive cells of the lane whose windows
  // start at the same bin accumulate in registers; a new start bin flushes the
  // previous window with direct adds.
  Acc acc[kWin][kWin];
#pragma unroll
  for (int kk = 0; kk < kWin; ++kk)
#pragma unroll
    for (int hh = 0; hh < kWin; ++hh) acc[kk][hh] = (Acc)0;
  int run_key = -1 - lane;  // no window yet: a key no other lane holds
  int run_k0 = 0, run_h0 = 0;
#pragma unroll
  for (int c = 0; c < kWsCellsPerLane; ++c) {
    if (!(live & (1u << c))) continue;
    int k0, k1, h0, h1;
    triangle_bin_range(nx[c], sxs[c], a.xl, a.inv_bsx, a.num_bins_x, k0, k1);
    triangle_bin_range(ny[c], sys[c], a.yl, a.inv_bsy, a.num_bins_y, h0, h1);
    const int nk = k1 - k0, nh = h1 - h0;
    if (nk > kWin || nh > kWin) {
      wide |= 1u << c;
      continue;
    }
    const int key = k0 * nby + h0;
    if (key != run_key) {
      if (run_key >= 0) flush_window<Acc>(acc, run_k0, run_h0, bk0, bh0, H, nby, use_tile, tile, map_f32, map_fx);
#pragma unroll
      for (int kk = 0; kk < kWin; ++kk)
#pragma unroll
        for (int hh = 0; hh < kWin; ++hh) acc[kk][hh] = (Acc)0;
      run_key = key;
      run_k0 = k0;
      run_h0 = h0;
    }
    float py[kWin];
#pragma unroll
    for (int hh = 0; hh < kWin; ++hh) py[hh] = hh < nh ? triangle_overlap(ny[c], sys[c], a.yl, h0 + hh, a.bsy) : 0.f;
#pragma unroll
    for (int kk = 0; kk < kWin; ++kk) {
      if (kk < nk) {
        const float pxr = fmul(triangle_overlap(nx[c], sxs[c], a.xl, k0 + kk, a.bsx), rr[c]);
#pragma unroll
        for (int hh = 0; hh < kWin; ++hh) {
          if (hh < nh) {
            const float area = fmul(pxr, py[hh]);
            acc[kk][hh] += kFixed ? (Acc)to_fixed(area, fx_scale) : (Acc)area;
          }
        }
      }
    }
  }
  // runs of lanes whose windows start at the same bin are summed into the
  // run's first lane; lanes without a window hold unique keys
  {
    const int prev = __shfl_up_sync(0xffffffffu, run_key, 1);
    const bool head = lane == 0 || prev != run_key;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const unsigned later = lane == 31 ? 0u : heads & (0xfffffffeu << lane);
    const int seg_end = later ? __ffs(later) - 2 : 31;
    const int run = head ? seg_end - lane + 1 : 0;
    const int longest = (int)__reduce_max_sync(0xffffffffu, (unsigned)run);
    for (int o = 1; o < longest; o <<= 1) {
      const bool take = lane + o <= seg_end;
#pragma unroll
      for (int kk = 0; kk < kWin; ++kk)
#pragma unroll
        for (int hh = 0; hh < kWin; ++hh) {
          const Acc t = __shfl_down_sync(0xffffffffu, acc[kk][hh], o);
          if (take) acc[kk][hh] += t;
        }
    }
    if (head && run_key >= 0) flush_window<Acc>(acc, run_k0, run_h0, bk0, bh0, H, nby, use_tile, tile, map_f32, map_fx);
  }
  // cells wider than the window: one add per bin
#pragma unroll
  for (int c = 0; c < kWsCellsPerLane; ++c) {
    if (!(wide & (1u << c))) continue;
    int k0, k1, h0, h1;
    triangle_bin_range(nx[c], sxs[c], a.xl, a.inv_bsx, a.num_bins_x, k0, k1);
    triangle_bin_range(ny[c], sys[c], a.yl, a.inv_bsy, a.num_bins_y, h0, h1);
    for (int k = k0; k < k1; ++k) {
      const float pxr = fmul(triangle_overlap(nx[c], sxs[c], a.xl, k, a.bsx), rr[c]);
      for (int h = h0; h < h1; ++h) {
        const float area = fmul(pxr, triangle_overlap(ny[c], sys[c], a.yl, h, a.bsy));
        add_to<Acc>(tile, map_f32, map_fx, use_tile, (k - bk0) * H + (h - bh0), k * nby + h,
                    kFixed ? (Acc)to_fixed(area, fx_scale) : (Acc)area);
      }
    }
  }
  if (use_tile) {
    __syncthreads();
    // one warp per box row, lanes along the row (no index division)
    for (int k = warp; k < bk1 - bk0; k += kWsThreads / 32) {
      const Acc* row = tile + k * H;
      const int gbase = (bk0 + k) * nby + bh0;
      for (int h = lane; h < H; h += 32) {
        const Acc v = row[h];
        if (v != (Acc)0) {
          if (kFixed)
            atomicAdd(map_fx + gbase + h, (unsigned long long)v);
          else
            atomicAdd(map_f32 + gbase + h, (float)v);
        }
      }
    }
  }
}

__global__ void gather_order_xy_kernel(const float2* __restrict__ xy, const int* __restrict__ order, int count,
                                       float2* __restrict__ xy_o, const int* __restrict__ gate) {
  if (gate_closed(gate)) return;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x)
    xy_o[idx] = xy[order[idx]];
}

__global__ void build_records_kernel(const float* __restrict__ sx, const float* __restrict__ sy,
                                     const float* __restrict__ ox, const float* __restrict__ oy,
                                     const float* __restrict__ ratio, const int* __restrict__ order, int count,
                                     float4* __restrict__ rec4, float* __restrict__ ratio_o,
                                     int* __restrict__ inv_order) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    const int i = order[idx];
    rec4[idx] = make_float4(sx[i], sy[i], ox[i], oy[i]);
    ratio_o[idx] = ratio[i];
    if (inv_order) inv_order[i] = idx;
  }
}

// out = (float)((double)init + (double)fixed * 2^-f)  (utility/src/atomic_ops.h:48-54)
__global__ void fixed_to_float_kernel(const long long* fixed, const float* init, double inv_scale,
                                      float* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double base = init ? (double)init[i] : 0.0;
    out[i] = (float)(base + (double)fixed[i] * inv_scale);
  }
}

__global__ void copy_kernel(const float4* __restrict__ src, float4* __restrict__ dst, int n4,
                            const int* __restrict__ gate) {
  if (gate_closed(gate)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x)
    dst[i] = src[i];
}

static int copy_map(const float* src, float* dst, int n, cudaStream_t s) {
  if (src == dst) return DP_OK;
  if ((n & 3) == 0 && ((uintptr_t)src & 15) == 0 && ((uintptr_t)dst & 15) == 0) {
    copy_kernel<<<grid_for(n / 4, 256), 256, 0, s>>>((const float4*)src, (float4*)dst, n / 4, trial_gate());
    return check_launch("copy_map");
  }
  cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) {
    set_error("copy_map: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  return DP_OK;
}

static int validate_triangle(const float* pos, int num_nodes, const float* sx, const float* sy,
                             const float* ox, const float* oy, const float* ratio, int nm, int nf,
                             int nbx, int nby, float bsx, float bsy, const float* out) {
  DP_REQUIRE(pos && sx && sy && ox && oy && ratio && out, "density_map: null pointer argument");
  DP_REQUIRE(num_nodes >= 0 && nm >= 0 && nf >= 0 && nm + nf <= num_nodes,
             "density_map: inconsistent node counts (nodes %d movable %d filler %d)", num_nodes, nm, nf);
  DP_REQUIRE(nbx > 0 && nby > 0 && (long long)nbx * nby < (1ll << 31), "density_map: bad bin grid %dx%d", nbx, nby);
  DP_REQUIRE(bsx > 0 && bsy > 0, "density_map: bin sizes must be positive");
  return DP_OK;
}

static TriangleArgs make_args(const float* pos, int num_nodes, const float* sx, const float* sy,
                              const float* ox, const float* oy, const float* ratio, float xl,
                              float yl, float bsx, float bsy, float ibx, float iby, int nm, int nf,
                              int nbx, int nby, const int* sorted) {
  TriangleArgs a;
  a.x = pos; a.y = pos + num_nodes;
  a.sx = sx; a.sy = sy; a.ox = ox; a.oy = oy; a.ratio = ratio;
  a.xl = xl; a.yl = yl; a.bsx = bsx; a.bsy = bsy; a.inv_bsx = ibx; a.inv_bsy = iby;
  a.num_bins_x = nbx; a.num_bins_y = nby;
  a.num_movable = nm; a.num_filler = nf; a.filler_begin = num_nodes - nf;
  a.sorted_node_map = sorted;
  return a;
}

// Exact-overlap scatter of one node range (fixed_node_flag selects the
// boundary-extension rule of exact_density_function).
template <bool kFixed>
__global__ void exact_scatter_kernel(const float* x, const float* y, const float* sx, const float* sy,
                                     const float* bcx, const float* bcy, int begin, int end,
                                     float xl, float yl, float xh, float yh, float bsx, float bsy,
                                     int nbx, int nby, bool fixed_node_flag, bool use_centers,
                                     float fx_scale, float* map_f32, unsigned long long* map_fx) {
  for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    float bxl = x[i], byl = y[i];
    float bxh = fadd(bxl, sx[i]), byh = fadd(byl, sy[i]);
    int k0 = max((int)__fdiv_rn(fsub(bxl, xl), bsx), 0);
    int k1 = min((int)ceilf(__fdiv_rn(fsub(bxh, xl), bsx)) + 1, nbx);
    int h0 = max((int)__fdiv_rn(fsub(byl, yl), bsy), 0);
    int h1 = min((int)ceilf(__fdiv_rn(fsub(byh, yl), bsy)) + 1, nby);
    float wx = fsub(bxh, bxl), wy = fsub(byh, byl);
    for (int k = k0; k < k1; ++k) {
      float cx = use_centers ? bcx[k] : fadd(fadd(xl, fmul((float)k, bsx)), bsx / 2);
      float px = exact_overlap(bxl, wx, cx, bsx, xl, xh, fixed_node_flag);
      for (int h = h0; h < h1; ++h) {
        float cy = use_centers ? bcy[h] : fadd(fadd(yl, fmul((float)h, bsy)), bsy / 2);
        float py = exact_overlap(byl, wy, cy, bsy, yl, yh, fixed_node_flag);
        float area = fmul(px, py);
        int bin = k * nby + h;
        if (kFixed)
          atomicAdd(map_fx + bin, (unsigned long long)to_fixed(area, fx_scale));
        else
          atomicAdd(map_f32 + bin, area);
      }
    }
  }
}

// DensityMap exact-overlap scatter (density_map/src/density_map.cpp:
// distributeBox2Bin): bin size (xh-xl)/num_bins in float, y range widened by
// two bins each side, the last bin in each direction extended to the cell edge.
template <bool kFixed>
__global__ void box_scatter_kernel(const float* x, const float* y, const float* sx, const float* sy, int begin,
                                   int end, float xl, float yl, float xh, float yh, int nbx, int nby,
                                   float fx_scale, float* map_f32, unsigned long long* map_fx) {
  const float bsx = __fdiv_rn(fsub(xh, xl), (float)nbx);
  const float bsy = __fdiv_rn(fsub(yh, yl), (float)nby);
  for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    float bxl = x[i], byl = y[i];
    float bxh = fadd(bxl, sx[i]), byh = fadd(byl, sy[i]);
    int k0 = max((int)__fdiv_rn(fsub(bxl, xl), bsx), 0);
    int k1 = min((int)ceilf(__fdiv_rn(fsub(bxh, xl), bsx)) + 1, nbx);
    float two_bsy = fmul(2.0f, bsy);
    int h0 = max((int)__fdiv_rn(fsub(fsub(byl, yl), two_bsy), bsy), 0);
    int h1 = min((int)ceilf(__fdiv_rn(fadd(fsub(byh, yl), two_bsy), bsy)) + 1, nby);
    for (int k = k0; k < k1; ++k) {
      float bin_xl = fadd(xl, fmul(bsx, (float)k));
      float bin_xh = fminf(fadd(bin_xl, bsx), xh);
      if (k + 1 == nbx) bin_xh = bxh;
      float px = fmaxf(0.0f, fsub(fminf(bxh, bin_xh), fmaxf(bxl, bin_xl)));
      for (int h = h0; h < h1; ++h) {
        float bin_yl = fadd(yl, fmul(bsy, (float)h));
        float bin_yh = fminf(fadd(bin_yl, bsy), yh);
        if (h + 1 == nby) bin_yh = byh;
        float py = fmaxf(0.0f, fsub(fminf(byh, bin_yh), fmaxf(byl, bin_yl)));
        float area = fmul(px, py);
        int bin = k * nby + h;
        if (kFixed)
          atomicAdd(map_fx + bin, (unsigned long long)to_fixed(area, fx_scale));
        else
          atomicAdd(map_f32 + bin, area);
      }
    }
  }
}

__global__ void clamp_max_kernel(float* map, int n, float vmax) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    map[i] = fminf(map[i], vmax);
}

// order-preserving float <-> uint32 key: key(a) < key(b) iff a < b; key 0 is
// below every float, so a zero-filled slot is a valid start for atomicMax
__device__ __forceinline__ unsigned float_key(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void overflow_kernel(const float* __restrict__ map, int n, double target_area,
                                double* partials, unsigned* maxkey) {
  double s = 0.0;
  float m = -INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float d = map[i];
    double over = (double)d - target_area;
    s += over > 0.0 ? over : 0.0;
    m = fmaxf(m, d);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxkey, float_key(m));  // max is order independent
  block_partial(s, partials);
}

// First map of the split scatter: converts it from fixed point (fixed != NULL)
// or reads it, optionally copies it to copy_to (start of the second map), and
// reduces its overflow sum and maximum as overflow_kernel does.
// The movable-only map (from the fixed-point sums, or as scattered) with its
// overflow partials and max (when partials is given), and the full map:
// copy_to = first, or copy_to += first when add_to_copy (copy_to then holds
// the fillers' own map).
__global__ void first_map_kernel(const long long* __restrict__ fixed, const float* __restrict__ init,
                                 double inv_scale, float* first, float* __restrict__ copy_to, int add_to_copy,
                                 int n, double target_area, double* partials, unsigned* maxkey,
                                 const int* __restrict__ gate) {
  if (gate_closed(gate)) return;
  double s = 0.0;
  float m = -INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float d;
    if (fixed) {
      d = (float)((init ? (double)init[i] : 0.0) + (double)fixed[i] * inv_scale);
      first[i] = d;
    } else {
      d = first[i];
    }
    if (copy_to) copy_to[i] = add_to_copy ? fadd(d, copy_to[i]) : d;
    const double over = (double)d - target_area;
    s += over > 0.0 ? over : 0.0;
    m = fmaxf(m, d);
  }
  if (!partials) return;  // uniform: no overflow wanted
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxkey, float_key(m));
  block_partial(s, partials);
}

__global__ void overflow_finish_kernel(double* out2, const unsigned* maxkey, double bin_area,
                                       float* out2_f32, const double* partials, int count) {
  double total = finish_sum(partials, count);
  if (threadIdx.x != 0) return;
  out2[0] = total;
  double mx = (double)key_float(*maxkey) / bin_area;
  out2[1] = mx;
  if (out2_f32) {
    out2_f32[0] = (float)out2[0];
    out2_f32[1] = (float)mx;
  }
}

}  // namespace dpb

using namespace dpb;

extern "C" int dp_density_map_f32(const float* pos, int num_nodes, const float* sx, const float* sy,
                                  const float* ox, const float* oy, const float* ratio,
                                  const float* init, float xl, float yl, float xh, float yh,
                                  float bsx, float bsy, float ibx, float iby, int nm, int nf,
                                  int nbx, int nby, const int* sorted, float* out,
                                  dp_stream_t stream) {
  int rc = validate_triangle(pos, num_nodes, sx, sy, ox, oy, ratio, nm, nf, nbx, nby, bsx, bsy, out);
  if (rc) return rc;
  cudaStream_t s = as_stream(stream);
  int nbins = nbx * nby;
  if (init) {
    rc = copy_map(init, out, nbins, s);
    if (rc) return rc;
  } else {
    cudaMemsetAsync(out, 0, sizeof(float) * nbins, s);
  }
  int total = nm + nf;
  if (total == 0) return DP_OK;
  TriangleArgs a = make_args(pos, num_nodes, sx, sy, ox, oy, ratio, xl, yl, bsx, bsy, ibx, iby, nm, nf, nbx, nby, sorted);
  triangle_scatter_kernel<false><<<grid_for(total, 256, 16), 256, 0, s>>>(a, total, 0.f, out, nullptr);
  return check_launch("dp_density_map_f32");
}

extern "C" int dp_density_map_fx64(const float* pos, int num_nodes, const float* sx, const float* sy,
                                   const float* ox, const float* oy, const float* ratio,
                                   const float* init, float xl, float yl, float xh, float yh,
                                   float bsx, float bsy, float ibx, float iby, int nm, int nf,
                                   int nbx, int nby, const int* sorted, int fraction_bits,
                                   int64_t* scratch, float* out, dp_stream_t stream) {
  int rc = validate_triangle(pos, num_nodes, sx, sy, ox, oy, ratio, nm, nf, nbx, nby, bsx, bsy, out);
  if (rc) return rc;
  DP_REQUIRE(scratch, "dp_density_map_fx64: scratch_fixed is required");
  DP_REQUIRE(fraction_bits >= 0 && fraction_bits <= 62, "dp_density_map_fx64: bad fraction_bits %d", fraction_bits);
  cudaStream_t s = as_stream(stream);
  int nbins = nbx * nby;
  cudaMemsetAsync(scratch, 0, sizeof(int64_t) * nbins, s);
  int total = nm + nf;
  float scale = ldexpf(1.0f, fraction_bits);
  if (total > 0) {
    TriangleArgs a = make_args(pos, num_nodes, sx, sy, ox, oy, ratio, xl, yl, bsx, bsy, ibx, iby, nm, nf, nbx, nby, sorted);
    triangle_scatter_kernel<true><<<grid_for(total, 256, 16), 256, 0, s>>>(
        a, total, scale, nullptr, reinterpret_cast<unsigned long long*>(scratch));
    rc = check_launch("dp_density_map_fx64 scatter");
    if (rc) return rc;
  }
  fixed_to_float_kernel<<<grid_for(nbins, 256), 256, 0, s>>>((const long long*)scratch, init,
                                                            ldexp(1.0, -fraction_bits), out, nbins);
  return check_launch("dp_density_map_fx64 convert");
}

extern "C" int dp_fixed_density_map(const float* pos, int num_nodes, const float* sx, const float* sy,
                                    const float* bcx, const float* bcy, float xl, float yl, float xh,
                                    float yh, float bsx, float bsy, int nm, int nt, int nbx, int nby,
                                    int deterministic, int fraction_bits, int64_t* scratch,
                                    float* out, dp_stream_t stream) {
  DP_REQUIRE(pos && sx && sy && bcx && bcy && out, "dp_fixed_density_map: null pointer argument");
  DP_REQUIRE(nm >= 0 && nt >= 0 && nm + nt <= num_nodes, "dp_fixed_density_map: bad node counts");
  DP_REQUIRE(nbx > 0 && nby > 0, "dp_fixed_density_map: bad bin grid");
  DP_REQUIRE(!deterministic || scratch, "dp_fixed_density_map: deterministic mode needs scratch_fixed");
  cudaStream_t s = as_stream(stream);
  int nbins = nbx * nby;
  cudaMemsetAsync(out, 0, sizeof(float) * nbins, s);
  if (nt == 0) return DP_OK;
  const float* x = pos;
  const float* y = pos + num_nodes;
  int blocks = grid_for(nt, 128, 8);
  if (deterministic) {
    cudaMemsetAsync(scratch, 0, sizeof(int64_t) * nbins, s);
    exact_scatter_kernel<true><<<blocks, 128, 0, s>>>(x, y, sx, sy, bcx, bcy, nm, nm + nt, xl, yl, xh, yh,
                                                      bsx, bsy, nbx, nby, true, true,
                                                      ldexpf(1.0f, fraction_bits), nullptr,
                                                      reinterpret_cast<unsigned long long*>(scratch));
    int rc = check_launch("dp_fixed_density_map scatter");
    if (rc) return rc;
    fixed_to_float_kernel<<<grid_for(nbins, 256), 256, 0, s>>>((const long long*)scratch, nullptr,
                                                              ldexp(1.0, -fraction_bits), out, nbins);
    rc = check_launch("dp_fixed_density_map convert");
    if (rc) return rc;
  } else {
    exact_scatter_kernel<false><<<blocks, 128, 0, s>>>(x, y, sx, sy, bcx, bcy, nm, nm + nt, xl, yl, xh, yh,
                                                       bsx, bsy, nbx, nby, true, true, 0.f, out, nullptr);
    int rc = check_launch("dp_fixed_density_map scatter");
    if (rc) return rc;
  }
  float vmax = (float)((double)bsx * (double)bsy);
  clamp_max_kernel<<<grid_for(nbins, 256), 256, 0, s>>>(out, nbins, vmax);
  return check_launch("dp_fixed_density_map clamp");
}

extern "C" int dp_density_map_exact(const float* pos, int num_nodes, const float* sx, const float* sy,
                                    const int* rb, const int* re, int nranges, float xl, float yl,
                                    float xh, float yh, int nbx, int nby, int deterministic,
                                    int fraction_bits, int64_t* scratch, float* out, dp_stream_t stream) {
  DP_REQUIRE(pos && sx && sy && out, "dp_density_map_exact: null pointer argument");
  DP_REQUIRE(nranges >= 0 && (nranges == 0 || (rb && re)), "dp_density_map_exact: bad ranges");
  DP_REQUIRE(nbx > 0 && nby > 0, "dp_density_map_exact: bad bin grid");
  DP_REQUIRE(!deterministic || scratch, "dp_density_map_exact: deterministic mode needs scratch_fixed");
  cudaStream_t s = as_stream(stream);
  int nbins = nbx * nby;
  const float* x = pos;
  const float* y = pos + num_nodes;
  for (int r = 0; r < nranges; ++r) {
    DP_REQUIRE(rb[r] >= 0 && re[r] <= num_nodes, "dp_density_map_exact: range %d out of bounds", r);
    int n = re[r] - rb[r];
    if (n <= 0) continue;
    if (deterministic) {
      // each range is converted onto the running map on its own, as the reference does
      cudaMemsetAsync(scratch, 0, sizeof(int64_t) * nbins, s);
      box_scatter_kernel<true><<<grid_for(n, 128, 8), 128, 0, s>>>(
          x, y, sx, sy, rb[r], re[r], xl, yl, xh, yh, nbx, nby, ldexpf(1.0f, fraction_bits), nullptr,
          reinterpret_cast<unsigned long long*>(scratch));
      int rc = check_launch("dp_density_map_exact scatter");
      if (rc) return rc;
      fixed_to_float_kernel<<<grid_for(nbins, 256), 256, 0, s>>>((const long long*)scratch, out,
                                                                ldexp(1.0, -fraction_bits), out, nbins);
      rc = check_launch("dp_density_map_exact convert");
      if (rc) return rc;
    } else {
      box_scatter_kernel<false><<<grid_for(n, 128, 8), 128, 0, s>>>(x, y, sx, sy, rb[r], re[r], xl, yl, xh, yh,
                                                                    nbx, nby, 0.f, out, nullptr);
      int rc = check_launch("dp_density_map_exact scatter");
      if (rc) return rc;
    }
  }
  return DP_OK;
}

extern "C" int dp_density_overflow(const float* map, int nbins, double target_area, double bin_area,
                                   double* out2, float* out2_f32, dp_stream_t stream) {
  DP_REQUIRE(map && out2 && nbins > 0, "dp_density_overflow: bad arguments");
  cudaStream_t s = as_stream(stream);
  // out2: [0] overflow, [1] max density, [2] max key, [3..] block partials
  int blocks = grid_for(nbins, 256, 4);
  unsigned* maxslot = reinterpret_cast<unsigned*>(out2 + 2);
  cudaMemsetAsync(maxslot, 0, sizeof(double), s);
  overflow_kernel<<<blocks, 256, 0, s>>>(map, nbins, target_area, out2 + 3, maxslot);
  int rc = check_launch("dp_density_overflow");
  if (rc) return rc;
  overflow_finish_kernel<<<1, kReduceThreads, 0, s>>>(out2, maxslot, bin_area, out2_f32, out2 + 3, blocks);
  return check_launch("dp_density_overflow finish");
}

// xy_o[idx] = xy[order[idx]]: positions in visiting order
extern "C" int dp_gather_order_xy(const float* xy, const int* order, int count, float* xy_o, dp_stream_t stream) {
  DP_REQUIRE(xy && xy_o && (count == 0 || order), "dp_gather_order_xy: null pointer");
  DP_REQUIRE(((uintptr_t)xy & 7) == 0 && ((uintptr_t)xy_o & 7) == 0, "dp_gather_order_xy: misaligned xy / xy_o");
  if (count == 0) return DP_OK;
  gather_order_xy_kernel<<<grid_for(count, 256, 8), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<const float2*>(xy), order, count, reinterpret_cast<float2*>(xy_o), trial_gate());
  return check_launch("dp_gather_order_xy");
}

// Per-cell records for the order-driven kernels: rec4[idx] = (sx, sy, ox, oy)
// and ratio_o[idx] of node order[idx]; inv_order[order[idx]] = idx (optional).
extern "C" int dp_build_cell_records(const float* sx, const float* sy, const float* ox, const float* oy,
                                     const float* ratio, const int* order, int count, float* rec4, float* ratio_o,
                                     int* inv_order, dp_stream_t stream) {
  DP_REQUIRE(sx && sy && ox && oy && ratio && order && rec4 && ratio_o, "dp_build_cell_records: null pointer");
  DP_REQUIRE(((uintptr_t)rec4 & 15) == 0, "dp_build_cell_records: rec4 must be 16-byte aligned");
  if (count == 0) return DP_OK;
  build_records_kernel<<<grid_for(count, 256, 8), 256, 0, as_stream(stream)>>>(
      sx, sy, ox, oy, ratio, order, count, reinterpret_cast<float4*>(rec4), ratio_o, inv_order);
  return check_launch("dp_build_cell_records");
}

// Order-driven scatter (see window_scatter_kernel): the cells order[0..count)
// with their records, positions interleaved in xy.
namespace {

struct OrderedScatter {
  TriangleArgs a;
  const float2* xy_o;  // visiting order, or node order when `order` is given
  const int* order;
  const float4* rec4;
  const float* ratio_o;
  cudaStream_t s;
};

// adds the cells of rg's two ranges of the visiting order onto their maps
// (fp32, or the fixed-point scratch maps), in one launch
template <int kRadixBits>
int scatter_ranges_r(const OrderedScatter& o, const WsRanges& rg, int deterministic, int fraction_bits) {
  int rc = deterministic ? opt_in_smem(window_scatter_kernel<true, kRadixBits>, kWsSmemBytes, "density scatter")
                         : opt_in_smem(window_scatter_kernel<false, kRadixBits>, kWsSmemBytes, "density scatter");
  if (rc) return rc;
  const int blocks = ceil_div(rg.b1 - rg.b0, kWsCells) + ceil_div(rg.b2 - rg.b1, kWsCells);
  if (blocks <= 0) return DP_OK;
  if (deterministic)
    window_scatter_kernel<true, kRadixBits><<<blocks, kWsThreads, kWsSmemBytes, o.s>>>(
        o.a, rg, o.xy_o, o.order, o.rec4, o.ratio_o, ldexpf(1.0f, fraction_bits), trial_gate());
  else
    window_scatter_kernel<false, kRadixBits><<<blocks, kWsThreads, kWsSmemBytes, o.s>>>(
        o.a, rg, o.xy_o, o.order, o.rec4, o.ratio_o, 0.f, trial_gate());
  return check_launch("dp_density_map_ordered scatter");
}

// adds cells [begin, end) of the visiting order onto out (fp32) or scratch (fixed)
int scatter_range(const OrderedScatter& o, int begin, int end, int deterministic, int fraction_bits, int64_t* scratch,
                  float* out, int sort_cells = 1) {
  if (end <= begin) return DP_OK;
  WsRanges rg;
  memset(&rg, 0, sizeof(rg));
  rg.b0 = begin;
  rg.b1 = rg.b2 = end;
  rg.sort0 = sort_cells;
  rg.map0_f32 = out;
  rg.map0_fx = reinterpret_cast<unsigned long long*>(scratch);
  return scatter_ranges_r<4>(o, rg, deterministic, fraction_bits);
}

int convert_fixed(const int64_t* scratch, const float* init, int fraction_bits, float* out, int nbins,
                  cudaStream_t s) {
  fixed_to_float_kernel<<<grid_for(nbins, 256), 256, 0, s>>>((const long long*)scratch, init,
                                                            ldexp(1.0, -fraction_bits), out, nbins);
  return check_launch("dp_density_map_ordered convert");
}

int start_map(const float* init, float* out, int nbins, cudaStream_t s) {
  if (init) return copy_map(init, out, nbins, s);
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * nbins, s);
  if (e != cudaSuccess) {
    set_error("dp_density_map_ordered: cudaMemsetAsync: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  return DP_OK;
}

int ordered_setup(const char* who, const float* xy_o, const int* order, const float* rec4, const float* ratio_o,
                  int count, float xl,
                  float yl, float bsx, float bsy, float ibx, float iby, int nbx, int nby, int deterministic,
                  int fraction_bits, int64_t* scratch, dp_stream_t stream, OrderedScatter& o) {
  DP_REQUIRE(xy_o && rec4 && ratio_o, "%s: null pointer", who);
  DP_REQUIRE(((uintptr_t)xy_o & 7) == 0 && ((uintptr_t)rec4 & 15) == 0, "%s: misaligned xy_o/rec4", who);
  DP_REQUIRE(nbx > 0 && nby > 0 && (long long)nbx * nby < (1ll << 31), "%s: bad bin grid", who);
  DP_REQUIRE(bsx > 0 && bsy > 0 && count >= 0, "%s: bad geometry", who);
  DP_REQUIRE(!deterministic || scratch, "%s: deterministic mode needs scratch_fixed", who);
  DP_REQUIRE(!deterministic || (fraction_bits >= 0 && fraction_bits <= 62), "%s: bad fraction_bits", who);
  memset(&o.a, 0, sizeof(o.a));
  o.a.xl = xl; o.a.yl = yl; o.a.bsx = bsx; o.a.bsy = bsy; o.a.inv_bsx = ibx; o.a.inv_bsy = iby;
  o.a.num_bins_x = nbx; o.a.num_bins_y = nby;
  o.xy_o = reinterpret_cast<const float2*>(xy_o);
  o.order = order;
  o.rec4 = reinterpret_cast<const float4*>(rec4);
  o.ratio_o = ratio_o;
  o.s = as_stream(stream);
  return DP_OK;
}

}  // namespace

// Order-driven scatter (see window_scatter_kernel): cells 0..count of the
// visiting order, positions (xy_o) and attributes (rec4, ratio_o) in that order.
extern "C" int dp_density_map_ordered(const float* xy_o, const int* order, const float* rec4, const float* ratio_o,
                                      int count,
                                      const float* init, float xl, float yl, float xh, float yh, float bsx,
                                      float bsy, float ibx, float iby, int nbx, int nby, int deterministic,
                                      int fraction_bits, int64_t* scratch, float* out, dp_stream_t stream) {
  OrderedScatter o;
  int rc = ordered_setup("dp_density_map_ordered", xy_o, order, rec4, ratio_o, count, xl, yl, bsx, bsy, ibx, iby, nbx, nby,
                         deterministic, fraction_bits, scratch, stream, o);
  if (rc) return rc;
  DP_REQUIRE(out, "dp_density_map_ordered: null output");
  const int nbins = nbx * nby;
  if (deterministic) {
    cudaMemsetAsync(scratch, 0, sizeof(int64_t) * nbins, o.s);
    rc = scatter_range(o, 0, count, 1, fraction_bits, scratch, nullptr);
    if (rc) return rc;
    return convert_fixed(scratch, init, fraction_bits, out, nbins, o.s);
  }
  rc = start_map(init, out, nbins, o.s);
  if (rc) return rc;
  return scatter_range(o, 0, count, 0, 0, nullptr, out);
}

// Two maps from one pass over the cells: out_first = init + cells
// [0, num_first), out_all = init + cells [0, count), and optionally the
// overflow reduction of out_first (as dp_density_overflow) fused into the
// pass that finishes it.  Fixed point: the int64 sums are exact, so both maps
// equal separate scatters bit for bit.  fp32: the second map continues from
// the first, i.e. the float additions happen in one of the orders the atomic
// scatter of all cells can take.  Only the first range gets the block-local
// sort (the second one is the engine's fillers, spread about one per bin, for
// which runs of equal start bins stay short anyway).
extern "C" int dp_density_map_ordered_split(const float* xy_o, const int* order, const float* rec4,
                                            const float* ratio_o, int num_first, int count, const float* init,
                                            float xl, float yl, float xh, float yh, float bsx, float bsy, float ibx,
                                            float iby, int nbx, int nby, int deterministic, int fraction_bits,
                                            int64_t* scratch, float* out_first, float* out_all, double target_area,
                                            double bin_area, double* overflow_out, dp_stream_t stream) {
  OrderedScatter o;
  int rc = ordered_setup("dp_density_map_ordered_split", xy_o, order, rec4, ratio_o, count, xl, yl, bsx, bsy, ibx, iby, nbx,
                         nby, deterministic, fraction_bits, scratch, stream, o);
  if (rc) return rc;
  DP_REQUIRE(out_first && out_all && out_first != out_all, "dp_density_map_ordered_split: bad outputs");
  DP_REQUIRE(num_first >= 0 && num_first <= count, "dp_density_map_ordered_split: bad num_first");
  DP_REQUIRE(!overflow_out || bin_area > 0, "dp_density_map_ordered_split: bad bin area");
  const int nbins = nbx * nby;
  const int blocks = grid_for(nbins, 256, 4);
  unsigned* maxslot = overflow_out ? reinterpret_cast<unsigned*>(overflow_out + 2) : nullptr;
  if (deterministic) {
    cudaMemsetAsync(scratch, 0, sizeof(int64_t) * nbins, o.s);
    rc = scatter_range(o, 0, num_first, 1, fraction_bits, scratch, nullptr);
    if (rc) return rc;
    if (overflow_out) {
      cudaMemsetAsync(maxslot, 0, sizeof(double), o.s);
      first_map_kernel<<<blocks, 256, 0, o.s>>>((const long long*)scratch, init, ldexp(1.0, -fraction_bits),
                                                 out_first, nullptr, 0, nbins, target_area, overflow_out + 3, maxslot,
                                                 trial_gate());
      rc = check_launch("dp_density_map_ordered_split first map");
      if (rc) return rc;
      overflow_finish_kernel<<<1, kReduceThreads, 0, o.s>>>(overflow_out, maxslot, bin_area, nullptr,
                                                            overflow_out + 3, blocks);
      rc = check_launch("dp_density_map_ordered_split overflow");
    } else {
      rc = convert_fixed(scratch, init, fraction_bits, out_first, nbins, o.s);
    }
    if (rc) return rc;
    rc = scatter_range(o, num_first, count, 1, fraction_bits, scratch, nullptr, 0);
    if (rc) return rc;
    return convert_fixed(scratch, init, fraction_bits, out_all, nbins, o.s);
  }
  // fp32: both ranges in one launch (the second range's blocks fill the
  // first's last wave), the first onto out_first = init, the second onto
  // out_all = 0; then out_all += out_first, with the overflow of out_first
  rc = start_map(init, out_first, nbins, o.s);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(out_all, 0, sizeof(float) * nbins, o.s);
  if (e != cudaSuccess) {
    set_error("dp_density_map_ordered_split: cudaMemsetAsync: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  WsRanges rg;
  memset(&rg, 0, sizeof(rg));
  rg.b0 = 0;
  rg.b1 = num_first;
  rg.b2 = count;
  rg.sort0 = 1;  // the movable cells: block-local sort (their order goes stale)
  rg.sort1 = 0;  // the fillers: about one per bin, runs stay short
  rg.map0_f32 = out_first;
  rg.map1_f32 = out_all;
  rc = scatter_ranges_r<4>(o, rg, 0, 0);
  if (rc) return rc;
  if (overflow_out) cudaMemsetAsync(maxslot, 0, sizeof(double), o.s);
  first_map_kernel<<<blocks, 256, 0, o.s>>>(nullptr, nullptr, 0.0, out_first, out_all, 1, nbins, target_area,
                                             overflow_out ? overflow_out + 3 : nullptr, maxslot, trial_gate());
  rc = check_launch("dp_density_map_ordered_split first map");
  if (rc || !overflow_out) return rc;
  overflow_finish_kernel<<<1, kReduceThreads, 0, o.s>>>(overflow_out, maxslot, bin_area, nullptr,
                                                        overflow_out + 3, blocks);
  return check_launch("dp_density_map_ordered_split overflow");
}

// ---------------------------------------------------------------- allocation-free variant
// Some callers of this library cannot allocate device memory at the point
// where they place: hosts that reserve the whole GPU up front under a fixed
// memory budget (another allocation would fail or evict their own data), and
// FFI hosts (Go / Java / JavaScript bindings) that never link the CUDA
// allocator.  dp_density_map_fx64_noalloc serves them: the deterministic
// scatter's int64 scratch map lives in the file-scope device array below, of
// at most DP_NOALLOC_MAX_BINS bins, which every GPU that loads the library
// holds until the process exits.
static __device__ __align__(256) unsigned long long g_noalloc_fixed_map[DP_NOALLOC_MAX_BINS];

// Host code may not use g_noalloc_fixed_map as an address: the symbol names a
// host-side stand-in.  The device address belongs to the CUDA context that
// loaded this library's module on the device, so it is looked up with that
// device current and cached per device together with the context's unique ID
// (cuCtxGetId, never reused within a process).  A call under another context
// -- the primary context re-created after cudaDeviceReset, or a context the
// host made itself with the driver API -- looks the address up again.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);

static int current_context_id(unsigned long long* id) {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PfnCtxGetId>(f);
  });
  DP_REQUIRE(get_current && get_id, "dp_density_map_fx64_noalloc: the driver offers no cuCtxGetCurrent / cuCtxGetId");
  *id = 0;  // 0: no context is current on this thread
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return DP_OK;
  if (get_id(ctx, id) != CUDA_SUCCESS) {
    set_error("dp_density_map_fx64_noalloc: cuCtxGetId failed");
    return DP_ERR_CUDA;
  }
  return DP_OK;
}

static int noalloc_scratch_address(int64_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("dp_density_map_fx64_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  constexpr int kMaxDevices = 64;
  DP_REQUIRE(dev >= 0 && dev < kMaxDevices, "dp_density_map_fx64_noalloc: device ordinal %d out of range", dev);
  unsigned long long ctx_id = 0;
  int rc = current_context_id(&ctx_id);
  if (rc) return rc;
  static void* addr[kMaxDevices] = {};
  static unsigned long long addr_ctx[kMaxDevices] = {};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev] || ctx_id == 0 || addr_ctx[dev] != ctx_id) {
    // (with no context current, this runtime call makes the device's primary
    // context current; its ID is read afterwards)
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_fixed_map);
    if (e != cudaSuccess || !p) {
      set_error("dp_density_map_fx64_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return DP_ERR_CUDA;
    }
    if (ctx_id == 0) {
      rc = current_context_id(&ctx_id);
      if (rc) return rc;
    }
    addr[dev] = p;
    addr_ctx[dev] = ctx_id;
  }
  *out = static_cast<int64_t*>(addr[dev]);
  return DP_OK;
}

extern "C" int dp_density_map_fx64_noalloc(const float* pos, int num_nodes, const float* sx, const float* sy,
                                           const float* ox, const float* oy, const float* ratio, const float* init,
                                           float xl, float yl, float xh, float yh, float bsx, float bsy, float ibx,
                                           float iby, int nm, int nf, int nbx, int nby, const int* sorted,
                                           int fraction_bits, float* out, dp_stream_t stream) {
  DP_REQUIRE(nbx > 0 && nby > 0, "dp_density_map_fx64_noalloc: bad bin grid %dx%d", nbx, nby);
  DP_REQUIRE((long long)nbx * nby <= DP_NOALLOC_MAX_BINS,
             "dp_density_map_fx64_noalloc: %d x %d bins exceed the built-in scratch of %d bins; "
             "use dp_density_map_fx64 with a caller-owned scratch map",
             nbx, nby, (int)DP_NOALLOC_MAX_BINS);
  int64_t* scratch = nullptr;
  int rc = noalloc_scratch_address(&scratch);
  if (rc) return rc;
  // the scratch is zero-filled inside dp_density_map_fx64 before the scatter
  return dp_density_map_fx64(pos, num_nodes, sx, sy, ox, oy, ratio, init, xl, yl, xh, yh, bsx, bsy, ibx, iby, nm,
                             nf, nbx, nby, sorted, fraction_bits, scratch, out, stream);
}

// ---------------------------------------------------------------- visiting order
// The scattered cells (movable, then fillers) bucketed by the bin where their
// stretched footprint starts: 16 x 16-bin tiles in serpentine order, bin
// inside the tile, movable cells before fillers.  A counting sort: one pass
// computes each cell's bucket and counts the buckets, an exclusive scan turns
// counts into starts, a second pass places the cells (the order inside a
// bucket is whatever the atomics give: every visiting order is valid for the
// scatter and the field gather).
namespace dpb {

constexpr int kScanThreads = 1024;

__device__ __forceinline__ unsigned cell_bucket(float x, float ox, float lo, float inv_bs, int nbins) {
  int b = (int)fmul(fsub(fadd(x, ox), lo), inv_bs);
  return (unsigned)min(max(b, 0), nbins - 1);
}

__global__ void order_keys_kernel(const float* __restrict__ pos, int num_nodes, const float* __restrict__ ox,
                                  const float* __restrict__ oy, int nm, int nf, float xl, float yl, float ibx,
                                  float iby, int nbx, int nby, unsigned tile_buckets, unsigned* __restrict__ keys,
                                  unsigned* __restrict__ hist) {
  const int count = nm + nf;
  const int tiles_y = (nby + 15) >> 4;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int node = i < nm ? i : num_nodes - nf + (i - nm);
    const unsigned kx = cell_bucket(pos[node], ox[node], xl, ibx, nbx);
    const unsigned hy = cell_bucket(pos[num_nodes + node], oy[node], yl, iby, nby);
    const unsigned tx = kx >> 4;
    unsigned ty = hy >> 4;
    if (tx & 1u) ty = (unsigned)tiles_y - 1u - ty;
    const unsigned key = (((tx * (unsigned)tiles_y + ty) << 8) | ((kx & 15u) << 4) | (hy & 15u)) +
                         (i < nm ? 0u : tile_buckets);
    keys[i] = key;
    atomicAdd(hist + key, 1u);
  }
}

// exclusive scan of n counts in place: per-block scans with block totals,
// then the totals (one block), then the totals added back
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* warp_sums, unsigned& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    unsigned w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  total = warp_sums[(blockDim.x >> 5) - 1];
  const unsigned before = warp == 0 ? 0u : warp_sums[warp - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_blocks_kernel(unsigned* data, int n, unsigned* block_totals) {
  __shared__ unsigned warp_sums[32];
  const int i = blockIdx.x * kScanThreads + threadIdx.x;
  const unsigned v = i < n ? data[i] : 0u;
  unsigned total;
  const unsigned ex = block_exclusive_scan(v, warp_sums, total);
  if (i < n) data[i] = ex;
  if (threadIdx.x == 0) block_totals[blockIdx.x] = total;
}

// one block scans the block totals (at most kScanThreads * kScanThreads blocks)
__global__ void __launch_bounds__(kScanThreads) scan_totals_kernel(unsigned* totals, int nblocks) {
  __shared__ unsigned warp_sums[32];
  __shared__ unsigned carry;
  if (threadIdx.x == 0) carry = 0u;
  __syncthreads();
  for (int base = 0; base < nblocks; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const unsigned v = i < nblocks ? totals[i] : 0u;
    unsigned total;
    const unsigned ex = block_exclusive_scan(v, warp_sums, total);
    if (i < nblocks) totals[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
}

__global__ void add_block_offsets_kernel(unsigned* data, int n, const unsigned* block_offsets) {
  const int i = blockIdx.x * kScanThreads + threadIdx.x;
  if (i < n) data[i] += block_offsets[blockIdx.x];
}

__global__ void order_place_kernel(const unsigned* __restrict__ keys, int num_nodes, int nm, int nf,
                                   unsigned* __restrict__ starts, int* __restrict__ order) {
  const int count = nm + nf;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const unsigned slot = atomicAdd(starts + keys[i], 1u);
    order[slot] = i < nm ? i : num_nodes - nf + (i - nm);
  }
}

// xy_o[idx] = (x, y) of node order[idx], from planar positions [x(n) | y(n)]
__global__ void gather_order_pos_kernel(const float* __restrict__ pos, int num_nodes, const int* __restrict__ order,
                                        int count, float2* __restrict__ xy_o) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    const int i = __ldg(order + idx);
    xy_o[idx] = make_float2(__ldg(pos + i), __ldg(pos + num_nodes + i));
  }
}

static unsigned order_tile_buckets(int nbx, int nby) {
  return (unsigned)(((nbx + 15) >> 4) * ((nby + 15) >> 4)) * 256u;
}

}  // namespace dpb

extern "C" size_t dp_order_cells_scratch_bytes(int num_movable, int num_filler, int num_bins_x, int num_bins_y) {
  using namespace dpb;
  if (num_movable < 0 || num_filler < 0 || num_bins_x <= 0 || num_bins_y <= 0) return 0;
  const size_t buckets = 2ull * order_tile_buckets(num_bins_x, num_bins_y);
  const size_t blocks = (buckets + kScanThreads - 1) / kScanThreads;
  return sizeof(unsigned) * (buckets + blocks + (size_t)num_movable + (size_t)num_filler) + 256;
}

extern "C" int dp_order_cells_by_bin(const float* pos, int num_nodes, const float* offset_x, const float* offset_y,
                                     int num_movable, int num_filler, float xl, float yl, float inv_bin_size_x,
                                     float inv_bin_size_y, int num_bins_x, int num_bins_y, void* scratch,
                                     size_t scratch_bytes, int* order, dp_stream_t stream) {
  using namespace dpb;
  DP_REQUIRE(pos && offset_x && offset_y && scratch && order, "dp_order_cells_by_bin: null pointer argument");
  DP_REQUIRE(num_movable >= 0 && num_filler >= 0 && num_movable + num_filler <= num_nodes,
             "dp_order_cells_by_bin: bad node counts");
  DP_REQUIRE(num_bins_x > 0 && num_bins_y > 0 && num_bins_x <= 65536 && num_bins_y <= 65536,
             "dp_order_cells_by_bin: bad bin grid %dx%d", num_bins_x, num_bins_y);
  const size_t need = dp_order_cells_scratch_bytes(num_movable, num_filler, num_bins_x, num_bins_y);
  DP_REQUIRE(scratch_bytes >= need, "dp_order_cells_by_bin: scratch of %zu bytes, %zu needed", scratch_bytes, need);
  DP_REQUIRE(((uintptr_t)scratch & 3) == 0, "dp_order_cells_by_bin: scratch must be 4-byte aligned");
  const int count = num_movable + num_filler;
  if (count == 0) return DP_OK;
  cudaStream_t s = as_stream(stream);
  const unsigned tile_buckets = order_tile_buckets(num_bins_x, num_bins_y);
  const int buckets = (int)(2u * tile_buckets);
  const int blocks = (buckets + kScanThreads - 1) / kScanThreads;
  unsigned* hist = static_cast<unsigned*>(scratch);
  unsigned* totals = hist + buckets;
  unsigned* keys = totals + blocks;
  cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(unsigned) * buckets, s);
  if (e != cudaSuccess) {
    set_error("dp_order_cells_by_bin: cudaMemsetAsync: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  order_keys_kernel<<<grid_for(count, 256, 8), 256, 0, s>>>(pos, num_nodes, offset_x, offset_y, num_movable,
                                                            num_filler, xl, yl, inv_bin_size_x, inv_bin_size_y,
                                                            num_bins_x, num_bins_y, tile_buckets, keys, hist);
  int rc = check_launch("dp_order_cells_by_bin keys");
  if (rc) return rc;
  scan_blocks_kernel<<<blocks, kScanThreads, 0, s>>>(hist, buckets, totals);
  rc = check_launch("dp_order_cells_by_bin scan");
  if (rc) return rc;
  scan_totals_kernel<<<1, kScanThreads, 0, s>>>(totals, blocks);
  rc = check_launch("dp_order_cells_by_bin scan totals");
  if (rc) return rc;
  add_block_offsets_kernel<<<blocks, kScanThreads, 0, s>>>(hist, buckets, totals);
  rc = check_launch("dp_order_cells_by_bin offsets");
  if (rc) return rc;
  order_place_kernel<<<grid_for(count, 256, 8), 256, 0, s>>>(keys, num_nodes, num_movable, num_filler, hist, order);
  return check_launch("dp_order_cells_by_bin place");
}

extern "C" int dp_gather_order_pos(const float* pos, int num_nodes, const int* order, int count, float* xy_o,
                                   dp_stream_t stream) {
  using namespace dpb;
  DP_REQUIRE(pos && xy_o && (count == 0 || order), "dp_gather_order_pos: null pointer argument");
  DP_REQUIRE(((uintptr_t)xy_o & 7) == 0, "dp_gather_order_pos: xy_o must be 8-byte aligned");
  if (count == 0) return DP_OK;
  gather_order_pos_kernel<<<grid_for(count, 256, 8), 256, 0, as_stream(stream)>>>(
      pos, num_nodes, order, count, reinterpret_cast<float2*>(xy_o));
  return check_launch("dp_gather_order_pos");
}
