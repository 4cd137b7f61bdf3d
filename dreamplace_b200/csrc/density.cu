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
  grid_dep_sync();
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

// ---------------------------------------------------------------- tile scatter
// Cells are visited in the caller's order (a spatial order refreshed every few
// iterations: cells sorted by the bin where their stretched footprint starts,
// see dp_order_cells_by_bin), read from per-cell records (stretched width,
// height, offsets, ratio) and positions stored in the same order, so every
// read of the scatter is contiguous.
//
// One block takes kTsCells consecutive cells of the order.  It reduces their
// bin bounding box (redux.sync per warp, then across the warps) and adds the
// cells into a shared-memory tile over that box; the tile is flushed with one
// global atomic per non-zero bin.  When the box exceeds the tile (cells that
// moved far since the order was refreshed), the tile becomes a window of
// kWinRows x kWinCols bins placed on the block's median cell, and the cells
// outside it add straight to the global map.  A stretched cell is at least
// sqrt(2) bins wide, so a standard cell covers 2 or 3 bins per axis: each
// thread forms a cell's 3 x 3 window (entries beyond the footprint are zero
// and land on a valid slot) and adds all nine, with no branch; cells wider
// than 3 bins take a per-bin loop of global atomics.
//
// The tile accumulates in int32 words, because shared-memory int32 atomics
// are single instructions while fp32 and int64 ones are compare-and-swap
// loops that serialise on contended bins:
//   * deterministic: the contribution's fixed-point value v = trunc(area * 2^f)
//     (the CPU op's `long(area * scale)`) is split exactly with float
//     arithmetic into hi = trunc(v / 2^22) and lo = v - hi * 2^22 (y = area *
//     2^(f-22) is exact; y - trunc(y) is its exact fraction), summed in two
//     planes, and recombined into one int64 at the flush.  512 contributions
//     of |lo| < 2^22 and |hi| < 2^22 stay inside int32, so the map equals the
//     CPU op's int64 sum bit for bit; a contribution with |hi| >= 2^22 (a bin
//     far larger than the die's share) adds its int64 value to the global map
//     directly;
//   * fp32: one plane of round(area * S), S = 2^s with 512 * bin area * S <
//     2^31 (a resolution of at most 2^-21 of the bin area), converted back
//     and added to the fp32 map with one float atomic per bin.
// The fixed-point map is independent of the summation order, so the
// deterministic result does not depend on the visiting order or the tiling.
//
// Contended bins are what limits the tile's atomics: lanes of one warp that
// add to the same word are serialised.  The visiting order therefore places
// the cells of each kTsCells block so that the 32 lanes of a warp hold cells
// kTsCells / 32 apart in sort order (different bins), while the block as a
// whole keeps its compact bin box; and a thread's two cells, adjacent in sort
// order, that start at the same bin add one merged window (fp32 mode).
constexpr int kTsThreads = 256;
constexpr int kTsCellsPerThread = 2;
constexpr int kTsCells = kTsThreads * kTsCellsPerThread;  // 512: the int32 plane bound above
constexpr int kTsTab = 128;                                // longest box side with a bin-edge table
constexpr int kTsSmemBytes = 16 * 1024;
constexpr float kTsLoSpan = 4194304.0f;                    // 2^22

// Cells [b0, b1) of the visiting order, added to map0, and [b1, b2), added to
// map1, in one launch: the first ceil((b1 - b0) / kTsCells) blocks take the
// first range, so the second range's blocks fill the first's last wave.
struct WsRanges {
  int b0, b1, b2;
  float* map0_f32;
  float* map1_f32;
  unsigned long long* map0_fx;
  unsigned long long* map1_fx;
};

template <bool kFixed>
__global__ void __launch_bounds__(kTsThreads) tile_scatter_kernel(TriangleArgs a, WsRanges rg,
                                                                  const float2* __restrict__ xy_o,
                                                                  const int* __restrict__ order,
                                                                  const float4* __restrict__ rec4,
                                                                  const float* __restrict__ ratio_o,
                                                                  float fx_scale, float plane_scale,
                                                                  float plane_unit, const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  constexpr int kPlanes = kFixed ? 2 : 1;
  constexpr int kCap = kTsSmemBytes / (4 * kPlanes);  // tile bins
  constexpr int kWinRows = 32;
  constexpr int kWinCols0 = kCap / kWinRows < kTsTab ? kCap / kWinRows : kTsTab;
  constexpr int kWinCols = (kWinCols0 & 1) ? kWinCols0 : kWinCols0 - 1;  // odd, so kWinRows * kWinCols <= kCap
  const int nb0 = (rg.b1 - rg.b0 + kTsCells - 1) / kTsCells;
  const bool second = (int)blockIdx.x >= nb0;
  const int begin = second ? rg.b1 : rg.b0;
  const int end = second ? rg.b2 : rg.b1;
  float* const map_f32 = second ? rg.map1_f32 : rg.map0_f32;
  unsigned long long* const map_fx = second ? rg.map1_fx : rg.map0_fx;
  const int bid = second ? (int)blockIdx.x - nb0 : (int)blockIdx.x;
  extern __shared__ __align__(16) unsigned char tile_raw[];
  int* const plane0 = reinterpret_cast<int*>(tile_raw);
  __shared__ int red[4][kTsThreads / 32];
  __shared__ int anchor[2];
  __shared__ float2 tabx[kTsTab], taby[kTsTab];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // a thread's cells are adjacent in the order (one 16-byte position load)
  float nx[kTsCellsPerThread], ny[kTsCellsPerThread], sx[kTsCellsPerThread], sy[kTsCellsPerThread],
      rr[kTsCellsPerThread];
  int k0[kTsCellsPerThread], h0[kTsCellsPerThread], nk[kTsCellsPerThread], nh[kTsCellsPerThread];
  int bk0 = INT_MAX, bk1 = INT_MIN, bh0 = INT_MAX, bh1 = INT_MIN;
#pragma unroll
  for (int c = 0; c < kTsCellsPerThread; ++c) {
    const int li = threadIdx.x * kTsCellsPerThread + c;
    const int idx = begin + bid * kTsCells + li;
    nk[c] = nh[c] = k0[c] = h0[c] = 0;
    nx[c] = ny[c] = sx[c] = sy[c] = rr[c] = 0.f;
    if (idx < end) {
      const float4 r4 = __ldg(rec4 + idx);
      // positions in visiting order, or in node order read through the order
      const float2 p = order ? __ldg(xy_o + __ldg(order + idx)) : __ldg(xy_o + idx);
      sx[c] = r4.x;
      sy[c] = r4.y;
      nx[c] = fadd(p.x, r4.z);
      ny[c] = fadd(p.y, r4.w);
      rr[c] = __ldg(ratio_o + idx);
      int ka, kb, ha, hb;
      triangle_bin_range(nx[c], sx[c], a.xl, a.inv_bsx, a.num_bins_x, ka, kb);
      triangle_bin_range(ny[c], sy[c], a.yl, a.inv_bsy, a.num_bins_y, ha, hb);
      if (kb > ka && hb > ha) {
        k0[c] = ka;
        h0[c] = ha;
        nk[c] = kb - ka;
        nh[c] = hb - ha;
        bk0 = min(bk0, ka);
        bk1 = max(bk1, kb);
        bh0 = min(bh0, ha);
        bh1 = max(bh1, hb);
      }
    }
    // the window anchor: slot 32 holds the block's median cell in the
    // block-spread order (any cell otherwise)
    if (li == 32) {
      anchor[0] = nk[c] ? k0[c] : INT_MIN;
      anchor[1] = h0[c];
    }
  }
  bk0 = __reduce_min_sync(0xffffffffu, bk0);
  bk1 = __reduce_max_sync(0xffffffffu, bk1);
  bh0 = __reduce_min_sync(0xffffffffu, bh0);
  bh1 = __reduce_max_sync(0xffffffffu, bh1);
  if (lane == 0) {
    red[0][warp] = bk0;
    red[1][warp] = bk1;
    red[2][warp] = bh0;
    red[3][warp] = bh1;
  }
  __syncthreads();
  {
    const bool w = lane < kTsThreads / 32;
    bk0 = __reduce_min_sync(0xffffffffu, w ? red[0][lane] : INT_MAX);
    bk1 = __reduce_max_sync(0xffffffffu, w ? red[1][lane] : INT_MIN);
    bh0 = __reduce_min_sync(0xffffffffu, w ? red[2][lane] : INT_MAX);
    bh1 = __reduce_max_sync(0xffffffffu, w ? red[3][lane] : INT_MIN);
  }
  if (bk1 <= bk0) return;  // nothing to scatter (uniform across the block)
  if ((long long)(bk1 - bk0) * ((bh1 - bh0) | 1) > kCap || bk1 - bk0 > kTsTab || bh1 - bh0 > kTsTab) {
    int km = anchor[0], hm = anchor[1];
    if (km == INT_MIN) {
      km = bk0;
      hm = bh0;
    }
    const int wk0 = max(bk0, min(km - kWinRows / 2, bk1 - kWinRows));
    const int wh0 = max(bh0, min(hm - kWinCols / 2, bh1 - kWinCols));
    bk1 = min(bk1, wk0 + kWinRows);
    bh1 = min(bh1, wh0 + kWinCols);
    bk0 = wk0;
    bh0 = wh0;
  }
  const int K = bk1 - bk0, H = bh1 - bh0;
  const int P = H | 1;  // odd row pitch: the bins of a tile column fall in different banks
  const int box = K * P;
  for (int t = threadIdx.x; t < kPlanes * box; t += kTsThreads) plane0[t] = 0;
  // bin edges of the box, in the reference's arithmetic (bin_xl = xl + k * bs)
  for (int t = threadIdx.x; t < K + H; t += kTsThreads) {
    if (t < K) {
      const float lo = fadd(a.xl, fmul((float)(bk0 + t), a.bsx));
      tabx[t] = make_float2(lo, fadd(lo, a.bsx));
    } else {
      const float lo = fadd(a.yl, fmul((float)(bh0 + t - K), a.bsy));
      taby[t - K] = make_float2(lo, fadd(lo, a.bsy));
    }
  }
  __syncthreads();
  int* const plane1 = plane0 + box;
  const int nby = a.num_bins_y;
  if (kFixed) {
#pragma unroll
  for (int c = 0; c < kTsCellsPerThread; ++c) {
    if (nk[c] == 0) continue;
    const int rk = k0[c] - bk0, rh = h0[c] - bh0;
    if (rk >= 0 && rh >= 0 && rk + nk[c] <= K && rh + nh[c] <= H && nk[c] <= 3 && nh[c] <= 3) {
      const float xh = fadd(nx[c], sx[c]), yh = fadd(ny[c], sy[c]);
      float pxr[3], py[3];
      int row[3], col[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const bool okx = j < nk[c], oky = j < nh[c];
        const float2 ex = tabx[okx ? rk + j : rk];
        const float2 ey = taby[oky ? rh + j : rh];
        // triangle_overlap: min(x + size, bin_xh) - max(x, bin_xl)
        pxr[j] = okx ? fmul(fsub(fminf(xh, ex.y), fmaxf(nx[c], ex.x)), rr[c]) : 0.f;
        py[j] = oky ? fsub(fminf(yh, ey.y), fmaxf(ny[c], ey.x)) : 0.f;
        row[j] = (okx ? rk + j : rk) * P + rh;
        col[j] = oky ? j : 0;
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float area = fmul(pxr[i], py[j]);
          const int slot = row[i] + col[j];
          const float y = fmul(area, plane_scale);
          const float hf = truncf(y);
          if (fabsf(hf) < kTsLoSpan) {
            atomicAdd(plane0 + slot, (int)hf);
            atomicAdd(plane1 + slot, (int)fmul(fsub(y, hf), kTsLoSpan));
          } else {
            atomicAdd(map_fx + (bk0 + rk + i) * nby + bh0 + rh + j, (unsigned long long)to_fixed(area, fx_scale));
          }
        }
    } else {
      // outside the tile, or wider than 3 bins: one global add per bin
      for (int k = k0[c]; k < k0[c] + nk[c]; ++k) {
        const float pxr = fmul(triangle_overlap(nx[c], sx[c], a.xl, k, a.bsx), rr[c]);
        for (int h = h0[c]; h < h0[c] + nh[c]; ++h) {
          const float area = fmul(pxr, triangle_overlap(ny[c], sy[c], a.yl, h, a.bsy));
          atomicAdd(map_fx + k * nby + h, (unsigned long long)to_fixed(area, fx_scale));
        }
      }
    }
  }
  } else {
    // fp32: each cell's nine rounded contributions are formed first; a
    // thread's two cells (adjacent in sort order) that start at the same bin
    // add one merged window, halving the atomics where cells crowd
    int vals[kTsCellsPerThread][9];
    bool ok[kTsCellsPerThread];
#pragma unroll
    for (int c = 0; c < kTsCellsPerThread; ++c) {
      const int rk = k0[c] - bk0, rh = h0[c] - bh0;
      ok[c] = nk[c] && rk >= 0 && rh >= 0 && rk + nk[c] <= K && rh + nh[c] <= H && nk[c] <= 3 && nh[c] <= 3;
      const float xh = fadd(nx[c], sx[c]), yh = fadd(ny[c], sy[c]);
      float pxr[3], py[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const bool okx = j < nk[c], oky = j < nh[c];
        // (table indices clamped into the tables: a cell outside the tile
        // computes values it does not use)
        const float2 ex = tabx[min(max(okx ? rk + j : rk, 0), kTsTab - 1)];
        const float2 ey = taby[min(max(oky ? rh + j : rh, 0), kTsTab - 1)];
        // triangle_overlap: min(x + size, bin_xh) - max(x, bin_xl)
        pxr[j] = okx ? fmul(fsub(fminf(xh, ex.y), fmaxf(nx[c], ex.x)), rr[c]) : 0.f;
        py[j] = oky ? fsub(fminf(yh, ey.y), fmaxf(ny[c], ey.x)) : 0.f;
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float y = fmul(fmul(pxr[i], py[j]), plane_scale);
          ok[c] = ok[c] && fabsf(y) < kTsLoSpan - 1.0f;  // |round(y)| < 2^22
          vals[c][3 * i + j] = __float2int_rn(y);
        }
    }
    // same start bin: cell 0 takes the merged window (the larger extents;
    // each cell's entries beyond its footprint are zero) and cell 1 adds none
    bool add1 = ok[1];
    int mk = nk[0], mh = nh[0];
    if (ok[0] && ok[1] && k0[0] == k0[1] && h0[0] == h0[1]) {
      add1 = false;
      mk = max(nk[0], nk[1]);
      mh = max(nh[0], nh[1]);
#pragma unroll
      for (int t = 0; t < 9; ++t) vals[0][t] += vals[1][t];
    }
    // one predicated pass per cell: a warp whose lanes all merged skips the second
#pragma unroll
    for (int c = 0; c < kTsCellsPerThread; ++c) {
      const bool add = c == 0 ? ok[0] : add1;
      if (!__any_sync(0xffffffffu, add)) continue;
      const int ek = c == 0 ? mk : nk[1], eh = c == 0 ? mh : nh[1];
      const int rk = k0[c] - bk0, rh = h0[c] - bh0;
      int row[3], col[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        row[j] = (j < ek ? rk + j : rk) * P + rh;
        col[j] = j < eh ? j : 0;
      }
      if (add) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) atomicAdd(plane0 + row[i] + col[j], vals[c][3 * i + j]);
      }
    }
    // outside the tile, wider than 3 bins, or beyond the plane's range: one
    // global add per bin
#pragma unroll
    for (int c = 0; c < kTsCellsPerThread; ++c) {
      if (nk[c] == 0 || ok[c]) continue;
      for (int k = k0[c]; k < k0[c] + nk[c]; ++k) {
        const float pxr = fmul(triangle_overlap(nx[c], sx[c], a.xl, k, a.bsx), rr[c]);
        for (int h = h0[c]; h < h0[c] + nh[c]; ++h)
          atomicAdd(map_f32 + k * nby + h, fmul(pxr, triangle_overlap(ny[c], sy[c], a.yl, h, a.bsy)));
      }
    }
  }
  __syncthreads();
  // flush: tile slot t is row t / P, column t % P (stepped without division
  // after the first; the pad column holds zeros)
  const float inv_p = __frcp_rn((float)P);
  int k = (int)((float)threadIdx.x * inv_p), h = (int)threadIdx.x - k * P;
  if (h < 0) { --k; h += P; } else if (h >= P) { ++k; h -= P; }
  int dk = (int)((float)kTsThreads * inv_p), dh = kTsThreads - dk * P;
  if (dh < 0) { --dk; dh += P; } else if (dh >= P) { ++dk; dh -= P; }
  for (int t = threadIdx.x; t < box; t += kTsThreads) {
    const int g = (bk0 + k) * nby + bh0 + h;
    if (kFixed) {
      const int hi = plane0[t], lo = plane1[t];
      if ((hi | lo) != 0)
        atomicAdd(map_fx + g, (unsigned long long)(((long long)hi << 22) + (long long)lo));
    } else {
      const int v = plane0[t];
      if (v != 0) atomicAdd(map_f32 + g, (float)v * plane_unit);
    }
    k += dk;
    h += dh;
    if (h >= P) {
      h -= P;
      ++k;
    }
  }
}

__global__ void gather_order_xy_kernel(const float2* __restrict__ xy, const int* __restrict__ order, int count,
                                       float2* __restrict__ xy_o, const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  // four independent gathers in flight per thread: the random 8-byte reads
  // are latency-bound, not bandwidth-bound
  const int stride = gridDim.x * blockDim.x;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  for (; (long long)idx + 3ll * stride < count; idx += 4 * stride) {
    int o[4];
    float2 q[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) o[u] = order[idx + u * stride];
#pragma unroll
    for (int u = 0; u < 4; ++u) q[u] = xy[o[u]];
#pragma unroll
    for (int u = 0; u < 4; ++u) xy_o[idx + u * stride] = q[u];
  }
  for (; idx < count; idx += stride) xy_o[idx] = xy[order[idx]];
}

__global__ void build_records_kernel(const float* __restrict__ sx, const float* __restrict__ sy,
                                     const float* __restrict__ ox, const float* __restrict__ oy,
                                     const float* __restrict__ ratio, const int* __restrict__ order, int count,
                                     float4* __restrict__ rec4, float* __restrict__ ratio_o,
                                     int* __restrict__ inv_order) {
  grid_dep_sync();
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
  grid_dep_sync();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double base = init ? (double)init[i] : 0.0;
    out[i] = (float)(base + (double)fixed[i] * inv_scale);
  }
}

__global__ void copy_kernel(const float4* __restrict__ src, float4* __restrict__ dst, int n4,
                            const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x)
    dst[i] = src[i];
}

static int copy_map(const float* src, float* dst, int n, cudaStream_t s) {
  if (src == dst) return DP_OK;
  if ((n & 3) == 0 && ((uintptr_t)src & 15) == 0 && ((uintptr_t)dst & 15) == 0) {
    launch_kernel(copy_kernel, grid_for(n / 4, 256), 256, 0, s, (const float4*)src, (float4*)dst, n / 4, trial_gate());
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
  grid_dep_sync();
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
  grid_dep_sync();
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
  grid_dep_sync();
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
  grid_dep_sync();
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
  grid_dep_sync();
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

// fp32 split scatter, second pass: first = init + first (the movable cells
// were scattered onto a zeroed map), all += first (all held the fillers), and
// the overflow sum and maximum of first as overflow_kernel does.  float4
// accesses when the three maps are 16-byte aligned.
__device__ __forceinline__ void finish_map_bin(float f, float in, float& first_out, float& all_io, double target_area,
                                               double& s, float& m) {
  const float d = fadd(in, f);
  first_out = d;
  all_io = fadd(d, all_io);
  const double over = (double)d - target_area;
  s += over > 0.0 ? over : 0.0;
  m = fmaxf(m, d);
}

__global__ void finish_maps_kernel(const float* __restrict__ init, float* __restrict__ first, float* __restrict__ all,
                                   int n, double target_area, double* partials, unsigned* maxkey,
                                   const int* __restrict__ gate) {
  grid_dep_sync();
  if (gate_closed(gate)) return;
  double s = 0.0;
  float m = -INFINITY;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  const bool vec = (((uintptr_t)first | (uintptr_t)all | (uintptr_t)init) & 15) == 0;
  int done = 0;
  if (vec) {
    const int n4 = n >> 2;
    for (int i = tid; i < n4; i += stride) {
      const float4 f = reinterpret_cast<const float4*>(first)[i];
      const float4 in = init ? reinterpret_cast<const float4*>(init)[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      float4 a = reinterpret_cast<const float4*>(all)[i];
      float4 o;
      finish_map_bin(f.x, in.x, o.x, a.x, target_area, s, m);
      finish_map_bin(f.y, in.y, o.y, a.y, target_area, s, m);
      finish_map_bin(f.z, in.z, o.z, a.z, target_area, s, m);
      finish_map_bin(f.w, in.w, o.w, a.w, target_area, s, m);
      reinterpret_cast<float4*>(first)[i] = o;
      reinterpret_cast<float4*>(all)[i] = a;
    }
    done = n4 << 2;
  }
  for (int i = done + tid; i < n; i += stride) {
    float o, a = all[i];
    finish_map_bin(first[i], init ? init[i] : 0.f, o, a, target_area, s, m);
    first[i] = o;
    all[i] = a;
  }
  if (!partials) return;  // uniform: no overflow wanted
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxkey, float_key(m));
  block_partial(s, partials);
}

__global__ void overflow_finish_kernel(double* out2, const unsigned* maxkey, double bin_area,
                                       float* out2_f32, const double* partials, int count) {
  grid_dep_sync();
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
  launch_kernel(triangle_scatter_kernel<false>, grid_for(total, 256, 16), 256, 0, s, a, total, 0.f, out, nullptr);
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
    launch_kernel(triangle_scatter_kernel<true>, grid_for(total, 256, 16), 256, 0, s, 
        a, total, scale, nullptr, reinterpret_cast<unsigned long long*>(scratch));
    rc = check_launch("dp_density_map_fx64 scatter");
    if (rc) return rc;
  }
  launch_kernel(fixed_to_float_kernel, grid_for(nbins, 256), 256, 0, s, (const long long*)scratch, init,
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
    launch_kernel(exact_scatter_kernel<true>, blocks, 128, 0, s, x, y, sx, sy, bcx, bcy, nm, nm + nt, xl, yl, xh, yh,
                                                      bsx, bsy, nbx, nby, true, true,
                                                      ldexpf(1.0f, fraction_bits), nullptr,
                                                      reinterpret_cast<unsigned long long*>(scratch));
    int rc = check_launch("dp_fixed_density_map scatter");
    if (rc) return rc;
    launch_kernel(fixed_to_float_kernel, grid_for(nbins, 256), 256, 0, s, (const long long*)scratch, nullptr,
                                                              ldexp(1.0, -fraction_bits), out, nbins);
    rc = check_launch("dp_fixed_density_map convert");
    if (rc) return rc;
  } else {
    launch_kernel(exact_scatter_kernel<false>, blocks, 128, 0, s, x, y, sx, sy, bcx, bcy, nm, nm + nt, xl, yl, xh, yh,
                                                       bsx, bsy, nbx, nby, true, true, 0.f, out, nullptr);
    int rc = check_launch("dp_fixed_density_map scatter");
    if (rc) return rc;
  }
  float vmax = (float)((double)bsx * (double)bsy);
  launch_kernel(clamp_max_kernel, grid_for(nbins, 256), 256, 0, s, out, nbins, vmax);
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
      launch_kernel(box_scatter_kernel<true>, grid_for(n, 128, 8), 128, 0, s, 
          x, y, sx, sy, rb[r], re[r], xl, yl, xh, yh, nbx, nby, ldexpf(1.0f, fraction_bits), nullptr,
          reinterpret_cast<unsigned long long*>(scratch));
      int rc = check_launch("dp_density_map_exact scatter");
      if (rc) return rc;
      launch_kernel(fixed_to_float_kernel, grid_for(nbins, 256), 256, 0, s, (const long long*)scratch, out,
                                                                ldexp(1.0, -fraction_bits), out, nbins);
      rc = check_launch("dp_density_map_exact convert");
      if (rc) return rc;
    } else {
      launch_kernel(box_scatter_kernel<false>, grid_for(n, 128, 8), 128, 0, s, x, y, sx, sy, rb[r], re[r], xl, yl, xh, yh,
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
  launch_kernel(overflow_kernel, blocks, 256, 0, s, map, nbins, target_area, out2 + 3, maxslot);
  int rc = check_launch("dp_density_overflow");
  if (rc) return rc;
  launch_kernel(overflow_finish_kernel, 1, kReduceThreads, 0, s, out2, maxslot, bin_area, out2_f32, out2 + 3, blocks);
  return check_launch("dp_density_overflow finish");
}

// xy_o[idx] = xy[order[idx]]: positions in visiting order
extern "C" int dp_gather_order_xy(const float* xy, const int* order, int count, float* xy_o, dp_stream_t stream) {
  DP_REQUIRE(xy && xy_o && (count == 0 || order), "dp_gather_order_xy: null pointer");
  DP_REQUIRE(((uintptr_t)xy & 7) == 0 && ((uintptr_t)xy_o & 7) == 0, "dp_gather_order_xy: misaligned xy / xy_o");
  if (count == 0) return DP_OK;
  launch_kernel(gather_order_xy_kernel, grid_for(count, 256, 8), 256, 0, as_stream(stream), 
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
  launch_kernel(build_records_kernel, grid_for(count, 256, 8), 256, 0, as_stream(stream), 
      sx, sy, ox, oy, ratio, order, count, reinterpret_cast<float4*>(rec4), ratio_o, inv_order);
  return check_launch("dp_build_cell_records");
}

// Order-driven scatter (see tile_scatter_kernel): the cells order[0..count)
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
int scatter_ranges(const OrderedScatter& o, const WsRanges& rg, int deterministic, int fraction_bits) {
  int rc = deterministic ? opt_in_smem(tile_scatter_kernel<true>, kTsSmemBytes, "density scatter")
                         : opt_in_smem(tile_scatter_kernel<false>, kTsSmemBytes, "density scatter");
  if (rc) return rc;
  const int blocks = ceil_div(rg.b1 - rg.b0, kTsCells) + ceil_div(rg.b2 - rg.b1, kTsCells);
  if (blocks <= 0) return DP_OK;
  if (deterministic) {
    // plane scale 2^(f - 22): hi = trunc(v / 2^22) of v = trunc(area * 2^f)
    const float fx_scale = ldexpf(1.0f, fraction_bits);
    launch_kernel(tile_scatter_kernel<true>, blocks, kTsThreads, kTsSmemBytes, o.s, 
        o.a, rg, o.xy_o, o.order, o.rec4, o.ratio_o, fx_scale, ldexpf(1.0f, fraction_bits - 22), 0.f,
        trial_gate());
  } else {
    // S = 2^s with (bin area) * S < 2^22 - 1: a block's 512 contributions of
    // at most one bin area each sum below 2^31
    const double bin_area = (double)o.a.bsx * (double)o.a.bsy;
    const int s = (int)floor(log2((4194302.0 / 1.0001) / bin_area));
    launch_kernel(tile_scatter_kernel<false>, blocks, kTsThreads, kTsSmemBytes, o.s, 
        o.a, rg, o.xy_o, o.order, o.rec4, o.ratio_o, 0.f, ldexpf(1.0f, s), ldexpf(1.0f, -s), trial_gate());
  }
  return check_launch("dp_density_map_ordered scatter");
}

// adds cells [begin, end) of the visiting order onto out (fp32) or scratch (fixed)
int scatter_range(const OrderedScatter& o, int begin, int end, int deterministic, int fraction_bits, int64_t* scratch,
                  float* out) {
  if (end <= begin) return DP_OK;
  WsRanges rg;
  memset(&rg, 0, sizeof(rg));
  rg.b0 = begin;
  rg.b1 = rg.b2 = end;
  rg.map0_f32 = out;
  rg.map0_fx = reinterpret_cast<unsigned long long*>(scratch);
  return scatter_ranges(o, rg, deterministic, fraction_bits);
}

int convert_fixed(const int64_t* scratch, const float* init, int fraction_bits, float* out, int nbins,
                  cudaStream_t s) {
  launch_kernel(fixed_to_float_kernel, grid_for(nbins, 256), 256, 0, s, (const long long*)scratch, init,
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

// Order-driven scatter (see tile_scatter_kernel): cells 0..count of the
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
      launch_kernel(first_map_kernel, blocks, 256, 0, o.s, (const long long*)scratch, init, ldexp(1.0, -fraction_bits),
                                                 out_first, nullptr, 0, nbins, target_area, overflow_out + 3, maxslot,
                                                 trial_gate());
      rc = check_launch("dp_density_map_ordered_split first map");
      if (rc) return rc;
      launch_kernel(overflow_finish_kernel, 1, kReduceThreads, 0, o.s, overflow_out, maxslot, bin_area, nullptr,
                                                            overflow_out + 3, blocks);
      rc = check_launch("dp_density_map_ordered_split overflow");
    } else {
      rc = convert_fixed(scratch, init, fraction_bits, out_first, nbins, o.s);
    }
    if (rc) return rc;
    rc = scatter_range(o, num_first, count, 1, fraction_bits, scratch, nullptr);
    if (rc) return rc;
    return convert_fixed(scratch, init, fraction_bits, out_all, nbins, o.s);
  }
  // fp32: both ranges in one launch (the second range's blocks fill the
  // first's last wave), the first onto out_first = 0, the second onto
  // out_all = 0; then out_first += init and out_all += out_first, with the
  // overflow of out_first
  cudaError_t e = cudaMemsetAsync(out_first, 0, sizeof(float) * nbins, o.s);
  if (e == cudaSuccess) e = cudaMemsetAsync(out_all, 0, sizeof(float) * nbins, o.s);
  if (e != cudaSuccess) {
    set_error("dp_density_map_ordered_split: cudaMemsetAsync: %s", cudaGetErrorString(e));
    return DP_ERR_CUDA;
  }
  WsRanges rg;
  memset(&rg, 0, sizeof(rg));
  rg.b0 = 0;
  rg.b1 = num_first;
  rg.b2 = count;
  rg.map0_f32 = out_first;
  rg.map1_f32 = out_all;
  rc = scatter_ranges(o, rg, 0, 0);
  if (rc) return rc;
  if (overflow_out) cudaMemsetAsync(maxslot, 0, sizeof(double), o.s);
  launch_kernel(finish_maps_kernel, blocks, 256, 0, o.s, init, out_first, out_all, nbins, target_area,
                                             overflow_out ? overflow_out + 3 : nullptr, maxslot, trial_gate());
  rc = check_launch("dp_density_map_ordered_split first map");
  if (rc || !overflow_out) return rc;
  launch_kernel(overflow_finish_kernel, 1, kReduceThreads, 0, o.s, overflow_out, maxslot, bin_area, nullptr,
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
// scatter and the field gather).  The sorted ranks are then placed block by
// block for the tile scatter (block_spread_slot).
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
  grid_dep_sync();
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
    // one atomic per distinct bucket of the warp (clustered cells share a few
    // buckets early in GP)
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(hist + key, (unsigned)__popc(peers));
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
  grid_dep_sync();
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
  grid_dep_sync();
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
  grid_dep_sync();
  const int i = blockIdx.x * kScanThreads + threadIdx.x;
  if (i < n) data[i] += block_offsets[blockIdx.x];
}

// Position of sorted rank `slot` of the range [b, e) (the movable cells or
// the fillers): inside each full block of kTsCells cells (the tile scatter's
// block), rank r goes to the slot read by lane r / (kTsCells / 32) of warp
// (r % (kTsCells / 32)) / kTsCellsPerThread, so the 32 lanes of a warp hold
// cells kTsCells / 32 apart in sort order while the block keeps its cells.
// A partial last block keeps the sorted order.
__device__ __forceinline__ int block_spread_slot(int slot, int b, int e) {
  constexpr int kStride = kTsCells / 32;
  const int q = slot - b;
  const int j = q / kTsCells;
  if ((j + 1) * kTsCells > e - b) return slot;
  const int r = q - j * kTsCells;
  const int lane = r / kStride, rem = r - lane * kStride;
  const int warp = rem / kTsCellsPerThread, c = rem - warp * kTsCellsPerThread;
  return b + j * kTsCells + (warp * 32 + lane) * kTsCellsPerThread + c;
}

__global__ void order_place_kernel(const unsigned* __restrict__ keys, int num_nodes, int nm, int nf,
                                   unsigned* __restrict__ starts, int* __restrict__ order) {
  grid_dep_sync();
  const int count = nm + nf;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    // warp-aggregated bucket slots: the leader of each group of lanes with one
    // key takes them all, each lane its rank among the group
    const unsigned key = keys[i];
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    const int lane = (int)(threadIdx.x & 31), leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(starts + key, (unsigned)__popc(peers));
    base = __shfl_sync(active, base, leader);
    const int slot = (int)(base + (unsigned)__popc(peers & ((1u << lane) - 1u)));
    if (i < nm)
      order[block_spread_slot(slot, 0, nm)] = i;
    else
      order[block_spread_slot(slot, nm, count)] = num_nodes - nf + (i - nm);
  }
}

// xy_o[idx] = (x, y) of node order[idx], from planar positions [x(n) | y(n)]
__global__ void gather_order_pos_kernel(const float* __restrict__ pos, int num_nodes, const int* __restrict__ order,
                                        int count, float2* __restrict__ xy_o) {
  grid_dep_sync();
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
  launch_kernel(order_keys_kernel, grid_for(count, 256, 8), 256, 0, s, pos, num_nodes, offset_x, offset_y, num_movable,
                                                            num_filler, xl, yl, inv_bin_size_x, inv_bin_size_y,
                                                            num_bins_x, num_bins_y, tile_buckets, keys, hist);
  int rc = check_launch("dp_order_cells_by_bin keys");
  if (rc) return rc;
  launch_kernel(scan_blocks_kernel, blocks, kScanThreads, 0, s, hist, buckets, totals);
  rc = check_launch("dp_order_cells_by_bin scan");
  if (rc) return rc;
  launch_kernel(scan_totals_kernel, 1, kScanThreads, 0, s, totals, blocks);
  rc = check_launch("dp_order_cells_by_bin scan totals");
  if (rc) return rc;
  launch_kernel(add_block_offsets_kernel, blocks, kScanThreads, 0, s, hist, buckets, totals);
  rc = check_launch("dp_order_cells_by_bin offsets");
  if (rc) return rc;
  launch_kernel(order_place_kernel, grid_for(count, 256, 8), 256, 0, s, keys, num_nodes, num_movable, num_filler, hist, order);
  return check_launch("dp_order_cells_by_bin place");
}

extern "C" int dp_gather_order_pos(const float* pos, int num_nodes, const int* order, int count, float* xy_o,
                                   dp_stream_t stream) {
  using namespace dpb;
  DP_REQUIRE(pos && xy_o && (count == 0 || order), "dp_gather_order_pos: null pointer argument");
  DP_REQUIRE(((uintptr_t)xy_o & 7) == 0, "dp_gather_order_pos: xy_o must be 8-byte aligned");
  if (count == 0) return DP_OK;
  launch_kernel(gather_order_pos_kernel, grid_for(count, 256, 8), 256, 0, as_stream(stream), 
      pos, num_nodes, order, count, reinterpret_cast<float2*>(xy_o));
  return check_launch("dp_gather_order_pos");
}
