/*
 * CPU oracle for the dreamplace_b200 hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the reference DREAMPlace CPU
 * algorithms, used by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  Nothing in the dreamplace_b200 package
 * links or calls it.  Float arithmetic follows the reference operation order
 * (compile with -ffp-contract=off so no FMA is formed), which makes the
 * fixed-point density map and the electric force bit-comparable.
 *
 * Pinned against the reference's own CPU ops (oracle/_ref, built from the
 * reference sources by oracle/build_ref.py) through tests/golden fixtures.
 * Paths below are relative to the reference's dreamplace/ops/.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline float fminf_(float a, float b) { return (b < a) ? b : a; } /* std::min */
static inline float fmaxf_(float a, float b) { return (a < b) ? b : a; } /* std::max */

/* electric_potential/src/density_function.h:12-17 */
static inline float triangle_density_function(float x, float node_size, float xl, int k, float bin_size) {
  float bin_xl = xl + (float)k * bin_size;
  return fminf_(x + node_size, bin_xl + bin_size) - fmaxf_(x, bin_xl);
}

/* electric_potential/src/density_function.h:19-36 */
static inline float exact_density_function(float x, float node_size, float bin_center, float bin_size, float l,
                                           float h, int flag) {
  float bin_xl = bin_center - bin_size / 2;
  float bin_xh = bin_center + bin_size / 2;
  if (!flag) {
    if (bin_xl <= l) bin_xl = fminf_(bin_xl, x);
    if (bin_xh >= h) bin_xh = fmaxf_(bin_xh, x + node_size);
  }
  return fmaxf_(0.0f, fminf_(x + node_size, bin_xh) - fmaxf_(x, bin_xl));
}

/* fraction bits of the deterministic mode:
 * electric_potential/src/electric_density_map.cpp:117-121 */
int oracle_fraction_bits(double xl, double yl, double xh, double yh) {
  double diearea = (xh - xl) * (yh - yl);
  int ib = (int)ceil(log2(diearea)) + 1;
  if (ib < 32) ib = 32;
  int fb = 64 - ib;
  return fb < 0 ? 0 : fb;
}

/* Triangle scatter of nodes [begin, end):
 * electric_potential/src/electric_density_map.cpp:216-268.
 * map_f32 != NULL: float accumulation; else map_fx (int64, scale 2^fb). */
void oracle_triangle_scatter(const float* x, const float* y, const float* sx, const float* sy, const float* ox,
                             const float* oy, const float* ratio, int begin, int end, int nbx, int nby,
                             double xl_d, double yl_d, double bsx_d, double bsy_d, float* map_f32,
                             int64_t* map_fx, int fraction_bits) {
  float xl = (float)xl_d, yl = (float)yl_d, bsx = (float)bsx_d, bsy = (float)bsy_d;
  float ibx = (float)(1.0 / (double)bsx);
  float iby = (float)(1.0 / (double)bsy);
  float scale = (float)((int64_t)1 << fraction_bits);
  for (int i = begin; i < end; ++i) {
    float nsx = sx[i], nsy = sy[i];
    float nx = x[i] + ox[i];
    float ny = y[i] + oy[i];
    float r = ratio[i];
    int kl = (int)((nx - xl) * ibx);
    int kh = (int)(((nx + nsx - xl) * ibx)) + 1;
    if (kl < 0) kl = 0;
    if (kh > nbx) kh = nbx;
    int hl = (int)((ny - yl) * iby);
    int hh = (int)(((ny + nsy - yl) * iby)) + 1;
    if (hl < 0) hl = 0;
    if (hh > nby) hh = nby;
    for (int k = kl; k < kh; ++k) {
      float px = triangle_density_function(nx, nsx, xl, k, bsx);
      float pxr = px * r;
      for (int h = hl; h < hh; ++h) {
        float py = triangle_density_function(ny, nsy, yl, h, bsy);
        float area = pxr * py;
        if (map_f32)
          map_f32[k * nby + h] += area;
        else
          map_fx[k * nby + h] += (int64_t)(area * scale);
      }
    }
  }
}

/* dst[i] = (float)((double)dst[i] + (double)src[i] * 2^-fb):
 * utility/src/atomic_ops.h:48-54 with scale 1.0 / scale_factor */
void oracle_fixed_to_float(const int64_t* src, float* dst, int n, int fraction_bits) {
  double inv = 1.0 / (double)((int64_t)1 << fraction_bits);
  for (int i = 0; i < n; ++i) dst[i] = (float)((double)dst[i] + (double)src[i] * inv);
}

/* Exact overlap of fixed nodes [begin, end) with fixed_node_flag = true:
 * electric_potential/src/electric_density_map.cpp:270-309 */
void oracle_exact_scatter(const float* x, const float* y, const float* sx, const float* sy, const float* bcx,
                          const float* bcy, int begin, int end, int nbx, int nby, double xl_d, double yl_d,
                          double xh_d, double yh_d, double bsx_d, double bsy_d, float* map_f32, int64_t* map_fx,
                          int fraction_bits) {
  float xl = (float)xl_d, yl = (float)yl_d, xh = (float)xh_d, yh = (float)yh_d;
  float bsx = (float)bsx_d, bsy = (float)bsy_d;
  float scale = (float)((int64_t)1 << fraction_bits);
  for (int i = begin; i < end; ++i) {
    float bxl = x[i], byl = y[i];
    float bxh = bxl + sx[i], byh = byl + sy[i];
    int kl = (int)((bxl - xl) / bsx);
    int kh = (int)ceilf((bxh - xl) / bsx) + 1;
    if (kl < 0) kl = 0;
    if (kh > nbx) kh = nbx;
    int hl = (int)((byl - yl) / bsy);
    int hh = (int)ceilf((byh - yl) / bsy) + 1;
    if (hl < 0) hl = 0;
    if (hh > nby) hh = nby;
    for (int k = kl; k < kh; ++k) {
      float px = exact_density_function(bxl, bxh - bxl, bcx[k], bsx, xl, xh, 1);
      for (int h = hl; h < hh; ++h) {
        float py = exact_density_function(byl, byh - byl, bcy[h], bsy, yl, yh, 1);
        float area = px * py;
        if (map_f32)
          map_f32[k * nby + h] += area;
        else
          map_fx[k * nby + h] += (int64_t)(area * scale);
      }
    }
  }
}

/* Electric force of nodes [begin, end) (without the grad_pos factor):
 * electric_potential/src/electric_force.cpp:114-166 */
void oracle_electric_force(const float* ex, const float* ey, const float* x, const float* y, const float* sx,
                           const float* sy, const float* ox, const float* oy, const float* ratio, int begin, int end,
                           int nbx, int nby, double xl_d, double yl_d, double bsx_d, double bsy_d, float* gx,
                           float* gy) {
  float xl = (float)xl_d, yl = (float)yl_d, bsx = (float)bsx_d, bsy = (float)bsy_d;
  float ibx = (float)(1.0 / (double)bsx);
  float iby = (float)(1.0 / (double)bsy);
  for (int i = begin; i < end; ++i) {
    float nsx = sx[i], nsy = sy[i];
    float nx = x[i] + ox[i];
    float ny = y[i] + oy[i];
    float r = ratio[i];
    int kl = (int)((nx - xl) * ibx);
    int kh = (int)(((nx + nsx - xl) * ibx)) + 1;
    if (kl < 0) kl = 0;
    if (kh > nbx) kh = nbx;
    int hl = (int)((ny - yl) * iby);
    int hh = (int)(((ny + nsy - yl) * iby)) + 1;
    if (hl < 0) hl = 0;
    if (hh > nby) hh = nby;
    float ax = 0.0f, ay = 0.0f;
    for (int k = kl; k < kh; ++k) {
      float px = triangle_density_function(nx, nsx, xl, k, bsx);
      for (int h = hl; h < hh; ++h) {
        float py = triangle_density_function(ny, nsy, yl, h, bsy);
        float area = px * py;
        int idx = k * nby + h;
        ax += area * ex[idx];
        ay += area * ey[idx];
      }
    }
    gx[i] = ax * r;
    gy[i] = ay * r;
  }
}

/* WA merged forward for one net range:
 * weighted_average_wirelength/src/weighted_average_wirelength_merged.cpp:31-128.
 * partial_wl[i] (unweighted), grad_x/grad_y at the pin ids. exp in double,
 * rounded to float. */
void oracle_wa_merged(const float* x, const float* y, const int* flat_netpin, const int* netpin_start,
                      const unsigned char* net_mask, int num_nets, float inv_gamma, float* partial_wl,
                      float* grad_x, float* grad_y) {
  for (int i = 0; i < num_nets; ++i) {
    partial_wl[i] = 0.0f;
    if (!net_mask[i]) continue;
    float x_max = -FLT_MAX, x_min = FLT_MAX, y_max = -FLT_MAX, y_min = FLT_MAX;
    for (int j = netpin_start[i]; j < netpin_start[i + 1]; ++j) {
      float xx = x[flat_netpin[j]], yy = y[flat_netpin[j]];
      x_max = fmaxf_(xx, x_max);
      x_min = fminf_(xx, x_min);
      y_max = fmaxf_(yy, y_max);
      y_min = fminf_(yy, y_min);
    }
    float xe_p = 0, xe_n = 0, e_p = 0, e_n = 0, ye_p = 0, ye_n = 0, f_p = 0, f_n = 0;
    for (int j = netpin_start[i]; j < netpin_start[i + 1]; ++j) {
      float xx = x[flat_netpin[j]], yy = y[flat_netpin[j]];
      float ex = (float)exp((double)((xx - x_max) * inv_gamma));
      float enx = (float)exp((double)((x_min - xx) * inv_gamma));
      xe_p += xx * ex;
      xe_n += xx * enx;
      e_p += ex;
      e_n += enx;
      float ey = (float)exp((double)((yy - y_max) * inv_gamma));
      float eny = (float)exp((double)((y_min - yy) * inv_gamma));
      ye_p += yy * ey;
      ye_n += yy * eny;
      f_p += ey;
      f_n += eny;
    }
    partial_wl[i] = xe_p / e_p - xe_n / e_n + ye_p / f_p - ye_n / f_n;
    float b_x = inv_gamma / e_p;
    float a_x = (float)((1.0 - (double)(b_x * xe_p)) / (double)e_p);
    float b_nx = -inv_gamma / e_n;
    float a_nx = (float)((1.0 - (double)(b_nx * xe_n)) / (double)e_n);
    float b_y = inv_gamma / f_p;
    float a_y = (float)((1.0 - (double)(b_y * ye_p)) / (double)f_p);
    float b_ny = -inv_gamma / f_n;
    float a_ny = (float)((1.0 - (double)(b_ny * ye_n)) / (double)f_n);
    for (int j = netpin_start[i]; j < netpin_start[i + 1]; ++j) {
      int p = flat_netpin[j];
      float xx = x[p], yy = y[p];
      float ex = (float)exp((double)((xx - x_max) * inv_gamma));
      float enx = (float)exp((double)((x_min - xx) * inv_gamma));
      grad_x[p] = (a_x + b_x * xx) * ex - (a_nx + b_nx * xx) * enx;
      float ey = (float)exp((double)((yy - y_max) * inv_gamma));
      float eny = (float)exp((double)((y_min - yy) * inv_gamma));
      grad_y[p] = (a_y + b_y * yy) * ey - (a_ny + b_ny * yy) * eny;
    }
  }
}

/* hpwl/src/hpwl.cpp: per-net max-min+max-min, weighted, summed in double */
double oracle_hpwl(const float* x, const float* y, const int* flat_netpin, const int* netpin_start,
                   const unsigned char* net_mask, const float* net_weights, int num_nets) {
  double total = 0.0;
  for (int i = 0; i < num_nets; ++i) {
    if (!net_mask[i]) continue;
    float max_x = -FLT_MAX, min_x = FLT_MAX, max_y = -FLT_MAX, min_y = FLT_MAX;
    for (int j = netpin_start[i]; j < netpin_start[i + 1]; ++j) {
      float xx = x[flat_netpin[j]], yy = y[flat_netpin[j]];
      min_x = fminf_(min_x, xx);
      max_x = fmaxf_(max_x, xx);
      min_y = fminf_(min_y, yy);
      max_y = fmaxf_(max_y, yy);
    }
    float h = max_x - min_x + max_y - min_y;
    if (net_weights) h *= net_weights[i];
    total += (double)h;
  }
  return total;
}

/* pin_pos/src/pin_pos.cpp: forward gather and node-by-node backward */
void oracle_pin_pos(const float* x, const float* y, const float* offx, const float* offy, const int* pin2node,
                    int num_pins, float* px, float* py) {
  for (int p = 0; p < num_pins; ++p) {
    px[p] = offx[p] + x[pin2node[p]];
    py[p] = offy[p] + y[pin2node[p]];
  }
}

void oracle_pin_pos_backward(const float* gpx, const float* gpy, const int* flat_node2pin, const int* node_start,
                             int num_physical, float* gx, float* gy) {
  for (int i = 0; i < num_physical; ++i) {
    float sx = 0.0f, sy = 0.0f;
    for (int j = node_start[i]; j < node_start[i + 1]; ++j) {
      sx += gpx[flat_node2pin[j]];
      sy += gpy[flat_node2pin[j]];
    }
    gx[i] = sx;
    gy[i] = sy;
  }
}
