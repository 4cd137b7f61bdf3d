/*
 * dreamplace_b200 C ABI: the global-placement hot path of DREAMPlace as plain
 * C entry points over device pointers (sm_100a).
 *
 * Conventions
 *  - Every pointer is a device pointer unless its name ends in `_host`.
 *  - `pos` arrays are [x(n), y(n)] float32, node order movable | fixed | filler.
 *  - Bin maps are x-major: index = k * num_bins_y + h.
 *  - Every call is asynchronous on `stream` (NULL = legacy default stream),
 *    performs no host synchronisation and allocates no memory; scratch
 *    buffers are passed by the caller.
 *  - Return value: DP_OK (0) or a negative DP_ERR_* code; dp_last_error()
 *    returns a message for the calling thread's most recent failure.
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the reference project's dreamplace/ops/).
 */
#ifndef DREAMPLACE_B200_H
#define DREAMPLACE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dp_stream_t; /* same type as cudaStream_t */

enum {
  DP_REDUCE_DOUBLES = 1280,         /* 1 result + per-block partials of a fixed-order fp64 sum */
  DP_NESTEROV_STATE_DOUBLES = 8,
  DP_NOALLOC_MAX_BINS = 1048576     /* 1024 x 1024: scratch of dp_density_map_fx64_noalloc */
};

enum {
  DP_OK = 0,
  DP_ERR_INVALID_ARGUMENT = -1,
  DP_ERR_CUDA = -2,
  DP_ERR_UNSUPPORTED = -3,
  DP_ERR_TIMEOUT = -4
};

/* DCT / Poisson-solve arithmetic */
enum {
  DP_PREC_FP32 = 0,       /* SIMT FFMA, fp32 operands (the plain form)            */
  DP_PREC_TF32 = 1,       /* tcgen05 kind::tf32, fp32 accumulate                   */
  DP_PREC_BF16 = 2,       /* tcgen05 kind::f16 bf16 x bf16, fp32 accumulate        */
  DP_PREC_SPLIT_BF16 = 3  /* hi*hi + hi*lo + lo*hi bf16 products, fp32 accumulate  */
};

const char* dp_last_error(void);
int dp_version(void);
/* Number of kernels this library has launched in the calling process. */
uint64_t dp_launch_count(void);

/* ---- density scatter (electric_potential/src/electric_density_map_cuda.cpp:71-136,
 *      CPU electric_potential/src/electric_density_map.cpp:100-152) ----------
 * density_map = initial_density_map + triangle-model scatter of the movable
 * cells (visited through sorted_node_map when it is non-NULL) and the last
 * num_filler_nodes nodes.  inv_bin_size_x/y are the float reciprocals the
 * reference uses for the bin range.  density_map may alias initial_density_map. */
int dp_density_map_f32(const float* pos, int num_nodes,
                       const float* node_size_x_clamped, const float* node_size_y_clamped,
                       const float* offset_x, const float* offset_y, const float* ratio,
                       const float* initial_density_map,
                       float xl, float yl, float xh, float yh,
                       float bin_size_x, float bin_size_y,
                       float inv_bin_size_x, float inv_bin_size_y,
                       int num_movable_nodes, int num_filler_nodes,
                       int num_bins_x, int num_bins_y,
                       const int* sorted_node_map,
                       float* density_map, dp_stream_t stream);

/* Deterministic mode: every bin update is trunc(area * 2^fraction_bits) added to a
 * 64-bit integer map (int64 two's complement, as the reference CPU op's `long`),
 * then density_map = (float)((double)initial + (double)fixed * 2^-fraction_bits),
 * the CPU op's conversion (utility/src/atomic_ops.h:48-54).
 * scratch_fixed: caller-owned int64 [num_bins_x*num_bins_y]; on return it holds
 * the integer map (bit-exact with the reference CPU op's `buf`). */
int dp_density_map_fx64(const float* pos, int num_nodes,
                        const float* node_size_x_clamped, const float* node_size_y_clamped,
                        const float* offset_x, const float* offset_y, const float* ratio,
                        const float* initial_density_map,
                        float xl, float yl, float xh, float yh,
                        float bin_size_x, float bin_size_y,
                        float inv_bin_size_x, float inv_bin_size_y,
                        int num_movable_nodes, int num_filler_nodes,
                        int num_bins_x, int num_bins_y,
                        const int* sorted_node_map, int fraction_bits,
                        int64_t* scratch_fixed, float* density_map, dp_stream_t stream);

/* No counterpart in the reference.  Same result as dp_density_map_fx64, for
 * callers that cannot allocate device memory (a host that reserved the GPU
 * under a fixed budget, FFI hosts without the CUDA allocator).  The int64
 * scratch map is a built-in device array of DP_NOALLOC_MAX_BINS bins (8 MiB,
 * held by every GPU that loads the library until exit); larger grids are
 * rejected with DP_ERR_INVALID_ARGUMENT.  The first call under a CUDA context
 * looks up the array's device address in that context (and caches it with
 * the context's ID; a device reset or another context makes the next call
 * look it up again), so make that first call before any stream capture.  All
 * calls share the one array (it keeps the last call's integer map; each call
 * zeroes it before its scatter): calls that overlap on the GPU -- different
 * streams or threads -- race. */
int dp_density_map_fx64_noalloc(const float* pos, int num_nodes,
                                const float* node_size_x_clamped, const float* node_size_y_clamped,
                                const float* offset_x, const float* offset_y, const float* ratio,
                                const float* initial_density_map,
                                float xl, float yl, float xh, float yh,
                                float bin_size_x, float bin_size_y,
                                float inv_bin_size_x, float inv_bin_size_y,
                                int num_movable_nodes, int num_filler_nodes,
                                int num_bins_x, int num_bins_y,
                                const int* sorted_node_map, int fraction_bits,
                                float* density_map, dp_stream_t stream);

/* Per-cell records of the order-driven kernels: for idx < count, rec4[4*idx..] =
 * (sx, sy, ox, oy) (stretched sizes and offsets) and ratio_o[idx] = ratio of node
 * order[idx]; inv_order[order[idx]] = idx when inv_order is non-NULL. */
int dp_build_cell_records(const float* node_size_x_clamped, const float* node_size_y_clamped,
                          const float* offset_x, const float* offset_y, const float* ratio,
                          const int* order, int count, float* rec4, float* ratio_o, int* inv_order,
                          dp_stream_t stream);

/* Positions in visiting order: xy_o[2*idx..2*idx+1] = xy[2*order[idx]..] for
 * idx < count (interleaved xy as dp_pack_xy writes it). */
int dp_gather_order_xy(const float* xy, const int* order, int count, float* xy_o, dp_stream_t stream);

/* Order-driven triangle scatter of the cells 0..count of a visiting order onto
 * initial_density_map (NULL = zeros); positions (xy_o, interleaved) and
 * records (rec4, ratio_o) are both stored in that order.  Same per-bin
 * contributions as dp_density_map_f32 / _fx64.  Blocks of 512 consecutive
 * cells accumulate in a shared-memory tile over their bin box (int32 words)
 * before touching global memory, so a spatial order turns most global atomics
 * into local ones.  deterministic != 0: int64 fixed point, bit-exact with the
 * CPU op (scratch_fixed [num_bins] required); otherwise the tile sums each
 * block's contributions at a resolution of at most 2^-21 of the bin area and
 * adds them to the fp32 map with float atomics.  order (optional): the visiting order
 * itself; then xy_o holds the positions in node order and cell idx is read at
 * xy_o[order[idx]], so no visiting-order copy of the positions is needed. */
int dp_density_map_ordered(const float* xy_o, const int* order, const float* rec4, const float* ratio_o,
                           int count, const float* initial_density_map,
                           float xl, float yl, float xh, float yh,
                           float bin_size_x, float bin_size_y,
                           float inv_bin_size_x, float inv_bin_size_y,
                           int num_bins_x, int num_bins_y, int deterministic, int fraction_bits,
                           int64_t* scratch_fixed, float* density_map, dp_stream_t stream);

/* Two maps from one pass over the cells: out_first = initial_density_map +
 * cells [0, num_first) of the order, out_all = initial_density_map + cells
 * [0, count).  Used for the movable-only map (overflow metric) and the
 * movable + filler map (Poisson input) of one position, so each cell is
 * scattered once.  Deterministic: both maps bit-exact with separate scatters.
 * overflow_out (optional, DP_REDUCE_DOUBLES doubles): dp_density_overflow of
 * out_first with target_area and bin_area, computed in the same pass.
 * order: as dp_density_map_ordered. */
int dp_density_map_ordered_split(const float* xy_o, const int* order, const float* rec4, const float* ratio_o,
                                 int num_first, int count, const float* initial_density_map,
                                 float xl, float yl, float xh, float yh,
                                 float bin_size_x, float bin_size_y,
                                 float inv_bin_size_x, float inv_bin_size_y,
                                 int num_bins_x, int num_bins_y, int deterministic, int fraction_bits,
                                 int64_t* scratch_fixed, float* out_first, float* out_all,
                                 double target_area, double bin_area, double* overflow_out, dp_stream_t stream);

/* Exact-overlap fixed-cell map (electric_potential/src/electric_density_map_cuda.cpp:139-183,
 * CPU electric_potential/src/electric_density_map.cpp:155-213): nodes
 * [num_movable_nodes, num_movable_nodes+num_terminals), fixed_node_flag=true,
 * then clamp_max(bin area).  deterministic != 0 uses the int64 fixed-point path
 * and needs scratch_fixed [num_bins]; otherwise scratch_fixed may be NULL. */
int dp_fixed_density_map(const float* pos, int num_nodes,
                         const float* node_size_x, const float* node_size_y,
                         const float* bin_center_x, const float* bin_center_y,
                         float xl, float yl, float xh, float yh,
                         float bin_size_x, float bin_size_y,
                         int num_movable_nodes, int num_terminals,
                         int num_bins_x, int num_bins_y,
                         int deterministic, int fraction_bits,
                         int64_t* scratch_fixed, float* density_map, dp_stream_t stream);

/* Exact-overlap DensityMap (density_map/src/density_map.cpp:distributeBox2Bin,
 * CUDA density_map/src/density_map_cuda_kernel.cu:69-170): nodes of each half-open
 * range [range_begin_host[i], range_end_host[i]) are added onto density_map, which
 * holds the caller's initial map.  Bin size is (xh-xl)/num_bins_x in float; the y
 * range is widened by two bins each side; the last bin extends to the cell edge.
 * Deterministic mode converts each range's int64 map onto density_map in turn. */
int dp_density_map_exact(const float* pos, int num_nodes,
                         const float* node_size_x, const float* node_size_y,
                         const int* range_begin_host, const int* range_end_host, int num_ranges,
                         float xl, float yl, float xh, float yh,
                         int num_bins_x, int num_bins_y,
                         int deterministic, int fraction_bits, int64_t* scratch_fixed,
                         float* density_map, dp_stream_t stream);

/* Overflow evaluation (electric_potential/electric_overflow.py:260-278):
 * out2_f64[0] = sum(max(D - target_area, 0)), out2_f64[1] = max(D)/bin_area, in fp64
 * with a fixed-order (reproducible) sum; out2_f64 holds DP_REDUCE_DOUBLES doubles,
 * [2..] are scratch.  out_f32 (optional, 2 floats) receives both rounded. */
int dp_density_overflow(const float* density_map, int num_bins, double target_area,
                        double bin_area, double* out2_f64, float* out2_f32,
                        dp_stream_t stream);

/* ---- field gather (electric_potential/src/electric_force_cuda.cpp:56-124,
 *      CPU electric_potential/src/electric_force.cpp:76-172) ---------------
 * grad_out[i] = scale * grad_pos[0] * ratio_i * sum_{k,h} px*py*E[k,h] for movable
 * (through sorted_node_map when non-NULL) and filler nodes; fixed nodes get 0.
 * The per-cell sum follows the CPU op's loop order without contraction, so
 * with scale = -1 the result is bit-identical to -electric_force_cpp(...). */
int dp_electric_force(const float* grad_pos, int num_bins_x, int num_bins_y,
                      const float* field_map_x, const float* field_map_y,
                      const float* pos, int num_nodes,
                      const float* node_size_x_clamped, const float* node_size_y_clamped,
                      const float* offset_x, const float* offset_y, const float* ratio,
                      float xl, float yl, float xh, float yh,
                      float bin_size_x, float bin_size_y,
                      float inv_bin_size_x, float inv_bin_size_y,
                      int num_movable_nodes, int num_filler_nodes,
                      const int* sorted_node_map, float scale,
                      float* grad_out, dp_stream_t stream);

/* Field gather of the cells 0..count of a visiting order (records as
 * dp_build_cell_records, positions in the same order in xy_o); force_o[2*idx..2*idx+1] = scale * grad_pos[0] *
 * ratio * sum(px py E), in the CPU op's per-cell order without contraction.
 * order: as dp_density_map_ordered. */
int dp_electric_force_ordered(const float* grad_pos, int num_bins_x, int num_bins_y,
                              const float* field_map_x, const float* field_map_y, const float* xy_o, const int* order,
                              const float* rec4, const float* ratio_o, int count,
                              float xl, float yl, float bin_size_x, float bin_size_y,
                              float inv_bin_size_x, float inv_bin_size_y, float scale, float* force_o,
                              dp_stream_t stream);

/* ---- Poisson solve as GEMMs (replaces dct/src/dct2_fft2_cuda.cpp:14-140) ------
 * C[m,n] = sum_k A[m,k] * B[n,k]; A [M x K], B [N x K], both K-contiguous.
 * Operands are fp32 for DP_PREC_FP32/TF32 (a_lo/b_lo ignored), bf16 hi for
 * DP_PREC_BF16, bf16 hi+lo for DP_PREC_SPLIT_BF16.  `count` independent
 * problems (1..3) run in one launch; each dp_gemm_problem names its operands
 * and its epilogue. */
enum {
  DP_EPI_STORE = 0,      /* out_f32[m*ldc+n] = alpha*C                                  */
  DP_EPI_STORE_T = 1,    /* C^T as the next GEMM's operand: out_hi/out_lo (or out_f32) at [n*ldc+m], times alpha */
  DP_EPI_SPECTRAL = 2,   /* a=alpha*C -> row-major operands a*wu/(wu^2+wv^2)/2, a*wv/(...)/2 and (optional) a/(...);
                            with energy_f64: += M N sum w_u w_v a^2/(wu^2+wv^2), w_0 = 1/2 (the potential energy,
                            sum rho * IDCT2(a/(...)), without forming the potential) */
  DP_EPI_ENERGY = 3      /* energy_f64 += sum alpha*C[m,n]*rho[m*ldc+n]; optional out_f32 store */
};

typedef struct dp_gemm_problem {
  const void* a_hi; const void* a_lo; const void* b_hi; const void* b_lo;
  int lda, ldb;         /* leading dimensions in elements */
  int epilogue;         /* DP_EPI_* */
  float alpha;
  int ldc;
  float* out_f32;       /* STORE / STORE_T(fp32 operand) / ENERGY(optional) */
  void* out_hi; void* out_lo;  /* STORE_T bf16 operand halves */
  void* spec_out_hi[3]; void* spec_out_lo[3]; float* spec_out_f32[3]; /* SPECTRAL */
  float wv_scale;       /* SPECTRAL: bin_size_x / bin_size_y */
  const float* spec_weights; /* SPECTRAL, optional: [3*M*N] tables wx | wy | winv from
                                dp_spectral_weights (same values, no per-element divide) */
  const float* rho;     /* ENERGY */
  double* energy_f64;   /* ENERGY / SPECTRAL energy accumulator (caller zeroes it) */
} dp_gemm_problem;

int dp_transform_gemm(int precision, int M, int N, int K,
                      const dp_gemm_problem* problems_host, int count, dp_stream_t stream);

/* Spectral weight tables of the Poisson solve (electric_potential.py:504-519), in
 * the reference's fp32 arithmetic: out[0:MN] = wu/(wu^2+wv^2)/2, out[MN:2MN] =
 * wv/(wu^2+wv^2)/2, out[2MN:3MN] = 1/(wu^2+wv^2) (0 at [0,0]). */
int dp_spectral_weights(int M, int N, float wv_scale, float* out, dp_stream_t stream);

/* Reads and clears the tensor-core kernels' device status word (0 = every
 * bounded wait completed; non-zero = a wait expired and the launch returned
 * early).  Synchronises the device. */
int dp_tc_status(int* status_out);
/* Bound of every mbarrier wait of the tensor-core kernels, in SM clock cycles
 * (default 4e9, about 2 s); on expiry a kernel records its status word (see
 * dp_tc_status), lets what it issued drain, frees its TMEM and returns.
 * Synchronous; applies to kernels launched afterwards. */
int dp_tc_set_wait_budget(long long cycles);
/* Test hook for the bounded waits: while set, the tensor-core kernels' TMA
 * producer issues no copy, so the MMA warp's wait on the first operand stage
 * runs out (status 2) and the kernel returns with nothing in flight; the
 * outputs are then undefined.  Synchronous. */
int dp_tc_set_skip_loads(int skip);

/* Operand preparation: out = scale * x, written in the operand format of
 * `precision` (fp32, bf16 hi, or bf16 hi+lo). */
int dp_prepare_operand(int precision, const float* x, size_t n, float scale,
                       float* out_f32, void* out_hi, void* out_lo, dp_stream_t stream);

/* ---- WA wirelength, merged algorithm
 *      (weighted_average_wirelength/src/weighted_average_wirelength_cuda_merged.cpp:63-160,
 *       CPU weighted_average_wirelength/src/weighted_average_wirelength_merged.cpp:31-231) ----
 * forward: per masked net, x and y: max/min, exp sums, partial WL and the per-pin
 * gradient grad_intermediate [2*num_pins] (unmasked nets' pins are left 0 --
 * the caller zero-fills).  wl_out_f64 holds DP_REDUCE_DOUBLES doubles: [0] =
 * sum_e w_e * partial_e (fixed-order fp64 sum), [1..] scratch; wl_out (optional)
 * receives it rounded.  partial_wl: per-net weighted WL [num_nets] or NULL. */
int dp_wa_merged_forward(const float* pin_pos, int num_pins,
                         const int* flat_netpin, const int* netpin_start, int num_nets,
                         const float* net_weights, const unsigned char* net_mask,
                         const float* inv_gamma, float* partial_wl, double* wl_out_f64,
                         float* wl_out, float* grad_intermediate, dp_stream_t stream);
/* backward: grad_intermediate *= grad_pos[0] * w_{net(p)} (net masked in), then
 * pins with pin_mask != 0 are zeroed (weighted_average_wirelength.py:197-213). */
int dp_wa_merged_backward(const float* grad_pos, const int* pin2net_map,
                          const float* net_weights, const unsigned char* net_mask,
                          const unsigned char* pin_mask, int num_pins,
                          float* grad_intermediate, dp_stream_t stream);

/* ---- adjacent ops on every iteration ---------------------------------------- */
/* pin_pos/src/pin_pos_cuda_kernel.cu:11-27: pin[p] = pos[node(p)] + offset[p] */
int dp_pin_pos_forward(const float* pos, int num_nodes, const float* pin_offset_x,
                       const float* pin_offset_y, const int* pin2node_map, int num_pins,
                       float* pin_pos, dp_stream_t stream);
/* pin_pos/src/pin_pos_cuda_kernel.cu:50-74: node grad = sum of its pins' grads */
int dp_pin_pos_backward(const float* grad_pin_pos, int num_pins,
                        const int* flat_node2pin_map, const int* flat_node2pin_start_map,
                        int num_physical_nodes, int num_nodes, float* grad_pos,
                        dp_stream_t stream);
/* hpwl/src/hpwl_cuda_kernel.cu:10-39 (net-by-net); out_f64 holds DP_REDUCE_DOUBLES
 * doubles, [0] = fixed-order fp64 total; out_f32 optional */
int dp_hpwl(const float* pin_pos, int num_pins, const int* flat_netpin,
            const int* netpin_start, int num_nets, const float* net_weights,
            const unsigned char* net_mask, double* out_f64, float* out_f32,
            dp_stream_t stream);
/* move_boundary/src/move_boundary_cuda_kernel.cu:10-35, in place */
int dp_move_boundary(float* pos, int num_nodes, const float* node_size_x,
                     const float* node_size_y, float xl, float yl, float xh, float yh,
                     int num_movable_nodes, int num_filler_nodes, dp_stream_t stream);
/* pin_weight_sum/src/pws_cuda_kernel.cu: node weight = sum of its pins' net weights */
int dp_pin_weight_sum(const float* net_weights, const int* flat_nodepin,
                      const int* nodepin_start, const int* pin2net_map,
                      int num_physical_nodes, int num_nodes, float* node_weights,
                      dp_stream_t stream);

/* ---- fused global-placement iteration (engine path) ------------------------- */
/* Nesterov step of NesterovAcceleratedGradientOptimizer.step_nobb
 * (dreamplace/NesterovAcceleratedGradientOptimizer.py:65-166) on device
 * scalars state[DP_NESTEROV_STATE_DOUBLES + 2 * DP_REDUCE_DOUBLES] (fp64):
 * alpha_k, a_k, a_{k+1}, coef, two norms, alpha_{k+1}, accept flag, then
 * reduction scratch. */
int dp_nesterov_init(double* state, double alpha, dp_stream_t stream);
/* u' = v - alpha g; v' = clamp_die(u' + coef (u' - u)) (move_boundary semantics);
 * xy_new (optional, 8-byte aligned) receives v' interleaved as (x, y) pairs */
int dp_nesterov_trial(const float* v, const float* g, const float* u, float* u_new, float* v_new,
                      float* xy_new, const double* state, const float* node_size_x,
                      const float* node_size_y, float xl, float yl, float xh, float yh, int num_nodes,
                      int num_movable, int num_filler, const int* inv_order, float* xy_order,
                      dp_stream_t stream);
/* xy[2i], xy[2i+1] = pos[i], pos[num_nodes + i] */
int dp_pack_xy(const float* pos, int num_nodes, float* xy, dp_stream_t stream);
/* g' /= max(1, pws + lambda*area) (dreamplace/PlaceObj.py:69-103), then
 * alpha' = |v'-v| / |g'-g| in fp64, accept = alpha' > 0.95 alpha, alpha <- alpha' */
int dp_precondition_step_size(float* g_new, const float* g, const float* v_new, const float* v,
                              const float* pws, const float* area, const float* lambda_, int num_nodes,
                              double* state, dp_stream_t stream);
/* Gradient assembly fused with the preconditioner and the step size: for each
 * node, g' = wl_scale * (pin sum of grad_node_order, nodes < num_movable; pin k
 * of the node-CSR order is element grad_index[k] when grad_index is non-NULL) +
 * force_o[inv_order[node]] (movable and filler nodes), then as
 * dp_precondition_step_size. */
int dp_assemble_precondition_step(const float* grad_node_order, const int* node_start,
                                  const float* wl_scale, const float* force_o, const int* inv_order,
                                  int num_movable, int num_filler, const float* pws, const float* area,
                                  const float* lambda_, int num_nodes, const float* v_new, const float* v,
                                  const float* g, float* g_new, double* state, const int* grad_index,
                                  dp_stream_t stream);
/* The GP loop's work between iteration k and k+1 (dreamplace/NonLinearPlace.py
 * main loop; dreamplace/PlaceObj.py:833-851 update_density_weight in RePlAce
 * HPWL mode, :901-915 update_gamma), on the device: state_new <- state_prev's
 * scalars, advanced (a_k <- a_{k+1}, next a_{k+1} and coef); sched = {k, HPWL of iteration k-1}
 * (fp64[2]) becomes {k + 1, hpwl_k[0]}; weights = {lambda, gamma, 1/gamma}
 * (float[3]): with f = k + 1, lambda <- lambda * (float)mu for f > 1,
 * mu = upper * max(0.9999^f, 0.98) when HPWL fell, else
 * upper * min(max(upper^(-(hpwl_k - hpwl_{k-1}) / ref_hpwl), lower), upper);
 * gamma = (float)(base_gamma * 10^((overflow_k[0] / total_area - 0.1) * 20 / 9 - 1)).
 * Lets iteration k+1 be enqueued before the host reads iteration k.  gate
 * (optional): set to 1 when state_prev's last trial was rejected (the
 * iteration was enqueued ahead and is void), else 0 (dp_set_trial_gate). */
int dp_iteration_head(const double* state_prev, double* state_new, const double* sched_prev, double* sched_new,
                      const double* hpwl_k, const double* overflow_k, const float* weights_prev,
                      float* weights_new, double base_gamma, double total_area, double ref_hpwl, double lower,
                      double upper, int* gate, dp_stream_t stream);
/* Trial gate.  dp_set_trial_gate installs a device word (NULL removes it):
 * the kernels of the trial pieces launched while it is installed (the trial
 * point, position gather, WA, density scatter, operand preparation, transform
 * GEMMs, field gather, assembly) receive it and return at once when it holds a
 * non-zero value at run time.  Meant for CUDA-graph capture of a trial that is
 * enqueued ahead of the decision it depends on.  dp_trial_gate sets the word:
 * 1 when accept_prev is given and *accept_prev == 0, else 0. */
int dp_set_trial_gate(const int* gate);
int dp_trial_gate(int* gate, const double* accept_prev, dp_stream_t stream);
/* Lane-per-net plan (host): nets of degree 1..8 grouped 32 at a time by degree,
 * in the order net_order_host gives (a permutation of the nets; NULL: net
 * index order) within a degree; nets of degree 9..32 four of one degree per
 * group; each larger net a group of its own.  The
 * order only places the nets in memory: ordering nets by where their pins
 * live in the node arrays makes the pin-position gathers and the gradient
 * gather of the assembly local.  Call with
 * NULL group_deg / group_base / group_net / lane_slot to get *num_groups and
 * *num_lane_slots, then with buffers of those sizes (group_net: 32 per group).
 * Group g of degree d <= 8 stores pin j of lane l at lane slot
 * group_base[g] + 32 j + l; a group of degree 9..32 stores pin j of its net s
 * (s < 4, net id group_net[32 g + s]) at group_base[g] + s d + j; a larger net
 * stores its pins contiguously from group_base[g].  lane_slot maps lane slots
 * to pin slots (flat_netpin order), -1 for padding; group_net holds net ids,
 * -1 for padding lanes. */
int dp_plan_net_lanes(const int* netpin_start_host, int num_nets, const int* net_order_host, int* num_groups,
                      int* num_lane_slots, int* group_deg, int* group_base, int* group_net, int* lane_slot);
/* WA forward over a lane plan: one warp per group, one lane per net (degree
 * <= 8, pins in registers, the reference's per-net loops in pin order), eight
 * lanes per net (degree 9..32) or the whole warp for a larger net.  ln_node / ln_offx / ln_offy / ln_csr are the
 * pin arrays gathered to lane-slot order (ln_csr: the pin's position in
 * node-CSR order, where its gradient is written; NULL writes the gradient of
 * lane slot p at p).  The per-pin gradient, times the net weight, is written
 * as an (x, y) pair into grad_node_order; masked nets write 0.  wl_f64 holds
 * DP_REDUCE_DOUBLES doubles: [0] receives the fp64 total, the rest is scratch
 * for the fixed-order (run-to-run reproducible) reduction.  hpwl_f64
 * (optional, DP_REDUCE_DOUBLES doubles): the HPWL of the same pins under
 * hpwl_mask, equal to dp_hpwl_lanes on the same plan. */
int dp_wa_lanes_forward(const float* xy, const int* group_deg, const int* group_base, const int* group_net,
                        int num_groups, const int* ln_node, const float* ln_offx, const float* ln_offy,
                        const int* ln_csr, const float* net_weights, const unsigned char* net_mask,
                        const float* inv_gamma, double* wl_f64, float* grad_node_order,
                        const unsigned char* hpwl_mask, double* hpwl_f64, dp_stream_t stream);
/* HPWL over a lane plan (hpwl/src/hpwl_cuda_kernel.cu:10-39); out_f64: DP_REDUCE_DOUBLES */
int dp_hpwl_lanes(const float* xy, const int* group_deg, const int* group_base, const int* group_net,
                  int num_groups, const int* ln_node, const float* ln_offx, const float* ln_offy,
                  const float* net_weights, const unsigned char* net_mask, double* out_f64, dp_stream_t stream);
/* grad_out[node] (+)= sum over k in node_start[node]..node_start[node+1] of the
 * (x, y) pair grad_node_order[2k..2k+1] * grad_pos[0]; nodes >= num_movable get 0
 * (pin mask of fixed cells) */
int dp_node_pin_sum(const float* grad_node_order, int num_slots, const int* node_start, const float* grad_pos,
                    int num_movable, int num_nodes, int accumulate, float* grad_out, dp_stream_t stream);
/* WA merged forward on pin positions (weighted_average_wirelength/src/
 * weighted_average_wirelength_cuda_merged.cpp:63-118 forward): the lane-plan
 * kernel of dp_wa_lanes_forward reading pin_pos = [x(num_pins) | y(num_pins)]
 * (the reference op's input layout); ln_pin holds the pin id of each lane
 * slot (0 for padding).  grad_lane receives the per-pin gradient times the net
 * weight as (x, y) pairs in lane-slot order; wl_f64 as in dp_wa_lanes_forward. */
int dp_wa_pins_forward(const float* pin_pos, int num_pins, const int* group_deg, const int* group_base,
                       const int* group_net, int num_groups, const int* ln_pin, const float* net_weights,
                       const unsigned char* net_mask, const float* inv_gamma, double* wl_f64, float* grad_lane,
                       dp_stream_t stream);
/* WA merged backward (weighted_average_wirelength_cuda_merged.cpp:121-160 and
 * weighted_average_wirelength.py:197-213): grad_pin_pos[p] =
 * grad_out[0] * grad_lane[lane_of_pin[p]] (x block, then y block), 0 where
 * pin_mask[p] (optional, one byte per pin) is set. */
int dp_wa_pins_backward(const float* grad_lane, const int* lane_of_pin, const unsigned char* pin_mask,
                        const float* grad_out, int num_pins, float* grad_pin_pos, dp_stream_t stream);
/* Visiting order of the scattered cells for the order-driven kernels (no
 * reference counterpart; the reference visits movable cells through
 * sorted_node_map, BasicPlace.py:186-188): order[0..num_movable) holds the
 * movable cells and order[num_movable..) the fillers, each bucketed by the bin
 * where the stretched footprint starts (pos + offset; 16 x 16-bin tiles in
 * serpentine order, then the bin inside the tile) by a counting sort; inside
 * a bucket the order is arbitrary.  Each full block of 512 cells of either
 * range is then laid out for the ordered scatter: slot (32 w + l) * 2 + c
 * holds sorted rank 16 l + 2 w + c, so the 32 lanes of a warp take cells 16
 * ranks apart.  scratch: dp_order_cells_scratch_bytes bytes, 4-byte aligned. */
size_t dp_order_cells_scratch_bytes(int num_movable, int num_filler, int num_bins_x, int num_bins_y);
int dp_order_cells_by_bin(const float* pos, int num_nodes, const float* offset_x, const float* offset_y,
                          int num_movable, int num_filler, float xl, float yl, float inv_bin_size_x,
                          float inv_bin_size_y, int num_bins_x, int num_bins_y, void* scratch, size_t scratch_bytes,
                          int* order, dp_stream_t stream);
/* xy_o[2 idx], xy_o[2 idx + 1] = pos[order[idx]], pos[num_nodes + order[idx]]:
 * planar node positions gathered into visiting order, interleaved */
int dp_gather_order_pos(const float* pos, int num_nodes, const int* order, int count, float* xy_o,
                        dp_stream_t stream);
/* out = 0 (2 num_nodes floats), then out[order[idx]] = vals_o[2 idx] and
 * out[num_nodes + order[idx]] = vals_o[2 idx + 1]: pairs kept in visiting
 * order (e.g. the field force of dp_electric_force_ordered) put back in the
 * reference's node layout [x(n) | y(n)] */
int dp_scatter_pairs_to_nodes(const float* vals_o, const int* order, int count, int num_nodes, float* out,
                              dp_stream_t stream);

/* out8 = {hpwl[0], overflow2[0], overflow2[1], state accept flag, state step
 * size, obj[0], wl[0], energy[0]}: a GP trial's metrics gathered into the one
 * row the host reads back (the engine's own bookkeeping, no reference
 * counterpart). */
int dp_trial_metrics(const double* hpwl, const double* overflow2, const double* state, const double* obj,
                     const double* wl, const double* energy, double* out8, dp_stream_t stream);
/* Zeroes bytes at ptr on the stream (a memset, no kernel). */
int dp_zero(void* ptr, size_t bytes, dp_stream_t stream);

/* obj = wl + lambda_eff * D (1 + c D), lambda_eff = factor_quad[0] *
 * density_weight, c = factor_quad[1] (0: no quadratic penalty);
 * grad_scale = d obj / d D.  All operands live on the device, so a captured
 * graph follows changes of the density factor and penalty.  Either output may
 * be NULL (wl may be NULL with obj): grad_scale needs only the energy, so the
 * field gather can start before the wirelength is summed. */
int dp_objective_finish(const double* wl, const double* energy, const float* density_weight,
                        const float* factor_quad, double* obj, float* grad_scale, dp_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif
