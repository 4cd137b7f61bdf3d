// PyTorch extension over the dreamplace_b200 C ABI.
//
// Each function checks its tensors the way the reference's pybind ops do
// (CHECK_FLAT_CUDA / CHECK_CONTIGUOUS / CHECK_EVEN, utility/src/torch.h:62-76),
// allocates outputs through the caching allocator, launches on the current
// stream and turns a non-zero C ABI status into a Python RuntimeError.
// Function names and argument order follow the reference ops they replace:
//   electric_potential_cuda.{density_map, fixed_density_map, electric_force}
//   weighted_average_wirelength_cuda_merged.{forward, backward}
//   pin_pos_cuda.{forward, backward}, hpwl_cuda.forward, move_boundary_cuda.forward,
//   pws_cuda.forward
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/extension.h>

#include <cmath>

#include "dreamplace_b200.h"

namespace py = pybind11;

#define CHECK_CUDA_T(x) TORCH_CHECK((x).is_cuda(), #x " must be a CUDA tensor")
#define CHECK_CONTIG(x) TORCH_CHECK((x).is_contiguous(), #x " must be contiguous")
#define CHECK_FLAT(x) TORCH_CHECK((x).is_cuda() && (x).is_contiguous() && (x).dim() == 1, #x " must be a flat contiguous CUDA tensor")
#define CHECK_EVEN(x) TORCH_CHECK(((x).numel() & 1) == 0, #x " must have an even number of elements")
#define CHECK_F32(x) TORCH_CHECK((x).scalar_type() == at::kFloat, #x " must be float32")
#define CHECK_I32(x) TORCH_CHECK((x).scalar_type() == at::kInt, #x " must be int32")
#define DP_CALL(expr)                                                        \
  do {                                                                       \
    int _rc = (expr);                                                        \
    TORCH_CHECK(_rc == DP_OK, "dreamplace_b200: ", dp_last_error(), " (status ", _rc, ")"); \
  } while (0)

static dp_stream_t cur_stream() { return (dp_stream_t)at::cuda::getCurrentCUDAStream().stream(); }
template <typename T>
static T* ptr(const at::Tensor& t) { return t.data_ptr<T>(); }
template <typename T>
static T* optr(const c10::optional<at::Tensor>& t) {
  return (t.has_value() && t->defined() && t->numel() > 0) ? t->data_ptr<T>() : nullptr;
}

// float reciprocal as the reference CPU op computes it: T(1.0 / (double)T(b))
static float inv_f(double b) { return (float)(1.0 / (double)(float)b); }

static int fraction_bits(double xl, double yl, double xh, double yh) {
  double diearea = (xh - xl) * (yh - yl);
  int integer_bits = std::max((int)std::ceil(std::log2(diearea)) + 1, 32);
  return std::max(64 - integer_bits, 0);
}

// ---------------------------------------------------------------- density
at::Tensor density_map(at::Tensor pos, at::Tensor sx, at::Tensor sy, at::Tensor ox, at::Tensor oy,
                       at::Tensor ratio, at::Tensor bcx, at::Tensor bcy, at::Tensor init, double target_density,
                       double xl, double yl, double xh, double yh, double bsx, double bsy, int num_movable,
                       int num_filler, int padding, int nbx, int nby, int, int, int, int,
                       int deterministic, c10::optional<at::Tensor> sorted_node_map) {
  CHECK_FLAT(pos); CHECK_EVEN(pos); CHECK_F32(pos);
  for (auto* t : {&sx, &sy, &ox, &oy, &ratio}) { CHECK_FLAT(*t); CHECK_F32(*t); }
  CHECK_CUDA_T(init); CHECK_CONTIG(init); CHECK_F32(init);
  TORCH_CHECK(init.numel() == (int64_t)nbx * nby, "initial_density_map has ", init.numel(), " elements, expected ", nbx * nby);
  const int* snm = nullptr;
  if (sorted_node_map.has_value() && sorted_node_map->defined()) {
    CHECK_FLAT(*sorted_node_map); CHECK_I32(*sorted_node_map);
    TORCH_CHECK(sorted_node_map->numel() >= num_movable, "sorted_node_map shorter than num_movable_nodes");
    snm = ptr<int>(*sorted_node_map);
  }
  c10::cuda::CUDAGuard guard(pos.device());
  int n = pos.numel() / 2;
  auto out = at::empty({nbx, nby}, pos.options());
  if (deterministic) {
    auto scratch = at::empty({(int64_t)nbx * nby}, pos.options().dtype(at::kLong));
    DP_CALL(dp_density_map_fx64(ptr<float>(pos), n, ptr<float>(sx), ptr<float>(sy), ptr<float>(ox), ptr<float>(oy),
                                ptr<float>(ratio), ptr<float>(init), xl, yl, xh, yh, bsx, bsy, inv_f(bsx), inv_f(bsy),
                                num_movable, num_filler, nbx, nby, snm, fraction_bits(xl, yl, xh, yh),
                                ptr<int64_t>(scratch), ptr<float>(out), cur_stream()));
  } else {
    DP_CALL(dp_density_map_f32(ptr<float>(pos), n, ptr<float>(sx), ptr<float>(sy), ptr<float>(ox), ptr<float>(oy),
                               ptr<float>(ratio), ptr<float>(init), xl, yl, xh, yh, bsx, bsy, inv_f(bsx), inv_f(bsy),
                               num_movable, num_filler, nbx, nby, snm, ptr<float>(out), cur_stream()));
  }
  return out.view({-1});
}

// Integer fixed-point map of the deterministic scatter (for bit-exact checks).
at::Tensor density_map_fixed_point(at::Tensor pos, at::Tensor sx, at::Tensor sy, at::Tensor ox, at::Tensor oy,
                                   at::Tensor ratio, double xl, double yl, double xh, double yh, double bsx,
                                   double bsy, int num_movable, int num_filler, int nbx, int nby,
                                   c10::optional<at::Tensor> sorted_node_map) {
  CHECK_FLAT(pos); CHECK_F32(pos);
  c10::cuda::CUDAGuard guard(pos.device());
  int n = pos.numel() / 2;
  auto out = at::empty({nbx, nby}, pos.options());
  auto scratch = at::empty({(int64_t)nbx * nby}, pos.options().dtype(at::kLong));
  const int* snm = sorted_node_map.has_value() && sorted_node_map->defined() ? ptr<int>(*sorted_node_map) : nullptr;
  DP_CALL(dp_density_map_fx64(ptr<float>(pos), n, ptr<float>(sx), ptr<float>(sy), ptr<float>(ox), ptr<float>(oy),
                              ptr<float>(ratio), nullptr, xl, yl, xh, yh, bsx, bsy, inv_f(bsx), inv_f(bsy),
                              num_movable, num_filler, nbx, nby, snm, fraction_bits(xl, yl, xh, yh),
                              ptr<int64_t>(scratch), ptr<float>(out), cur_stream()));
  return scratch;
}

at::Tensor fixed_density_map(at::Tensor pos, at::Tensor sx, at::Tensor sy, at::Tensor bcx, at::Tensor bcy, double xl,
                             double yl, double xh, double yh, double bsx, double bsy, int num_movable,
                             int num_terminals, int nbx, int nby, int, int, int deterministic) {
  CHECK_FLAT(pos); CHECK_EVEN(pos); CHECK_F32(pos);
  c10::cuda::CUDAGuard guard(pos.device());
  int n = pos.numel() / 2;
  auto out = at::empty({nbx, nby}, pos.options());
  at::Tensor scratch;
  if (deterministic) scratch = at::empty({(int64_t)nbx * nby}, pos.options().dtype(at::kLong));
  DP_CALL(dp_fixed_density_map(ptr<float>(pos), n, ptr<float>(sx), ptr<float>(sy), ptr<float>(bcx), ptr<float>(bcy),
                               xl, yl, xh, yh, bsx, bsy, num_movable, num_terminals, nbx, nby, deterministic,
                               fraction_bits(xl, yl, xh, yh), deterministic ? ptr<int64_t>(scratch) : nullptr,
                               ptr<float>(out), cur_stream()));
  return out;
}

at::Tensor density_map_exact(at::Tensor pos, at::Tensor sx, at::Tensor sy, std::vector<int64_t> range_list,
                             at::Tensor initial, double xl, double yl, double xh, double yh, int nbx, int nby,
                             int deterministic) {
  CHECK_FLAT(pos); CHECK_F32(pos);
  c10::cuda::CUDAGuard guard(pos.device());
  int n = pos.numel() / 2;
  auto out = initial.clone().contiguous();
  std::vector<int> rb, re;
  for (size_t i = 0; i + 1 < range_list.size(); i += 2) {
    rb.push_back((int)range_list[i]);
    re.push_back((int)range_list[i + 1]);
  }
  at::Tensor scratch;
  if (deterministic) scratch = at::empty({(int64_t)nbx * nby}, pos.options().dtype(at::kLong));
  DP_CALL(dp_density_map_exact(ptr<float>(pos), n, ptr<float>(sx), ptr<float>(sy), rb.data(), re.data(), (int)rb.size(),
                               xl, yl, xh, yh, nbx, nby, deterministic, fraction_bits(xl, yl, xh, yh),
                               deterministic ? ptr<int64_t>(scratch) : nullptr, ptr<float>(out), cur_stream()));
  return out;
}

// overflow evaluation: returns fp64 [overflow, max_density]
at::Tensor density_overflow(at::Tensor density_map, double target_area, double bin_area) {
  CHECK_CUDA_T(density_map); CHECK_CONTIG(density_map); CHECK_F32(density_map);
  c10::cuda::CUDAGuard guard(density_map.device());
  auto out = at::empty({DP_REDUCE_DOUBLES}, density_map.options().dtype(at::kDouble));
  DP_CALL(dp_density_overflow(ptr<float>(density_map), density_map.numel(), target_area, bin_area, ptr<double>(out),
                              nullptr, cur_stream()));
  return out.narrow(0, 0, 2);
}

at::Tensor electric_force(at::Tensor grad_pos, int nbx, int nby, int, int, int, int, at::Tensor ex, at::Tensor ey,
                          at::Tensor pos, at::Tensor sx, at::Tensor sy, at::Tensor ox, at::Tensor oy, at::Tensor ratio,
                          at::Tensor bcx, at::Tensor bcy, double xl, double yl, double xh, double yh, double bsx,
                          double bsy, int num_movable, int num_filler, int deterministic,
                          c10::optional<at::Tensor> sorted_node_map, double scale) {
  CHECK_FLAT(pos); CHECK_EVEN(pos); CHECK_F32(pos);
  CHECK_CUDA_T(grad_pos); CHECK_F32(grad_pos);
  CHECK_CUDA_T(ex); CHECK_CONTIG(ex); CHECK_CUDA_T(ey); CHECK_CONTIG(ey);
  TORCH_CHECK(ex.numel() == (int64_t)nbx * nby && ey.numel() == (int64_t)nbx * nby, "field maps must be num_bins_x*num_bins_y");
  c10::cuda::CUDAGuard guard(pos.device());
  int n = pos.numel() / 2;
  auto out = at::empty_like(pos);
  auto g = grad_pos.contiguous();
  const int* snm = sorted_node_map.has_value() && sorted_node_map->defined() ? ptr<int>(*sorted_node_map) : nullptr;
  DP_CALL(dp_electric_force(ptr<float>(g), nbx, nby, ptr<float>(ex), ptr<float>(ey), ptr<float>(pos), n, ptr<float>(sx),
                            ptr<float>(sy), ptr<float>(ox), ptr<float>(oy), ptr<float>(ratio), xl, yl, xh, yh, bsx, bsy,
                            inv_f(bsx), inv_f(bsy), num_movable, num_filler, snm, (float)scale, ptr<float>(out),
                            cur_stream()));
  return out;
}

// ---------------------------------------------------------------- Poisson GEMMs
static void* tensor_ptr(const py::dict& d, const char* key) {
  if (!d.contains(key)) return nullptr;
  py::object o = d[key];
  if (o.is_none()) return nullptr;
  at::Tensor t = o.cast<at::Tensor>();
  TORCH_CHECK(t.is_cuda() && t.is_contiguous(), "transform_gemm: '", key, "' must be a contiguous CUDA tensor");
  return t.data_ptr();
}
template <typename T>
static T dict_get(const py::dict& d, const char* key, T dflt) {
  return d.contains(key) ? d[key].cast<T>() : dflt;
}

void transform_gemm(int precision, int M, int N, int K, py::list problems) {
  std::vector<dp_gemm_problem> probs;
  for (auto item : problems) {
    py::dict d = item.cast<py::dict>();
    dp_gemm_problem q;
    memset(&q, 0, sizeof(q));
    q.a_hi = tensor_ptr(d, "a_hi"); q.a_lo = tensor_ptr(d, "a_lo");
    q.b_hi = tensor_ptr(d, "b_hi"); q.b_lo = tensor_ptr(d, "b_lo");
    q.lda = dict_get<int>(d, "lda", K); q.ldb = dict_get<int>(d, "ldb", K);
    q.epilogue = dict_get<int>(d, "epilogue", DP_EPI_STORE);
    q.alpha = dict_get<float>(d, "alpha", 1.0f);
    q.ldc = dict_get<int>(d, "ldc", q.epilogue == DP_EPI_STORE_T ? M : N);
    q.out_f32 = (float*)tensor_ptr(d, "out_f32");
    q.out_hi = tensor_ptr(d, "out_hi"); q.out_lo = tensor_ptr(d, "out_lo");
    const char* kf[3] = {"sp0_f32", "sp1_f32", "sp2_f32"};
    const char* kh[3] = {"sp0_hi", "sp1_hi", "sp2_hi"};
    const char* kl[3] = {"sp0_lo", "sp1_lo", "sp2_lo"};
    for (int i = 0; i < 3; ++i) {
      q.spec_out_f32[i] = (float*)tensor_ptr(d, kf[i]);
      q.spec_out_hi[i] = tensor_ptr(d, kh[i]);
      q.spec_out_lo[i] = tensor_ptr(d, kl[i]);
    }
    q.wv_scale = dict_get<float>(d, "wv_scale", 1.0f);
    q.spec_weights = (const float*)tensor_ptr(d, "spec_weights");
    q.rho = (const float*)tensor_ptr(d, "rho");
    q.energy_f64 = (double*)tensor_ptr(d, "energy");
    probs.push_back(q);
  }
  DP_CALL(dp_transform_gemm(precision, M, N, K, probs.data(), (int)probs.size(), cur_stream()));
}

void prepare_operand(int precision, at::Tensor x, double scale, c10::optional<at::Tensor> out_f32,
                     c10::optional<at::Tensor> out_hi, c10::optional<at::Tensor> out_lo) {
  CHECK_CUDA_T(x); CHECK_CONTIG(x); CHECK_F32(x);
  DP_CALL(dp_prepare_operand(precision, ptr<float>(x), x.numel(), (float)scale, optr<float>(out_f32),
                             out_hi.has_value() ? out_hi->data_ptr() : nullptr,
                             out_lo.has_value() ? out_lo->data_ptr() : nullptr, cur_stream()));
}

at::Tensor spectral_weights(int M, int N, double wv_scale, at::Device device) {
  auto out = at::empty({3, M, N}, at::TensorOptions().dtype(at::kFloat).device(device));
  DP_CALL(dp_spectral_weights(M, N, (float)wv_scale, ptr<float>(out), cur_stream()));
  return out;
}

int tc_status() {
  int s = 0;
  DP_CALL(dp_tc_status(&s));
  return s;
}

// ---------------------------------------------------------------- wirelength
std::vector<at::Tensor> wa_merged_forward(at::Tensor pos, at::Tensor flat_netpin, at::Tensor netpin_start,
                                          at::Tensor pin2net_map, at::Tensor net_weights, at::Tensor net_mask,
                                          at::Tensor inv_gamma) {
  CHECK_FLAT(pos); CHECK_EVEN(pos); CHECK_F32(pos);
  CHECK_FLAT(flat_netpin); CHECK_I32(flat_netpin);
  CHECK_FLAT(netpin_start); CHECK_I32(netpin_start);
  CHECK_FLAT(net_mask);
  CHECK_CUDA_T(inv_gamma); CHECK_F32(inv_gamma);
  c10::cuda::CUDAGuard guard(pos.device());
  int num_nets = netpin_start.numel() - 1;
  int num_pins = pos.numel() / 2;
  auto grad_intermediate = at::empty_like(pos);
  auto wl = at::empty({}, pos.options());
  auto wl64 = at::empty({DP_REDUCE_DOUBLES}, pos.options().dtype(at::kDouble));
  auto ig = inv_gamma.contiguous();
  DP_CALL(dp_wa_merged_forward(ptr<float>(pos), num_pins, ptr<int>(flat_netpin), ptr<int>(netpin_start), num_nets,
                               net_weights.numel() ? ptr<float>(net_weights) : nullptr, net_mask.data_ptr<uint8_t>(),
                               ptr<float>(ig), nullptr, ptr<double>(wl64), ptr<float>(wl), ptr<float>(grad_intermediate),
                               cur_stream()));
  return {wl, grad_intermediate};
}

at::Tensor wa_merged_backward(at::Tensor grad_pos, at::Tensor pos, at::Tensor grad_intermediate, at::Tensor flat_netpin,
                              at::Tensor netpin_start, at::Tensor pin2net_map, at::Tensor net_weights,
                              at::Tensor net_mask, at::Tensor inv_gamma, c10::optional<at::Tensor> pin_mask) {
  CHECK_FLAT(grad_intermediate); CHECK_EVEN(grad_intermediate); CHECK_F32(grad_intermediate);
  CHECK_CUDA_T(grad_pos); CHECK_F32(grad_pos);
  CHECK_FLAT(pin2net_map); CHECK_I32(pin2net_map);
  c10::cuda::CUDAGuard guard(grad_intermediate.device());
  int num_pins = grad_intermediate.numel() / 2;
  auto g = grad_pos.contiguous();
  const uint8_t* pm = nullptr;
  if (pin_mask.has_value() && pin_mask->defined()) {
    CHECK_FLAT(*pin_mask);
    TORCH_CHECK(pin_mask->element_size() == 1, "pin_mask must be bool or uint8");
    pm = (const uint8_t*)pin_mask->data_ptr();
  }
  DP_CALL(dp_wa_merged_backward(ptr<float>(g), ptr<int>(pin2net_map),
                                net_weights.numel() ? ptr<float>(net_weights) : nullptr, net_mask.data_ptr<uint8_t>(),
                                pm, num_pins, ptr<float>(grad_intermediate), cur_stream()));
  return grad_intermediate;
}

at::Tensor pin_pos_forward(at::Tensor pos, at::Tensor offx, at::Tensor offy, at::Tensor pin2node) {
  CHECK_FLAT(pos); CHECK_EVEN(pos); CHECK_F32(pos); CHECK_I32(pin2node);
  c10::cuda::CUDAGuard guard(pos.device());
  int num_pins = offx.numel();
  auto out = at::empty({2 * (int64_t)num_pins}, pos.options());
  DP_CALL(dp_pin_pos_forward(ptr<float>(pos), pos.numel() / 2, ptr<float>(offx), ptr<float>(offy), ptr<int>(pin2node),
                             num_pins, ptr<float>(out), cur_stream()));
  return out;
}

at::Tensor pin_pos_backward(at::Tensor grad_out, at::Tensor pos, at::Tensor flat_node2pin, at::Tensor node2pin_start,
                            int num_physical_nodes) {
  CHECK_FLAT(grad_out); CHECK_EVEN(grad_out); CHECK_F32(grad_out);
  CHECK_I32(flat_node2pin); CHECK_I32(node2pin_start);
  c10::cuda::CUDAGuard guard(pos.device());
  auto out = at::empty_like(pos);
  DP_CALL(dp_pin_pos_backward(ptr<float>(grad_out), grad_out.numel() / 2, ptr<int>(flat_node2pin),
                              ptr<int>(node2pin_start), num_physical_nodes, pos.numel() / 2, ptr<float>(out),
                              cur_stream()));
  return out;
}

// returns fp64 [1] total
at::Tensor hpwl_forward(at::Tensor pin_pos, at::Tensor flat_netpin, at::Tensor netpin_start, at::Tensor net_weights,
                        at::Tensor net_mask) {
  CHECK_FLAT(pin_pos); CHECK_EVEN(pin_pos); CHECK_F32(pin_pos);
  c10::cuda::CUDAGuard guard(pin_pos.device());
  auto out = at::empty({DP_REDUCE_DOUBLES}, pin_pos.options().dtype(at::kDouble));
  DP_CALL(dp_hpwl(ptr<float>(pin_pos), pin_pos.numel() / 2, ptr<int>(flat_netpin), ptr<int>(netpin_start),
                  netpin_start.numel() - 1, net_weights.numel() ? ptr<float>(net_weights) : nullptr,
                  net_mask.data_ptr<uint8_t>(), ptr<double>(out), nullptr, cur_stream()));
  return out.narrow(0, 0, 1);
}

at::Tensor move_boundary_forward(at::Tensor pos, at::Tensor sx, at::Tensor sy, double xl, double yl, double xh,
                                 double yh, int num_movable, int num_filler) {
  CHECK_FLAT(pos); CHECK_EVEN(pos); CHECK_F32(pos);
  c10::cuda::CUDAGuard guard(pos.device());
  DP_CALL(dp_move_boundary(ptr<float>(pos), pos.numel() / 2, ptr<float>(sx), ptr<float>(sy), xl, yl, xh, yh,
                           num_movable, num_filler, cur_stream()));
  return pos;
}

at::Tensor pws_forward(at::Tensor net_weights, at::Tensor flat_nodepin, at::Tensor nodepin_start, at::Tensor pin2net,
                       int num_nodes) {
  CHECK_FLAT(net_weights); CHECK_F32(net_weights);
  c10::cuda::CUDAGuard guard(net_weights.device());
  auto out = at::empty({num_nodes}, net_weights.options());
  DP_CALL(dp_pin_weight_sum(ptr<float>(net_weights), ptr<int>(flat_nodepin), ptr<int>(nodepin_start),
                            ptr<int>(pin2net), nodepin_start.numel() - 1, num_nodes, ptr<float>(out), cur_stream()));
  return out;
}

// ---------------------------------------------------------------- engine kernels
static void* vp(const at::Tensor& t) { return t.data_ptr(); }
static void* ovp(const c10::optional<at::Tensor>& t) {
  return (t.has_value() && t->defined() && t->numel() > 0) ? t->data_ptr() : nullptr;
}

void nesterov_init(at::Tensor state, double alpha) { DP_CALL(dp_nesterov_init(ptr<double>(state), alpha, cur_stream())); }

void nesterov_trial(at::Tensor v, at::Tensor g, at::Tensor u, at::Tensor u_new, at::Tensor v_new,
                    c10::optional<at::Tensor> xy_new, at::Tensor state, at::Tensor sx, at::Tensor sy, double xl,
                    double yl, double xh, double yh, int num_movable, int num_filler,
                    c10::optional<at::Tensor> inv_order, c10::optional<at::Tensor> xy_order) {
  TORCH_CHECK(!xy_order.has_value() || inv_order.has_value(), "xy_order needs inv_order");
  DP_CALL(dp_nesterov_trial(ptr<float>(v), ptr<float>(g), ptr<float>(u), ptr<float>(u_new), ptr<float>(v_new),
                            (float*)ovp(xy_new), ptr<double>(state), ptr<float>(sx), ptr<float>(sy), xl, yl, xh, yh,
                            v.numel() / 2, num_movable, num_filler, (const int*)ovp(inv_order),
                            (float*)ovp(xy_order), cur_stream()));
}

void gather_order_xy(at::Tensor xy, at::Tensor order, int count, at::Tensor xy_o) {
  CHECK_FLAT(xy); CHECK_F32(xy); CHECK_I32(order); CHECK_F32(xy_o);
  TORCH_CHECK(count <= order.numel() && 2 * count <= xy_o.numel(), "gather_order_xy: buffers smaller than count");
  DP_CALL(dp_gather_order_xy(ptr<float>(xy), ptr<int>(order), count, ptr<float>(xy_o), cur_stream()));
}

void pack_xy(at::Tensor pos, at::Tensor xy) {
  CHECK_F32(pos); CHECK_F32(xy);
  TORCH_CHECK(xy.numel() == pos.numel(), "xy must have as many elements as pos");
  DP_CALL(dp_pack_xy(ptr<float>(pos), pos.numel() / 2, ptr<float>(xy), cur_stream()));
}

void precondition_step_size(at::Tensor g_new, at::Tensor g, at::Tensor v_new, at::Tensor v, at::Tensor pws,
                            at::Tensor area, at::Tensor lam, at::Tensor state) {
  DP_CALL(dp_precondition_step_size(ptr<float>(g_new), ptr<float>(g), ptr<float>(v_new), ptr<float>(v),
                                    ptr<float>(pws), ptr<float>(area), ptr<float>(lam), g_new.numel() / 2,
                                    ptr<double>(state), cur_stream()));
}

void iteration_head(at::Tensor state_prev, at::Tensor state_new, at::Tensor sched_prev, at::Tensor sched_new,
                    at::Tensor hpwl_k, at::Tensor overflow_k, at::Tensor weights_prev, at::Tensor weights_new,
                    double base_gamma, double total_area, double ref_hpwl, double lower, double upper,
                    c10::optional<at::Tensor> gate) {
  TORCH_CHECK(state_prev.scalar_type() == at::kDouble && state_new.scalar_type() == at::kDouble &&
                  sched_prev.scalar_type() == at::kDouble && sched_new.scalar_type() == at::kDouble &&
                  hpwl_k.scalar_type() == at::kDouble && overflow_k.scalar_type() == at::kDouble,
              "iteration_head: state, sched and metrics must be float64");
  TORCH_CHECK(state_prev.numel() >= DP_NESTEROV_STATE_DOUBLES && state_new.numel() >= DP_NESTEROV_STATE_DOUBLES &&
                  sched_prev.numel() >= 2 && sched_new.numel() >= 2 && weights_prev.numel() >= 3 &&
                  weights_new.numel() >= 3,
              "iteration_head: buffers too small");
  CHECK_F32(weights_prev); CHECK_F32(weights_new);
  DP_CALL(dp_iteration_head(ptr<double>(state_prev), ptr<double>(state_new), ptr<double>(sched_prev),
                            ptr<double>(sched_new), ptr<double>(hpwl_k), ptr<double>(overflow_k),
                            ptr<float>(weights_prev), ptr<float>(weights_new), base_gamma, total_area, ref_hpwl,
                            lower, upper, gate.has_value() ? ptr<int>(*gate) : nullptr, cur_stream()));
}

// the installed gate word must stay alive while graphs captured with it exist
void set_trial_gate(c10::optional<at::Tensor> gate) {
  if (gate.has_value()) {
    CHECK_I32(*gate);
    TORCH_CHECK(gate->is_cuda(), "trial gate must be a CUDA tensor");
  }
  DP_CALL(dp_set_trial_gate(gate.has_value() ? ptr<int>(*gate) : nullptr));
}

void trial_gate(at::Tensor gate, c10::optional<at::Tensor> accept_prev) {
  CHECK_I32(gate);
  DP_CALL(dp_trial_gate(ptr<int>(gate), accept_prev.has_value() ? ptr<double>(*accept_prev) : nullptr,
                        cur_stream()));
}

void objective_finish(c10::optional<at::Tensor> wl, at::Tensor energy, at::Tensor density_weight,
                      at::Tensor factor_quad, c10::optional<at::Tensor> obj, c10::optional<at::Tensor> grad_scale) {
  CHECK_F32(factor_quad);
  TORCH_CHECK(factor_quad.numel() >= 2, "factor_quad holds (density_factor, quad_c)");
  DP_CALL(dp_objective_finish(wl.has_value() ? ptr<double>(*wl) : nullptr, ptr<double>(energy),
                              ptr<float>(density_weight), ptr<float>(factor_quad),
                              obj.has_value() ? ptr<double>(*obj) : nullptr,
                              grad_scale.has_value() ? ptr<float>(*grad_scale) : nullptr, cur_stream()));
}

void build_cell_records(at::Tensor sx, at::Tensor sy, at::Tensor ox, at::Tensor oy, at::Tensor ratio,
                        at::Tensor order, int count, at::Tensor rec4, at::Tensor ratio_o,
                        c10::optional<at::Tensor> inv_order) {
  CHECK_I32(order); CHECK_F32(rec4); CHECK_F32(ratio_o);
  TORCH_CHECK(count <= order.numel() && 4 * count <= rec4.numel() && count <= ratio_o.numel(),
              "build_cell_records: buffers smaller than count");
  DP_CALL(dp_build_cell_records(ptr<float>(sx), ptr<float>(sy), ptr<float>(ox), ptr<float>(oy), ptr<float>(ratio),
                                ptr<int>(order), count, ptr<float>(rec4), ptr<float>(ratio_o), (int*)ovp(inv_order),
                                cur_stream()));
}

void density_map_ordered_into(at::Tensor xy_o, at::Tensor rec4, at::Tensor ratio_o, int count,
                              c10::optional<at::Tensor> init, double xl, double yl, double xh, double yh, double bsx,
                              double bsy, int nbx, int nby, int deterministic, c10::optional<at::Tensor> scratch,
                              at::Tensor out, c10::optional<at::Tensor> order) {
  CHECK_FLAT(xy_o); CHECK_F32(xy_o); CHECK_F32(rec4);
  if (order.has_value()) {
    CHECK_I32(*order);
    TORCH_CHECK(order->numel() >= count, "density_map_ordered_into: order shorter than count");
  }
  TORCH_CHECK(2 * count <= xy_o.numel() && 4 * count <= rec4.numel() && count <= ratio_o.numel(),
              "density_map_ordered_into: buffers smaller than count");
  TORCH_CHECK(out.numel() == (int64_t)nbx * nby, "density_map_ordered_into: output is not num_bins_x*num_bins_y");
  TORCH_CHECK(!deterministic || scratch.has_value(), "deterministic mode needs the int64 scratch map");
  DP_CALL(dp_density_map_ordered(ptr<float>(xy_o), (const int*)ovp(order), ptr<float>(rec4), ptr<float>(ratio_o),
                                 count,
                                 (const float*)ovp(init), xl, yl, xh, yh, bsx, bsy, inv_f(bsx), inv_f(bsy), nbx, nby,
                                 deterministic, fraction_bits(xl, yl, xh, yh), (int64_t*)ovp(scratch),
                                 ptr<float>(out), cur_stream()));
}

void density_map_ordered_split(at::Tensor xy_o, at::Tensor rec4, at::Tensor ratio_o, int num_first,
                               int count, c10::optional<at::Tensor> init, double xl, double yl, double xh, double yh,
                               double bsx, double bsy, int nbx, int nby, int deterministic,
                               c10::optional<at::Tensor> scratch, at::Tensor out_first, at::Tensor out_all,
                               double target_area, double bin_area, c10::optional<at::Tensor> overflow_out,
                               c10::optional<at::Tensor> order) {
  if (order.has_value()) {
    CHECK_I32(*order);
    TORCH_CHECK(order->numel() >= count, "density_map_ordered_split: order shorter than count");
  }
  TORCH_CHECK(!overflow_out.has_value() || (overflow_out->scalar_type() == at::kDouble &&
                                            overflow_out->numel() >= DP_REDUCE_DOUBLES),
              "overflow_out needs DP_REDUCE_DOUBLES doubles");
  CHECK_FLAT(xy_o); CHECK_F32(xy_o); CHECK_F32(rec4);
  TORCH_CHECK(2 * count <= xy_o.numel() && 4 * count <= rec4.numel() && count <= ratio_o.numel(),
              "density_map_ordered_split: buffers smaller than count");
  TORCH_CHECK(out_first.numel() == (int64_t)nbx * nby && out_all.numel() == out_first.numel(),
              "density_map_ordered_split: outputs are not num_bins_x*num_bins_y");
  TORCH_CHECK(!deterministic || scratch.has_value(), "deterministic mode needs the int64 scratch map");
  DP_CALL(dp_density_map_ordered_split(ptr<float>(xy_o), (const int*)ovp(order), ptr<float>(rec4),
                                       ptr<float>(ratio_o),
                                       num_first, count, (const float*)ovp(init), xl, yl, xh, yh, bsx, bsy,
                                       inv_f(bsx), inv_f(bsy), nbx, nby, deterministic, fraction_bits(xl, yl, xh, yh),
                                       (int64_t*)ovp(scratch), ptr<float>(out_first), ptr<float>(out_all),
                                       target_area, bin_area, (double*)ovp(overflow_out), cur_stream()));
}

void electric_force_ordered(at::Tensor grad_scale, at::Tensor ex, at::Tensor ey, at::Tensor xy_o, at::Tensor rec4,
                            at::Tensor ratio_o, int count, double xl, double yl, double bsx, double bsy, int nbx,
                            int nby, double scale, at::Tensor force_o, c10::optional<at::Tensor> order) {
  CHECK_FLAT(xy_o); CHECK_F32(force_o);
  if (order.has_value()) {
    CHECK_I32(*order);
    TORCH_CHECK(order->numel() >= count, "electric_force_ordered: order shorter than count");
  }
  TORCH_CHECK(2 * count <= xy_o.numel() && 4 * count <= rec4.numel() && 2 * count <= force_o.numel(),
              "electric_force_ordered: buffers smaller than count");
  TORCH_CHECK(ex.numel() == (int64_t)nbx * nby && ey.numel() == ex.numel(), "electric_force_ordered: field map size");
  DP_CALL(dp_electric_force_ordered(ptr<float>(grad_scale), nbx, nby, ptr<float>(ex), ptr<float>(ey), ptr<float>(xy_o),
                                    (const int*)ovp(order),
                                    ptr<float>(rec4), ptr<float>(ratio_o), count, xl, yl, bsx, bsy,
                                    inv_f(bsx), inv_f(bsy), (float)scale, ptr<float>(force_o), cur_stream()));
}

void assemble_precondition_step(at::Tensor grad_node_order, at::Tensor node_start, at::Tensor wl_scale,
                                at::Tensor force_o, at::Tensor inv_order, int num_movable, int num_filler,
                                at::Tensor pws, at::Tensor area, at::Tensor lambda_, at::Tensor v_new, at::Tensor v,
                                at::Tensor g, at::Tensor g_new, at::Tensor state, c10::optional<at::Tensor> grad_index) {
  CHECK_I32(node_start); CHECK_I32(inv_order);
  int n = v.numel() / 2;
  TORCH_CHECK(inv_order.numel() >= n && node_start.numel() >= num_movable + 1 && g_new.numel() == 2 * n,
              "assemble_precondition_step: size mismatch");
  DP_CALL(dp_assemble_precondition_step(ptr<float>(grad_node_order), ptr<int>(node_start), ptr<float>(wl_scale),
                                        ptr<float>(force_o), ptr<int>(inv_order), num_movable, num_filler,
                                        ptr<float>(pws), ptr<float>(area), ptr<float>(lambda_), n, ptr<float>(v_new),
                                        ptr<float>(v), ptr<float>(g), ptr<float>(g_new), ptr<double>(state),
                                        (const int*)ovp(grad_index), cur_stream()));
}

void density_overflow_into(at::Tensor density_map, double target_area, double bin_area, at::Tensor out2) {
  DP_CALL(dp_density_overflow(ptr<float>(density_map), density_map.numel(), target_area, bin_area, ptr<double>(out2),
                              nullptr, cur_stream()));
}

void electric_force_into(at::Tensor grad_scale, at::Tensor ex, at::Tensor ey, at::Tensor pos, at::Tensor sx,
                         at::Tensor sy, at::Tensor ox, at::Tensor oy, at::Tensor ratio, double xl, double yl,
                         double xh, double yh, double bsx, double bsy, int nbx, int nby, int num_movable,
                         int num_filler, c10::optional<at::Tensor> sorted_node_map, double scale, at::Tensor out) {
  DP_CALL(dp_electric_force(ptr<float>(grad_scale), nbx, nby, ptr<float>(ex), ptr<float>(ey), ptr<float>(pos),
                            pos.numel() / 2, ptr<float>(sx), ptr<float>(sy), ptr<float>(ox), ptr<float>(oy),
                            ptr<float>(ratio), xl, yl, xh, yh, bsx, bsy, inv_f(bsx), inv_f(bsy), num_movable,
                            num_filler, (const int*)ovp(sorted_node_map), (float)scale, ptr<float>(out), cur_stream()));
}

std::vector<at::Tensor> plan_net_lanes(at::Tensor netpin_start_cpu, c10::optional<at::Tensor> net_order_cpu) {
  TORCH_CHECK(!netpin_start_cpu.is_cuda() && netpin_start_cpu.scalar_type() == at::kInt,
              "netpin_start must be int32 on CPU");
  auto ns = netpin_start_cpu.contiguous();
  const int num_nets = ns.numel() - 1;
  at::Tensor order;
  if (net_order_cpu.has_value()) {
    order = net_order_cpu->contiguous();
    TORCH_CHECK(!order.is_cuda() && order.scalar_type() == at::kInt && order.numel() == num_nets,
                "net_order must be int32 on CPU with one entry per net");
  }
  const int* op = order.defined() ? order.data_ptr<int>() : nullptr;
  int groups = 0, slots = 0;
  DP_CALL(dp_plan_net_lanes(ns.data_ptr<int>(), num_nets, op, &groups, &slots, nullptr, nullptr, nullptr, nullptr));
  auto opt = ns.options();
  auto deg = at::empty({groups}, opt), base = at::empty({groups}, opt);
  auto net = at::empty({32 * (int64_t)groups}, opt), slot = at::empty({slots}, opt);
  DP_CALL(dp_plan_net_lanes(ns.data_ptr<int>(), num_nets, op, &groups, &slots, deg.data_ptr<int>(),
                            base.data_ptr<int>(), net.data_ptr<int>(), slot.data_ptr<int>()));
  return {deg, base, net, slot};
}

void wa_lanes_forward(at::Tensor xy, at::Tensor group_deg, at::Tensor group_base, at::Tensor group_net,
                      at::Tensor ln_node, at::Tensor ln_offx, at::Tensor ln_offy, c10::optional<at::Tensor> ln_csr,
                      c10::optional<at::Tensor> net_weights, at::Tensor net_mask, at::Tensor inv_gamma,
                      at::Tensor wl_f64, at::Tensor grad_node_order, c10::optional<at::Tensor> hpwl_mask,
                      c10::optional<at::Tensor> hpwl_f64) {
  CHECK_FLAT(xy); CHECK_F32(xy); CHECK_I32(group_deg); CHECK_I32(group_base); CHECK_I32(group_net);
  CHECK_I32(ln_node); CHECK_F32(grad_node_order);
  TORCH_CHECK(group_net.numel() == 32 * group_deg.numel() && group_base.numel() == group_deg.numel(),
              "wa_lanes_forward: inconsistent plan");
  TORCH_CHECK(wl_f64.scalar_type() == at::kDouble && wl_f64.numel() >= DP_REDUCE_DOUBLES, "wl_f64 too small");
  TORCH_CHECK(!hpwl_f64.has_value() || (hpwl_mask.has_value() && hpwl_f64->scalar_type() == at::kDouble &&
                                        hpwl_f64->numel() >= DP_REDUCE_DOUBLES),
              "hpwl_f64 needs hpwl_mask and DP_REDUCE_DOUBLES doubles");
  DP_CALL(dp_wa_lanes_forward(ptr<float>(xy), ptr<int>(group_deg), ptr<int>(group_base), ptr<int>(group_net),
                              group_deg.numel(), ptr<int>(ln_node), ptr<float>(ln_offx), ptr<float>(ln_offy),
                              (const int*)ovp(ln_csr), (const float*)ovp(net_weights), net_mask.data_ptr<uint8_t>(),
                              ptr<float>(inv_gamma), ptr<double>(wl_f64), ptr<float>(grad_node_order),
                              hpwl_mask.has_value() ? hpwl_mask->data_ptr<uint8_t>() : nullptr,
                              (double*)ovp(hpwl_f64), cur_stream()));
}

void hpwl_lanes(at::Tensor xy, at::Tensor group_deg, at::Tensor group_base, at::Tensor group_net, at::Tensor ln_node,
                at::Tensor ln_offx, at::Tensor ln_offy, c10::optional<at::Tensor> net_weights, at::Tensor net_mask,
                at::Tensor out_f64) {
  CHECK_FLAT(xy); CHECK_I32(group_deg); CHECK_I32(group_base); CHECK_I32(group_net); CHECK_I32(ln_node);
  TORCH_CHECK(group_net.numel() == 32 * group_deg.numel(), "hpwl_lanes: inconsistent plan");
  TORCH_CHECK(out_f64.scalar_type() == at::kDouble && out_f64.numel() >= DP_REDUCE_DOUBLES, "out_f64 too small");
  DP_CALL(dp_hpwl_lanes(ptr<float>(xy), ptr<int>(group_deg), ptr<int>(group_base), ptr<int>(group_net),
                        group_deg.numel(), ptr<int>(ln_node), ptr<float>(ln_offx), ptr<float>(ln_offy),
                        (const float*)ovp(net_weights), net_mask.data_ptr<uint8_t>(), ptr<double>(out_f64),
                        cur_stream()));
}

void node_pin_sum(at::Tensor grad_node_order, at::Tensor node_start, at::Tensor grad_pos, int num_movable,
                  int accumulate, at::Tensor grad_out) {
  CHECK_F32(grad_node_order); CHECK_F32(grad_out); CHECK_I32(node_start);
  DP_CALL(dp_node_pin_sum(ptr<float>(grad_node_order), grad_node_order.numel() / 2, ptr<int>(node_start),
                          ptr<float>(grad_pos), num_movable, grad_out.numel() / 2, accumulate, ptr<float>(grad_out),
                          cur_stream()));
}

void wa_pins_forward(at::Tensor pin_pos, at::Tensor group_deg, at::Tensor group_base, at::Tensor group_net,
                     at::Tensor ln_pin, c10::optional<at::Tensor> net_weights, at::Tensor net_mask,
                     at::Tensor inv_gamma, at::Tensor wl_f64, at::Tensor grad_lane) {
  CHECK_FLAT(pin_pos); CHECK_F32(pin_pos); CHECK_EVEN(pin_pos); CHECK_I32(group_deg); CHECK_I32(group_base);
  CHECK_I32(group_net); CHECK_I32(ln_pin); CHECK_F32(grad_lane); CHECK_F32(inv_gamma);
  TORCH_CHECK(group_net.numel() == 32 * group_deg.numel() && group_base.numel() == group_deg.numel(),
              "wa_pins_forward: inconsistent plan");
  TORCH_CHECK(grad_lane.numel() >= 2 * ln_pin.numel(), "wa_pins_forward: grad_lane smaller than the lane slots");
  TORCH_CHECK(wl_f64.scalar_type() == at::kDouble && wl_f64.numel() >= DP_REDUCE_DOUBLES, "wl_f64 too small");
  DP_CALL(dp_wa_pins_forward(ptr<float>(pin_pos), pin_pos.numel() / 2, ptr<int>(group_deg), ptr<int>(group_base),
                             ptr<int>(group_net), group_deg.numel(), ptr<int>(ln_pin), (const float*)ovp(net_weights),
                             net_mask.data_ptr<uint8_t>(), ptr<float>(inv_gamma), ptr<double>(wl_f64),
                             ptr<float>(grad_lane), cur_stream()));
}

at::Tensor wa_pins_backward(at::Tensor grad_lane, at::Tensor lane_of_pin, c10::optional<at::Tensor> pin_mask,
                            at::Tensor grad_out) {
  CHECK_F32(grad_lane); CHECK_I32(lane_of_pin); CHECK_F32(grad_out);
  const int64_t P = lane_of_pin.numel();
  TORCH_CHECK(!pin_mask.has_value() || (pin_mask->numel() == P && pin_mask->element_size() == 1),
              "wa_pins_backward: pin_mask must hold one byte per pin");
  auto out = at::empty({2 * P}, grad_lane.options());
  DP_CALL(dp_wa_pins_backward(ptr<float>(grad_lane), ptr<int>(lane_of_pin),
                              pin_mask.has_value() ? (const unsigned char*)pin_mask->data_ptr() : nullptr,
                              ptr<float>(grad_out), (int)P, ptr<float>(out), cur_stream()));
  return out;
}

int64_t order_cells_scratch_bytes(int num_movable, int num_filler, int nbx, int nby) {
  return (int64_t)dp_order_cells_scratch_bytes(num_movable, num_filler, nbx, nby);
}

void order_cells_by_bin(at::Tensor pos, at::Tensor ox, at::Tensor oy, int num_movable, int num_filler, double xl,
                        double yl, double bsx, double bsy, int nbx, int nby, at::Tensor scratch, at::Tensor order) {
  CHECK_FLAT(pos); CHECK_F32(pos); CHECK_EVEN(pos); CHECK_I32(order); CHECK_CUDA_T(scratch); CHECK_CONTIG(scratch);
  TORCH_CHECK(order.numel() >= num_movable + num_filler, "order_cells_by_bin: order too small");
  DP_CALL(dp_order_cells_by_bin(ptr<float>(pos), pos.numel() / 2, ptr<float>(ox), ptr<float>(oy), num_movable,
                                num_filler, xl, yl, inv_f(bsx), inv_f(bsy), nbx, nby, scratch.data_ptr(),
                                (size_t)scratch.numel() * scratch.element_size(), ptr<int>(order), cur_stream()));
}

void gather_order_pos(at::Tensor pos, at::Tensor order, int count, at::Tensor xy_o) {
  CHECK_FLAT(pos); CHECK_F32(pos); CHECK_I32(order); CHECK_F32(xy_o);
  TORCH_CHECK(order.numel() >= count && xy_o.numel() >= 2 * count, "gather_order_pos: buffers smaller than count");
  DP_CALL(dp_gather_order_pos(ptr<float>(pos), pos.numel() / 2, ptr<int>(order), count, ptr<float>(xy_o),
                              cur_stream()));
}

at::Tensor scatter_pairs_to_nodes(at::Tensor vals_o, at::Tensor order, int count, int num_nodes) {
  CHECK_F32(vals_o); CHECK_I32(order);
  TORCH_CHECK(order.numel() >= count && vals_o.numel() >= 2 * count, "scatter_pairs_to_nodes: buffers too small");
  auto out = at::empty({2 * (int64_t)num_nodes}, vals_o.options());
  DP_CALL(dp_scatter_pairs_to_nodes(ptr<float>(vals_o), ptr<int>(order), count, num_nodes, ptr<float>(out),
                                    cur_stream()));
  return out;
}

uint64_t launch_count() { return dp_launch_count(); }

// Launches an instantiated CUDA graph (torch.cuda.CUDAGraph.raw_cuda_graph_exec)
// on a stream (raw handle): the replay of a captured GP trial without
// torch's per-replay bookkeeping, which only serves graphs that draw random
// numbers (these do not).
void graph_launch(int64_t graph_exec, int64_t stream) {
  TORCH_CHECK(graph_exec != 0, "graph_launch: null graph");
  cudaError_t e = cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(graph_exec),
                                  reinterpret_cast<cudaStream_t>(stream));
  TORCH_CHECK(e == cudaSuccess, "graph_launch: ", cudaGetErrorString(e));
}

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "dreamplace_b200 native ops (sm_100a) over the C ABI";
  m.def("density_map", &density_map);
  m.def("wa_pins_forward", &wa_pins_forward);
  m.def("wa_pins_backward", &wa_pins_backward);
  m.def("order_cells_scratch_bytes", &order_cells_scratch_bytes);
  m.def("order_cells_by_bin", &order_cells_by_bin);
  m.def("gather_order_pos", &gather_order_pos);
  m.def("scatter_pairs_to_nodes", &scatter_pairs_to_nodes);
  m.def("density_map_fixed_point", &density_map_fixed_point);
  m.def("fixed_density_map", &fixed_density_map);
  m.def("density_map_exact", &density_map_exact);
  m.def("density_overflow", &density_overflow);
  m.def("electric_force", &electric_force);
  m.def("transform_gemm", &transform_gemm);
  m.def("prepare_operand", &prepare_operand);
  m.def("tc_status", &tc_status);
  m.def("trial_metrics", [](at::Tensor hpwl, at::Tensor overflow2, at::Tensor state, at::Tensor obj, at::Tensor wl,
                            at::Tensor energy, at::Tensor out8) {
    TORCH_CHECK(out8.scalar_type() == at::kDouble && out8.numel() >= 8, "trial_metrics: out8 needs 8 doubles");
    DP_CALL(dp_trial_metrics(ptr<double>(hpwl), ptr<double>(overflow2), ptr<double>(state), ptr<double>(obj),
                             ptr<double>(wl), ptr<double>(energy), ptr<double>(out8), cur_stream()));
  });
  m.def("zero_", [](at::Tensor t) {
    CHECK_CUDA_T(t); CHECK_CONTIG(t);
    DP_CALL(dp_zero(t.data_ptr(), (size_t)t.numel() * t.element_size(), cur_stream()));
  });
  m.def("tc_set_wait_budget", [](long long cycles) { DP_CALL(dp_tc_set_wait_budget(cycles)); });
  m.def("tc_set_skip_loads", [](int skip) { DP_CALL(dp_tc_set_skip_loads(skip)); });
  m.def("spectral_weights", &spectral_weights);
  m.def("wa_merged_forward", &wa_merged_forward);
  m.def("wa_merged_backward", &wa_merged_backward);
  m.def("pin_pos_forward", &pin_pos_forward);
  m.def("pin_pos_backward", &pin_pos_backward);
  m.def("hpwl_forward", &hpwl_forward);
  m.def("move_boundary_forward", &move_boundary_forward);
  m.def("pws_forward", &pws_forward);
  m.def("launch_count", &launch_count);
  m.def("graph_launch", &graph_launch);
  m.def("nesterov_init", &nesterov_init);
  m.def("nesterov_trial", &nesterov_trial);
  m.def("precondition_step_size", &precondition_step_size);
  m.def("iteration_head", &iteration_head, py::arg("state_prev"), py::arg("state_new"), py::arg("sched_prev"),
        py::arg("sched_new"), py::arg("hpwl_k"), py::arg("overflow_k"), py::arg("weights_prev"),
        py::arg("weights_new"), py::arg("base_gamma"), py::arg("total_area"), py::arg("ref_hpwl"), py::arg("lower"),
        py::arg("upper"), py::arg("gate") = py::none());
  m.def("set_trial_gate", &set_trial_gate);
  m.def("trial_gate", &trial_gate, py::arg("gate"), py::arg("accept_prev") = py::none());
  m.def("pack_xy", &pack_xy);
  m.def("objective_finish", &objective_finish);
  m.def("density_overflow_into", &density_overflow_into);
  m.def("density_map_ordered_into", &density_map_ordered_into, py::arg("xy_o"), py::arg("rec4"), py::arg("ratio_o"),
        py::arg("count"), py::arg("init"), py::arg("xl"), py::arg("yl"), py::arg("xh"), py::arg("yh"), py::arg("bsx"),
        py::arg("bsy"), py::arg("nbx"), py::arg("nby"), py::arg("deterministic"), py::arg("scratch"), py::arg("out"),
        py::arg("order") = py::none());
  m.def("build_cell_records", &build_cell_records);
  m.def("gather_order_xy", &gather_order_xy);
  m.def("density_map_ordered_split", &density_map_ordered_split, py::arg("xy_o"), py::arg("rec4"),
        py::arg("ratio_o"), py::arg("num_first"), py::arg("count"), py::arg("init"), py::arg("xl"), py::arg("yl"),
        py::arg("xh"), py::arg("yh"), py::arg("bsx"), py::arg("bsy"), py::arg("nbx"), py::arg("nby"),
        py::arg("deterministic"), py::arg("scratch"), py::arg("out_first"), py::arg("out_all"),
        py::arg("target_area"), py::arg("bin_area"), py::arg("overflow_out"), py::arg("order") = py::none());
  m.def("electric_force_ordered", &electric_force_ordered, py::arg("grad_scale"), py::arg("ex"), py::arg("ey"),
        py::arg("xy_o"), py::arg("rec4"), py::arg("ratio_o"), py::arg("count"), py::arg("xl"), py::arg("yl"),
        py::arg("bsx"), py::arg("bsy"), py::arg("nbx"), py::arg("nby"), py::arg("scale"), py::arg("force_o"),
        py::arg("order") = py::none());
  m.def("assemble_precondition_step", &assemble_precondition_step);
  m.def("plan_net_lanes", &plan_net_lanes, py::arg("netpin_start_cpu"), py::arg("net_order_cpu") = py::none());
  m.def("wa_lanes_forward", &wa_lanes_forward);
  m.def("hpwl_lanes", &hpwl_lanes);
  m.def("node_pin_sum", &node_pin_sum);
  m.def("electric_force_into", &electric_force_into);
  m.def("version", &dp_version);
}
