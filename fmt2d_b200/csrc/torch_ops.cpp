// PyTorch operators on the C ABI (include/fmt2d_gpu.h): torch.ops.fmt2d.*
//
// The Python scripts of the reference reach the forward, the ray backtrace
// and the LSQR through these operators with CUDA tensors.  A context is the
// fmt2d_ctx* of the C ABI passed as an int64 (Fmt2d.h.value on the Python
// side).  Every operator orders the context's stream after the caller's
// current CUDA stream (an event, no host wait) before it reads the caller's
// tensors, and its outputs are complete when it returns (each C ABI call
// finishes its own work before returning).  Errors raise with the library's
// message.
#include <torch/library.h>
#include <ATen/ATen.h>
#include <ATen/cuda/CUDAContext.h>
#include <cuda_runtime.h>

#include <string>
#include <tuple>
#include <vector>

#include "../../include/fmt2d_gpu.h"

namespace {

fmt2d_ctx* ctx_of(int64_t h) {
  TORCH_CHECK(h != 0, "fmt2d: null context");
  return reinterpret_cast<fmt2d_ctx*>(static_cast<intptr_t>(h));
}

void check(fmt2d_ctx* c, int rc, const char* what) {
  if (rc == FMT2D_OK) return;
  char buf[512] = {0};
  fmt2d_last_error(c, buf, sizeof(buf));
  TORCH_CHECK(false, what, " failed (", rc, "): ", buf);
}

// Make the context's stream wait for the work queued so far on the caller's
// current stream of `device`.
void after_current_stream(fmt2d_ctx* c, int device) {
  void* s = nullptr;
  check(c, fmt2d_stream(c, &s), "fmt2d_stream");
  const cudaStream_t cur = at::cuda::getCurrentCUDAStream(device).stream();
  cudaEvent_t ev;
  TORCH_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess,
              "fmt2d: cudaEventCreate failed");
  cudaEventRecord(ev, cur);
  cudaStreamWaitEvent(static_cast<cudaStream_t>(s), ev, 0);
  cudaEventDestroy(ev);
}

// The CUDA device outputs are placed on: the caller's current device, which
// must be the context's (Fmt2d(device) makes it current).
int device_of_ctx(fmt2d_ctx* c) {
  (void)c;
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

at::Tensor host_f64(const at::Tensor& t, const char* name) {
  TORCH_CHECK(t.scalar_type() == at::kDouble, "fmt2d: ", name, " must be float64");
  return t.to(at::kCPU).contiguous();
}

at::Tensor host_i32(const at::Tensor& t, const char* name) {
  TORCH_CHECK(t.scalar_type() == at::kInt, "fmt2d: ", name, " must be int32");
  return t.to(at::kCPU).contiguous();
}

}  // namespace

namespace fmt2d_ops {

// run_forward2d's stage loop for every source (fmt2d_forward); src_x: float64
// OBS x positions (CPU or CUDA).
void forward(int64_t ctx, const at::Tensor& src_x, int64_t phase_mask) {
  fmt2d_ctx* c = ctx_of(ctx);
  if (src_x.is_cuda()) after_current_stream(c, src_x.get_device());
  const at::Tensor x = host_f64(src_x, "src_x");
  check(c, fmt2d_forward(c, x.data_ptr<double>(), (int)x.numel(), (int)phase_mask),
        "fmt2d_forward");
}

// Time field tf of source src in its region's node order as CUDA float64
// tensors (T, dT/dx, dT/dz) on the context's device (fmt2d_get_field_device).
std::tuple<at::Tensor, at::Tensor, at::Tensor> field(int64_t ctx, int64_t src, int64_t tf) {
  static const int kRegion[13] = {0, 5, 2, 2, 6, 6, 1, 1, 1, 1, 1, 5, 1};
  fmt2d_ctx* c = ctx_of(ctx);
  TORCH_CHECK(tf >= 1 && tf <= 12, "fmt2d: tf must be 1..12");
  int n = 0;
  check(c, fmt2d_region_nodes(c, kRegion[tf], &n, nullptr, nullptr, nullptr),
        "fmt2d_region_nodes");
  const int dev = device_of_ctx(c);
  auto opt = at::TensorOptions().dtype(at::kDouble).device(at::kCUDA, dev);
  at::Tensor T = at::empty({n}, opt), gx = at::empty({n}, opt), gz = at::empty({n}, opt);
  after_current_stream(c, dev);
  check(c, fmt2d_get_field_device(c, (int)src, (int)tf, T.data_ptr<double>(),
                                  gx.data_ptr<double>(), gz.data_ptr<double>()),
        "fmt2d_get_field_device");
  return {T, gx, gz};
}

// Ray backtrace and Frechet rows of a batch of picks on the last forward's
// fields (fmt2d_trace): src, phase int32; rx, rz float64.  Returns (t_calc,
// valid as int32, nnz) on the device of rx.
std::tuple<at::Tensor, at::Tensor, int64_t> trace(int64_t ctx, const at::Tensor& src,
                                                   const at::Tensor& phase, const at::Tensor& rx,
                                                   const at::Tensor& rz) {
  fmt2d_ctx* c = ctx_of(ctx);
  if (rx.is_cuda()) after_current_stream(c, rx.get_device());
  const at::Tensor s = host_i32(src, "src"), p = host_i32(phase, "phase");
  const at::Tensor x = host_f64(rx, "rx"), z = host_f64(rz, "rz");
  const int64_t n = s.numel();
  TORCH_CHECK(p.numel() == n && x.numel() == n && z.numel() == n,
              "fmt2d: src, phase, rx, rz must have one entry per pick");
  at::Tensor t = at::empty({n}, at::kDouble), v = at::empty({n}, at::kInt);
  long long nnz = 0;
  check(c, fmt2d_trace(c, s.data_ptr<int>(), p.data_ptr<int>(), x.data_ptr<double>(),
                       z.data_ptr<double>(), (int)n, t.data_ptr<double>(), v.data_ptr<int>(), &nnz),
        "fmt2d_trace");
  return {t.to(rx.device()), v.to(rx.device()), (int64_t)nnz};
}

// CSR (row_ptr, gindx, gval) of the last trace over its npick picks
// (fmt2d_frechet_rows); index_base 1 gives read_frechet_data2d's layout.
std::tuple<at::Tensor, at::Tensor, at::Tensor> frechet_rows(int64_t ctx, int64_t npick,
                                                            int64_t nnz, int64_t index_base) {
  fmt2d_ctx* c = ctx_of(ctx);
  at::Tensor rp = at::empty({npick + 1}, at::kInt);
  at::Tensor gi = at::empty({std::max<int64_t>(nnz, 1)}, at::kInt);
  at::Tensor gv = at::empty({std::max<int64_t>(nnz, 1)}, at::kDouble);
  check(c, fmt2d_frechet_rows(c, rp.data_ptr<int>(), gi.data_ptr<int>(), gv.data_ptr<double>(),
                              (int)index_base),
        "fmt2d_frechet_rows");
  return {rp, gi.narrow(0, 0, nnz), gv.narrow(0, 0, nnz)};
}

// run_lsqr on the context's G (fmt2d_lsqr).  gtg_diag and dm_sum may be
// empty tensors (computed from G / zeros).  Returns (dm on the device of
// residual, iterations, rnorm, bnorm, test2).
std::tuple<at::Tensor, int64_t, double, double, double> lsqr(
    int64_t ctx, const at::Tensor& residual, const at::Tensor& gtg_diag,
    const at::Tensor& dm_sum, int64_t smooth_type, int64_t max_iter, double wdv,
    double wdv_iface, double w_smooth, double w_smooth_iface, double eps_min) {
  fmt2d_ctx* c = ctx_of(ctx);
  if (residual.is_cuda()) after_current_stream(c, residual.get_device());
  const at::Tensor r = host_f64(residual, "residual");
  const bool has_g = gtg_diag.numel() > 0, has_s = dm_sum.numel() > 0;
  const at::Tensor g = has_g ? host_f64(gtg_diag, "gtg_diag") : at::Tensor();
  const at::Tensor s = has_s ? host_f64(dm_sum, "dm_sum") : at::Tensor();
  int nvp = 0, np = 0;
  // nparm: the model's inversion parameters (fmt2d_lsqr requires G to have them)
  check(c, fmt2d_inv_index(c, nullptr, &nvp, &np), "fmt2d_inv_index");
  TORCH_CHECK(!has_g || g.numel() == np, "fmt2d: gtg_diag needs nparm entries");
  TORCH_CHECK(!has_s || s.numel() == np, "fmt2d: dm_sum needs nparm entries");
  at::Tensor dm = at::zeros({np}, at::kDouble);
  fmt2d_lsqr_params p;
  p.smooth_type = (int)smooth_type;
  p.max_iter = (int)max_iter;
  p.wdv = wdv;
  p.wdv_iface = wdv_iface;
  p.w_smooth = w_smooth;
  p.w_smooth_iface = w_smooth_iface;
  p.eps_min = eps_min;
  int it = 0;
  double rn = 0, bn = 0, t2 = 0;
  check(c, fmt2d_lsqr(c, &p, r.data_ptr<double>(), has_g ? g.data_ptr<double>() : nullptr,
                      has_s ? s.data_ptr<double>() : nullptr, dm.data_ptr<double>(), &it, &rn,
                      &bn, &t2),
        "fmt2d_lsqr");
  return {dm.to(residual.device()), (int64_t)it, rn, bn, t2};
}

}  // namespace fmt2d_ops

TORCH_LIBRARY(fmt2d, m) {
  m.def("forward(int ctx, Tensor src_x, int phase_mask) -> ()", &fmt2d_ops::forward);
  m.def("field(int ctx, int src, int tf) -> (Tensor, Tensor, Tensor)", &fmt2d_ops::field);
  m.def("trace(int ctx, Tensor src, Tensor phase, Tensor rx, Tensor rz) -> (Tensor, Tensor, int)",
        &fmt2d_ops::trace);
  m.def("frechet_rows(int ctx, int npick, int nnz, int index_base) -> (Tensor, Tensor, Tensor)",
        &fmt2d_ops::frechet_rows);
  m.def("lsqr(int ctx, Tensor residual, Tensor gtg_diag, Tensor dm_sum, int smooth_type, "
        "int max_iter, float wdv, float wdv_iface, float w_smooth, float w_smooth_iface, "
        "float eps_min) -> (Tensor, int, float, float, float)",
        &fmt2d_ops::lsqr);
}
