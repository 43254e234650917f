// C ABI entry points (include/fmt2d_gpu.h).
#include "../../include/fmt2d_gpu.h"
#include "engine.h"
#include "lsqr.h"
#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

struct fmt2d_ctx {
  std::unique_ptr<fmt2d::Engine> eng;   // null for a host-only context
  std::unique_ptr<fmt2d::Lsqr> lsqr;    // G products and LSQR (device contexts)
  fmt2d::Model model;
  std::string err;
  bool has_model = false;
  bool param_grid = false;              // the LSQR smooths on an explicit parameter grid
  int param_count = 0;                  // its parameters
  bool need_gpu(int& code) {
    if (eng) return true;
    err = "host-only context (device -1): no GPU work possible";
    code = FMT2D_ERR_STATE;
    return false;
  }
  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
};

extern "C" {

int fmt2d_ctx_create(fmt2d_ctx** out, int device) {
  if (!out) return FMT2D_ERR_ARG;
  *out = nullptr;
  if (device == -1) {  // host-only: model build and tables, no device work
    fmt2d_ctx* c = new (std::nothrow) fmt2d_ctx();
    if (!c) return FMT2D_ERR_ARG;
    *out = c;
    return FMT2D_OK;
  }
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return FMT2D_ERR_CUDA;
  fmt2d_ctx* c = new (std::nothrow) fmt2d_ctx();
  if (!c) return FMT2D_ERR_ARG;
  c->eng.reset(new fmt2d::Engine(device));
  c->lsqr.reset(new fmt2d::Lsqr(device, c->eng->stream()));
  if (cudaGetLastError() != cudaSuccess) {
    delete c;
    return FMT2D_ERR_CUDA;
  }
  *out = c;
  return FMT2D_OK;
}

int fmt2d_ctx_destroy(fmt2d_ctx* ctx) {
  delete ctx;
  return FMT2D_OK;
}

int fmt2d_last_error(fmt2d_ctx* ctx, char* buf, int len) {
  if (!ctx || !buf || len <= 0) return FMT2D_ERR_ARG;
  std::strncpy(buf, ctx->err.c_str(), (size_t)len - 1);
  buf[len - 1] = '\0';
  return FMT2D_OK;
}

int fmt2d_upload_model(fmt2d_ctx* ctx, const fmt2d_model_desc* d) {
  if (!ctx || !d) return FMT2D_ERR_ARG;
  if (!d->xpos || !d->topo || !d->zrel || !d->vel || !d->sed_z || !d->moho_z)
    return ctx->fail(FMT2D_ERR_ARG, "null model array");
  if (d->nx < 3 || d->nzs < 2) return ctx->fail(FMT2D_ERR_ARG, "model too small");
  ctx->has_model = false;
  std::string e = fmt2d::build_model(ctx->model, d->nx, d->nzs, d->xpos, d->topo, d->zrel,
                                     d->vel, d->vwater, d->sed_z, d->moho_z, d->iface_inv);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_MODEL, e);
  if (ctx->eng) {
    e = ctx->eng->upload(ctx->model);
    if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
    e = ctx->lsqr->set_geometry(ctx->model);
    if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
  }
  ctx->param_grid = false;
  ctx->has_model = true;
  return FMT2D_OK;
}

int fmt2d_model_info(fmt2d_ctx* ctx, int* nx, int* nz, double* dx, double* x0) {
  if (!ctx) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  const fmt2d::Model& m = ctx->model;
  if (nx) *nx = m.nx;
  if (nz) *nz = m.nz;
  if (dx) *dx = m.dx;
  if (x0) *x0 = m.x0;
  return FMT2D_OK;
}

int fmt2d_model_velocity(fmt2d_ctx* ctx, double* vel) {
  if (!ctx || !vel) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  std::copy(ctx->model.vel.begin(), ctx->model.vel.end(), vel);
  return FMT2D_OK;
}

int fmt2d_model_interface(fmt2d_ctx* ctx, int k, double* z) {
  if (!ctx || !z || k < 1 || k > 5) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  std::copy(ctx->model.ifc[k].z.begin(), ctx->model.ifc[k].z.end(), z);
  return FMT2D_OK;
}

int fmt2d_update_model(fmt2d_ctx* ctx, const double* vel, const double* iface_z) {
  if (!ctx) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  fmt2d::Model next = ctx->model;
  std::string e = fmt2d::update_model(next, vel, iface_z);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_MODEL, e);
  ctx->has_model = false;
  ctx->model = std::move(next);
  if (ctx->eng) {
    e = ctx->eng->upload(ctx->model);
    if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
    e = ctx->lsqr->set_geometry(ctx->model);
    if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
  }
  ctx->param_grid = false;
  ctx->has_model = true;
  return FMT2D_OK;
}

int fmt2d_region_nodes(fmt2d_ctx* ctx, int region, int* nnode, int* i1, int* i2, int* i3) {
  if (!ctx || region < 1 || region > 6) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  const fmt2d::Model& m = ctx->model;
  const fmt2d::Region& r = m.reg[region];
  if (nnode) *nnode = r.nnode;
  if (!i1 && !i2 && !i3) return FMT2D_OK;
  for (int ix = 0; ix < m.nx; ++ix)
    for (int iz = r.r0[ix]; iz <= r.r1[ix]; ++iz) {
      const int id = r.col_base[ix] + (iz - r.r0[ix]);
      if (i1) i1[id] = ix + 1;
      if (i2) i2[id] = iz + 1;
      if (i3) i3[id] = 0;
    }
  for (int k = 0; k < m.nx; ++k) {
    const int a = r.ngnode + k, b = r.ngnode + m.nx + k;
    if (i1) { i1[a] = 0; i1[b] = 0; }
    if (i2) { i2[a] = r.itop; i2[b] = r.ibot; }
    if (i3) { i3[a] = k + 1; i3[b] = k + 1; }
  }
  return FMT2D_OK;
}

int fmt2d_region_geometry(fmt2d_ctx* ctx, int region, double* x, double* z, double* vel) {
  if (!ctx || region < 1 || region > 6) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  const fmt2d::Model& m = ctx->model;
  const fmt2d::Region& r = m.reg[region];
  for (int id = 0; id < r.nnode; ++id) {
    const int s = r.slot_of_node[id];
    if (vel) vel[id] = r.vel64[s];
    if (id < r.ngnode) {
      const int ix = s % r.pitch, iz = s / r.pitch + r.z_lo;
      if (x) x[id] = m.x0 + (double)ix * m.dx;
      if (z) z[id] = (double)iz * m.dx;
    } else {
      const int k = (id - r.ngnode) % m.nx;
      const bool top = id - r.ngnode < m.nx;
      if (x) x[id] = m.xpos[k];
      if (z) z[id] = m.ifc[top ? r.itop : r.ibot].z[k];
    }
  }
  return FMT2D_OK;
}

int fmt2d_gauss_smooth(fmt2d_ctx* ctx, int which, double corr_x, double corr_z,
                       double corr_x_iface, const double* mvscale, int* row_ptr, int* col,
                       double* val, long long* nnz) {
  if (!ctx || !mvscale || !nnz || which < 0 || which > 2) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  std::vector<int> rp, c;
  std::vector<double> v;
  const std::string e = fmt2d::gauss_smooth_csr(ctx->model, which, corr_x, corr_z, corr_x_iface,
                                                mvscale, rp, c, v);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_ARG, e);
  *nnz = (long long)c.size();
  if (row_ptr) std::copy(rp.begin(), rp.end(), row_ptr);
  if (col) std::copy(c.begin(), c.end(), col);
  if (val) std::copy(v.begin(), v.end(), val);
  return FMT2D_OK;
}

int fmt2d_select_data(int npick, const int* phase, const double* obs, const double* t_calc,
                      const int* valid, const int* row_ptr, const int* gindx, const double* gval,
                      int nparm, const double* mvscale, double crit_chi, double wt_psed,
                      double wt_pmp, double wt_pgss, int* ndata, int* row_ptr_out,
                      int* gindx_out, double* gval_out, double* residual, double* data_wt,
                      int* pick_of_row) {
  if (npick < 0 || nparm <= 0 || !ndata || !row_ptr_out) return FMT2D_ERR_ARG;
  if (npick > 0 && (!phase || !obs || !t_calc || !valid || !row_ptr || !mvscale || !residual ||
                    !data_wt || !pick_of_row))
    return FMT2D_ERR_ARG;
  if (npick > 0 && row_ptr[npick] > row_ptr[0] && (!gindx || !gval || !gindx_out || !gval_out))
    return FMT2D_ERR_ARG;
  if (npick > 0 && row_ptr[0] != 1) return FMT2D_ERR_ARG;
  for (int p = 0; p < npick; ++p)
    if (row_ptr[p + 1] < row_ptr[p]) return FMT2D_ERR_ARG;
  const double wt[3] = {wt_psed, wt_pmp, wt_pgss};
  *ndata = fmt2d::select_data(npick, phase, obs, t_calc, valid, row_ptr, gindx, gval, nparm,
                              mvscale, crit_chi, wt, row_ptr_out, gindx_out, gval_out, residual,
                              data_wt, pick_of_row);
  return FMT2D_OK;
}

int fmt2d_projection(fmt2d_ctx* ctx, int kx, int kz, int ki, int* nxc, int* nzc, int* nvp_c,
                     int* npar_c, int* coarse_idx, int* p_row_ptr, int* p_col, double* p_val,
                     long long* p_nnz) {
  if (!ctx || !nxc || !nzc || !nvp_c || !npar_c || !p_nnz) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  std::vector<int> cidx, rp, col;
  std::vector<double> val;
  const std::string e = fmt2d::projection(ctx->model, kx, kz, ki, cidx, *nxc, *nzc, *nvp_c,
                                          *npar_c, rp, col, val);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_ARG, e);
  *p_nnz = (long long)col.size();
  if (coarse_idx) std::copy(cidx.begin(), cidx.end(), coarse_idx);
  if (p_row_ptr) std::copy(rp.begin(), rp.end(), p_row_ptr);
  if (p_col) std::copy(col.begin(), col.end(), p_col);
  if (p_val) std::copy(val.begin(), val.end(), p_val);
  return FMT2D_OK;
}

int fmt2d_project_rows(int ndata, const int* row_ptr, const int* gindx, const double* gval,
                       int nfine, const int* p_row_ptr, const int* p_col, const double* p_val,
                       int* row_ptr_out, int* gindx_out, double* gval_out, long long* nnz) {
  if (ndata < 0 || nfine <= 0 || !row_ptr || !p_row_ptr || !nnz) return FMT2D_ERR_ARG;
  if (row_ptr[0] != 1 || p_row_ptr[0] != 1) return FMT2D_ERR_ARG;
  for (int i = 0; i < ndata; ++i)
    if (row_ptr[i + 1] < row_ptr[i]) return FMT2D_ERR_ARG;
  for (int f = 0; f < nfine; ++f)
    if (p_row_ptr[f + 1] < p_row_ptr[f]) return FMT2D_ERR_ARG;
  if (row_ptr[ndata] > 1 && (!gindx || !gval)) return FMT2D_ERR_ARG;
  if (p_row_ptr[nfine] > 1 && (!p_col || !p_val)) return FMT2D_ERR_ARG;
  std::vector<int> rp, col;
  std::vector<double> val;
  fmt2d::project_rows(ndata, row_ptr, gindx, gval, nfine, p_row_ptr, p_col, p_val, rp, col, val);
  *nnz = (long long)col.size();
  if (row_ptr_out) std::copy(rp.begin(), rp.end(), row_ptr_out);
  if (gindx_out) std::copy(col.begin(), col.end(), gindx_out);
  if (gval_out) std::copy(val.begin(), val.end(), gval_out);
  return FMT2D_OK;
}

int fmt2d_inv_index(fmt2d_ctx* ctx, int* inv_idx, int* nvp, int* npar) {
  if (!ctx) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  const fmt2d::Model& m = ctx->model;
  if (inv_idx) std::memcpy(inv_idx, m.inv_idx.data(), m.inv_idx.size() * sizeof(int));
  if (nvp) *nvp = m.n_vel_parms;
  if (npar) *npar = m.n_inv_parms;
  return FMT2D_OK;
}

int fmt2d_forward(fmt2d_ctx* ctx, const double* src_x, int nsrc, int phase_mask) {
  if (!ctx || !src_x || nsrc <= 0 || (phase_mask & ~31) || !phase_mask) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const std::string e = ctx->eng->forward(src_x, nsrc, phase_mask);
  if (!e.empty())
    return ctx->fail(ctx->eng->not_converged() ? FMT2D_ERR_CONVERGE : FMT2D_ERR_CUDA, e);
  return FMT2D_OK;
}

int fmt2d_forward_batch(fmt2d_ctx* const* ctxs, int n, const double* const* src_x,
                        const int* nsrc, const int* phase_mask, int* status) {
  if (!ctxs || n <= 0 || !src_x || !nsrc || !phase_mask) return FMT2D_ERR_ARG;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j)
      if (ctxs[i] == ctxs[j]) return FMT2D_ERR_ARG;   // one forward per context
  std::vector<int> rc(n, FMT2D_OK);
  auto run = [&](int i) { rc[i] = fmt2d_forward(ctxs[i], src_x[i], nsrc[i], phase_mask[i]); };
  std::vector<std::thread> th;
  th.reserve(n > 1 ? n - 1 : 0);
  for (int i = 1; i < n; ++i) th.emplace_back(run, i);
  run(0);
  for (std::thread& t : th) t.join();
  int first = FMT2D_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = rc[i];
    if (first == FMT2D_OK && rc[i] != FMT2D_OK) first = rc[i];
  }
  return first;
}

int fmt2d_get_field(fmt2d_ctx* ctx, int src, int tf, double* T, double* gx, double* gz) {
  if (!ctx) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const std::string e = ctx->eng->get_field(src, tf, T, gx, gz);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_ARG, e);
  return FMT2D_OK;
}

int fmt2d_get_field_device(fmt2d_ctx* ctx, int src, int tf, double* T, double* gx, double* gz) {
  if (!ctx) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const std::string e = ctx->eng->get_field_device(src, tf, T, gx, gz);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_ARG, e);
  return FMT2D_OK;
}

int fmt2d_stats(fmt2d_ctx* ctx, double* values, int n) {
  if (!ctx || !values || n < 0) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const fmt2d::SolveStats& s = ctx->eng->stats();
  const double v[FMT2D_N_STATS] = {
      (double)s.rounds,    (double)s.batches, (double)s.final_passes, (double)s.passed,
      s.round_ms,          (double)s.launches, (double)s.nodes,       (double)s.evals,
      (double)s.steps_sum, (double)s.capped,  (double)s.writes,       (double)s.unsettled,
      s.cycles[0],         s.cycles[1],       s.cycles[2],            s.cycles[3],
      s.cycles[4],         (double)s.cut_evals, (double)s.cut_steps};
  for (int i = 0; i < n && i < FMT2D_N_STATS; ++i) values[i] = v[i];
  return FMT2D_OK;
}

int fmt2d_trace(fmt2d_ctx* ctx, const int* src, const int* phase, const double* rx,
                const double* rz, int npick, double* t_calc, int* valid, long long* nnz) {
  if (!ctx || npick < 0 || (npick > 0 && (!src || !phase || !rx || !rz || !t_calc || !valid)))
    return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  if (ctx->eng->nsrc() == 0) return ctx->fail(FMT2D_ERR_STATE, "no forward solved");
  const std::string e = ctx->eng->trace(src, phase, rx, rz, npick, t_calc, valid, nnz);
  if (!e.empty())
    return ctx->fail(e.find("range") != std::string::npos ? FMT2D_ERR_ARG : FMT2D_ERR_CUDA, e);
  return FMT2D_OK;
}

int fmt2d_misfit_gradient(fmt2d_ctx* ctx, const int* src, const int* phase, const double* rx,
                          const double* rz, const double* t_obs, const double* sigma, int npick,
                          double* misfit, double* t_calc, int* valid, double* grad_slow,
                          double* grad_vel, double* grad_iface, double* info) {
  if (!ctx || !misfit || npick < 0 ||
      (npick > 0 && (!src || !phase || !rx || !rz || !t_obs || !sigma || !t_calc || !valid)))
    return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  if (ctx->eng->nsrc() == 0) return ctx->fail(FMT2D_ERR_STATE, "no forward solved");
  const fmt2d::Model& m = ctx->eng->model();
  const size_t nn = (size_t)m.nx * m.nz;
  std::vector<double> gv((grad_slow || grad_vel) ? nn : 0);
  const std::string e = ctx->eng->misfit_gradient(src, phase, rx, rz, t_obs, sigma, npick, misfit,
                                                  t_calc, valid, gv.empty() ? nullptr : gv.data(),
                                                  grad_iface, info);
  if (!e.empty()) {
    const bool arg = e.find("range") != std::string::npos || e.find("phases") != std::string::npos ||
                     e.find("sigma") != std::string::npos;
    const bool state = e.find("not solved") != std::string::npos ||
                       e.find("missing") != std::string::npos;
    return ctx->fail(arg ? FMT2D_ERR_ARG : state ? FMT2D_ERR_STATE : FMT2D_ERR_CUDA, e);
  }
  if (grad_vel) std::copy(gv.begin(), gv.end(), grad_vel);
  // s = 1/v: dJ/ds = -v^2 dJ/dv
  if (grad_slow)
    for (size_t i = 0; i < nn; ++i) grad_slow[i] = -(m.vel[i] * m.vel[i]) * gv[i];
  return FMT2D_OK;
}

int fmt2d_trace_times(fmt2d_ctx* ctx, const int* src, const int* phase, const double* rx,
                      const double* rz, int npick, double* t_calc, int* valid) {
  if (!ctx || npick < 0 || (npick > 0 && (!src || !phase || !rx || !rz || !t_calc || !valid)))
    return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  if (ctx->eng->nsrc() == 0) return ctx->fail(FMT2D_ERR_STATE, "no forward solved");
  const std::string e =
      ctx->eng->trace(src, phase, rx, rz, npick, t_calc, valid, nullptr, /*rows=*/false);
  if (!e.empty())
    return ctx->fail(e.find("range") != std::string::npos ? FMT2D_ERR_ARG : FMT2D_ERR_CUDA, e);
  return FMT2D_OK;
}

int fmt2d_frechet_rows(fmt2d_ctx* ctx, int* row_ptr, int* gindx, double* gval, int index_base) {
  if (!ctx || (index_base != 0 && index_base != 1)) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const std::string e = ctx->eng->frechet_rows(row_ptr, gindx, gval, index_base);
  if (!e.empty())
    return ctx->fail(e.find("no picks") != std::string::npos ? FMT2D_ERR_STATE : FMT2D_ERR_CUDA,
                     e);
  return FMT2D_OK;
}

int fmt2d_trace_entries(fmt2d_ctx* ctx, double* water_time, double* entry_x, double* entry_z) {
  if (!ctx) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const std::string e = ctx->eng->trace_entries(water_time, entry_x, entry_z);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_STATE, e);
  return FMT2D_OK;
}

int fmt2d_set_frechet(fmt2d_ctx* ctx, int ndata, int nparm, const int* row_ptr,
                      const int* gindx, const double* gval, int index_base) {
  if (!ctx || !row_ptr || ndata < 0 || nparm <= 0 || (index_base != 0 && index_base != 1))
    return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  const std::string e = ctx->lsqr->set_matrix(ndata, nparm, row_ptr, gindx, gval, index_base);
  if (!e.empty()) return ctx->fail(e.find("CUDA") != std::string::npos ||
                                       e.find("allocation") != std::string::npos
                                       ? FMT2D_ERR_CUDA : FMT2D_ERR_ARG, e);
  return FMT2D_OK;
}

int fmt2d_spmv(fmt2d_ctx* ctx, int transpose, const double* x, double* y) {
  if (!ctx || !x || !y) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (ctx->lsqr->nparm() == 0) return ctx->fail(FMT2D_ERR_STATE, "no matrix set");
  const std::string e = ctx->lsqr->spmv(transpose != 0, x, y);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
  return FMT2D_OK;
}

int fmt2d_gtg_diag(fmt2d_ctx* ctx, double* gtg) {
  if (!ctx || !gtg) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (ctx->lsqr->nparm() == 0) return ctx->fail(FMT2D_ERR_STATE, "no matrix set");
  const std::string e = ctx->lsqr->gtg_diag(gtg);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
  return FMT2D_OK;
}

int fmt2d_set_smoothing(fmt2d_ctx* ctx, double corr_x, double corr_z, double corr_x_iface,
                        const double* mvscale) {
  if (!ctx || !mvscale) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  const std::string e = ctx->lsqr->set_smoothing(ctx->model, corr_x, corr_z, corr_x_iface, mvscale);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_ARG, e);
  return FMT2D_OK;
}

int fmt2d_set_param_grid(fmt2d_ctx* ctx, int nxc, int nzc, const int* coarse_idx,
                         int n_vel_parms, int iface_nodes) {
  if (!ctx) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  const std::string e =
      coarse_idx ? ctx->lsqr->set_param_grid(nxc, nzc, coarse_idx, n_vel_parms, iface_nodes)
                 : ctx->lsqr->set_geometry(ctx->model);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_ARG, e);
  ctx->param_grid = coarse_idx != nullptr;
  ctx->param_count = n_vel_parms + iface_nodes;
  return FMT2D_OK;
}

int fmt2d_lsqr(fmt2d_ctx* ctx, const fmt2d_lsqr_params* p, const double* residual,
               const double* gtg_diag, const double* dm_sum, double* dm, int* iters, double* rnorm,
               double* bnorm, double* test2) {
  if (!ctx || !p || !dm) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  if (ctx->lsqr->nparm() == 0) return ctx->fail(FMT2D_ERR_STATE, "no matrix set");
  if (p->smooth_type < 1 || p->smooth_type > 3)
    return ctx->fail(FMT2D_ERR_ARG, "smooth_type must be 1, 2 or 3");
  if (p->max_iter < 1) return ctx->fail(FMT2D_ERR_ARG, "max_iter must be >= 1");
  if (ctx->lsqr->nparm() != (ctx->param_grid ? ctx->param_count : ctx->model.n_inv_parms))
    return ctx->fail(FMT2D_ERR_STATE, "G columns differ from the inversion parameters");
  fmt2d::LsqrParams q;
  q.smooth_type = p->smooth_type;
  q.max_iter = p->max_iter;
  q.wdv = p->wdv;
  q.wdv_iface = p->wdv_iface;
  q.w_smooth = p->w_smooth;
  q.w_smooth_iface = p->w_smooth_iface;
  q.eps_min = p->eps_min;
  fmt2d::LsqrOut o;
  const std::string e = ctx->lsqr->solve(q, residual, gtg_diag, dm_sum, dm, &o);
  if (!e.empty()) return ctx->fail(FMT2D_ERR_CUDA, e);
  if (iters) *iters = o.iters;
  if (rnorm) *rnorm = o.rnorm;
  if (bnorm) *bnorm = o.bnorm;
  if (test2) *test2 = o.test2;
  return FMT2D_OK;
}

int fmt2d_lsqr_noalloc(fmt2d_ctx* ctx, const fmt2d_lsqr_params* p, const double* residual,
                       const double* gtg_diag, const double* dm_sum, double* dm, int* iters,
                       double* rnorm, double* bnorm, double* test2) {
  if (!ctx || !p || !dm) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  if (ctx->lsqr->nparm() == 0) return ctx->fail(FMT2D_ERR_STATE, "no matrix set");
  if (p->smooth_type != 1) return ctx->fail(FMT2D_ERR_ARG, "smooth_type must be 1 (Laplacian)");
  if (p->max_iter < 1) return ctx->fail(FMT2D_ERR_ARG, "max_iter must be >= 1");
  if (ctx->lsqr->nparm() != (ctx->param_grid ? ctx->param_count : ctx->model.n_inv_parms))
    return ctx->fail(FMT2D_ERR_STATE, "G columns differ from the inversion parameters");
  fmt2d::LsqrParams q;
  q.smooth_type = p->smooth_type;
  q.max_iter = p->max_iter;
  q.wdv = p->wdv;
  q.wdv_iface = p->wdv_iface;
  q.w_smooth = p->w_smooth;
  q.w_smooth_iface = p->w_smooth_iface;
  q.eps_min = p->eps_min;
  fmt2d::LsqrOut o;
  const std::string e = ctx->lsqr->solve_noalloc(q, residual, gtg_diag, dm_sum, dm, &o);
  if (!e.empty())
    return ctx->fail(e.find("too large") != std::string::npos ||
                             e.find("null") != std::string::npos ? FMT2D_ERR_ARG : FMT2D_ERR_CUDA,
                     e);
  if (iters) *iters = o.iters;
  if (rnorm) *rnorm = o.rnorm;
  if (bnorm) *bnorm = o.bnorm;
  if (test2) *test2 = o.test2;
  return FMT2D_OK;
}

int fmt2d_lsqr_stats(fmt2d_ctx* ctx, double* ms, int* launches) {
  if (!ctx) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  if (ms) *ms = ctx->lsqr->last_ms();
  if (launches) *launches = ctx->lsqr->last_launches();
  return FMT2D_OK;
}

int fmt2d_set_schedule(fmt2d_ctx* ctx, double window_cells, int max_passes,
                       long long max_steps) {
  if (!ctx || !(window_cells >= 0.0) || window_cells > 1.0e6 || max_passes < 1 || max_passes > 64 ||
      max_steps < 0)
    return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  ctx->eng->window_cells = window_cells;
  ctx->eng->max_passes = max_passes;
  ctx->eng->max_steps = max_steps > 0 ? max_steps : fmt2d::Engine::kDefaultMaxSteps;
  return FMT2D_OK;
}

int fmt2d_set_iface_window(fmt2d_ctx* ctx, double cells) {
  if (!ctx || !(cells >= 0.0) || cells > 1.0e6) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  ctx->eng->iface_window_cells = cells;
  return FMT2D_OK;
}

int fmt2d_set_solve_threads(fmt2d_ctx* ctx, int threads) {
  if (!ctx) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  int n = 0;
  const int* sizes = fmt2d::e64_solve_sizes(&n);
  bool ok = threads == 0;
  for (int k = 0; k < n; ++k) ok = ok || threads == sizes[k];
  if (!ok) return ctx->fail(FMT2D_ERR_ARG, "solve block size must be 0 or one of 256, 384, 512");
  ctx->eng->solve_threads = threads;
  return FMT2D_OK;
}

int fmt2d_autotune(fmt2d_ctx* ctx, const double* src_x, int nsrc, int phase_mask, int* threads,
                   double* ms) {
  if (!ctx || !src_x || nsrc <= 0 || (phase_mask & ~31) || !phase_mask) return FMT2D_ERR_ARG;
  if (!ctx->has_model) return ctx->fail(FMT2D_ERR_STATE, "no model uploaded");
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  int n = 0;
  const int* sizes = fmt2d::e64_solve_sizes(&n);
  // one untimed forward (field stores and solver scratch are allocated once)
  std::string e = ctx->eng->forward(src_x, nsrc, phase_mask);
  if (!e.empty())
    return ctx->fail(ctx->eng->not_converged() ? FMT2D_ERR_CONVERGE : FMT2D_ERR_CUDA, e);
  int best = 0;
  double best_ms = 1.0e300;
  for (int k = 0; k < n; ++k) {
    ctx->eng->solve_threads = sizes[k];
    const auto t0 = std::chrono::steady_clock::now();
    e = ctx->eng->forward(src_x, nsrc, phase_mask);
    const double t = std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t0).count();
    if (!e.empty())
      return ctx->fail(ctx->eng->not_converged() ? FMT2D_ERR_CONVERGE : FMT2D_ERR_CUDA, e);
    if (ms) ms[k] = t;
    if (t < best_ms) { best_ms = t; best = sizes[k]; }
  }
  ctx->eng->solve_threads = best;
  if (threads) *threads = best;
  return FMT2D_OK;
}

int fmt2d_stream(fmt2d_ctx* ctx, void** stream) {
  if (!ctx || !stream) return FMT2D_ERR_ARG;
  int code = 0;
  if (!ctx->need_gpu(code)) return code;
  *stream = (void*)ctx->eng->stream();
  return FMT2D_OK;
}

}  // extern "C"
