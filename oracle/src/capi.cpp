// C interface of the oracle.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "../fmt2d_oracle.h"
#include "oracle.hpp"
#include "lsqr.hpp"
#include "smooth.hpp"
#include <map>
#include <memory>
#include <algorithm>

namespace {
struct Handle {
  orc::Model m;
  std::map<int, std::unique_ptr<orc::Source>> src;
  std::vector<double> topo;
  orc::Source& slot(int k) {
    auto& p = src[k];
    if (!p) p.reset(new orc::Source());
    return *p;
  }
};
Handle* H(void* h) { return static_cast<Handle*>(h); }

// invert2d_main.f90:906-931 (interpolate_iface_z on the seafloor interface)
double seafloor_z(const orc::Model& m, double px) {
  const orc::Isec& sf = m.isec[2];
  const int n = sf.nnode;
  if (n < 2) return sf.z[1];
  const double dx = sf.x[2] - sf.x[1];
  const int ixx = (int)std::floor((px - sf.x[1]) / dx) + 1;
  if (ixx < 1) return sf.z[1];
  if (ixx >= n) return sf.z[n];
  const double w = std::min(1.0, std::max(0.0, (px - sf.x[ixx]) / dx));
  return (1.0 - w) * sf.z[ixx] + w * sf.z[ixx + 1];
}
}  // namespace

extern "C" {

void* orc_create(int nx, int nzs, const double* xpos, const double* topo, const double* zrel,
                 const double* vel, double vwater, const double* sed_z, const double* moho_z,
                 int iface_inv) {
  Handle* h = new Handle();
  int nz = 0;
  double zmax = 0;
  std::vector<double> vp;
  orc::resample_smesh(nx, nzs, xpos, topo, zrel, vel, vwater, &nz, vp, &zmax);
  double maxtopo = topo[0];
  for (int i = 1; i < nx; ++i) maxtopo = std::max(maxtopo, topo[i]);
  std::vector<double> iz((size_t)5 * nx);
  for (int i = 0; i < nx; ++i) {
    iz[i] = 0.0;
    iz[(size_t)nx + i] = topo[i];
    iz[(size_t)2 * nx + i] = sed_z[i];
    iz[(size_t)3 * nx + i] = moho_z[i];
    iz[(size_t)4 * nx + i] = zrel[nzs - 1] + maxtopo;
  }
  const double dx = xpos[1] - xpos[0];
  orc::build_model(h->m, nx, nz, dx, xpos, vp.data(), iz.data(), vwater, iface_inv);
  return h;
}

void orc_destroy(void* h) { delete H(h); }

void orc_grid_info(void* h, int* nx, int* nz, double* dx, double* x0) {
  const orc::Grid& g = H(h)->m.grid;
  *nx = g.nx; *nz = g.nz; *dx = g.dx; *x0 = g.x0;
}

void orc_pgrid_velocity(void* h, double* out) {
  const orc::Grid& g = H(h)->m.grid;
  std::copy(g.vel.begin(), g.vel.end(), out);
}

void orc_iface_z(void* h, int iface, double* out) {
  const orc::Isec& is = H(h)->m.isec[iface];
  for (int i = 1; i <= is.nnode; ++i) out[i - 1] = is.z[i];
}

void orc_iface_vel(void* h, int iface, double* vt, double* vb) {
  const orc::Isec& is = H(h)->m.isec[iface];
  for (int i = 1; i <= is.nnode; ++i) { vt[i - 1] = is.vel_top[i]; vb[i - 1] = is.vel_bot[i]; }
}

int orc_region_nnode(void* h, int reg, int* ngnode) {
  const orc::Region& r = H(h)->m.reg[reg];
  if (ngnode) *ngnode = r.ngnode;
  return r.nnode;
}

void orc_region_tables(void* h, int reg, int* i1, int* i2, int* i3, double* x, double* z,
                       double* vel, int* rid) {
  const orc::Region& r = H(h)->m.reg[reg];
  for (int n = 1; n <= r.nnode; ++n) {
    if (i1) i1[n - 1] = r.i1[n];
    if (i2) i2[n - 1] = r.i2[n];
    if (i3) i3[n - 1] = r.i3[n];
    if (x) x[n - 1] = r.x[n];
    if (z) z[n - 1] = r.z[n];
    if (vel) vel[n - 1] = r.vel[n];
  }
  if (rid) std::copy(r.rid.begin(), r.rid.end(), rid);
}

void orc_fully_regular(void* h, uint8_t* out) {
  const orc::Grid& g = H(h)->m.grid;
  std::copy(g.fully_regular.begin(), g.fully_regular.end(), out);
}

void orc_cut_cells(void* h, int iface, int* ncc, int* cx, int* cz) {
  const orc::Isec& is = H(h)->m.isec[iface];
  *ncc = is.n_ccells;
  for (int c = 1; c <= is.n_ccells; ++c) {
    if (cx) cx[c - 1] = is.cc_ix[c];
    if (cz) cz[c - 1] = is.cc_iz[c];
  }
}

int orc_inv_idx(void* h, int* out, int* nvp) {
  const orc::Model& m = H(h)->m;
  std::copy(m.inv_idx.begin(), m.inv_idx.end(), out);
  if (nvp) *nvp = m.n_vel_parms;
  return m.n_inv_parms;
}

int orc_forward(void* h, int slot, double sx, int phase_mask) {
  Handle* hh = H(h);
  orc::Source& s = hh->slot(slot);
  s.x = sx;
  s.z = seafloor_z(hh->m, sx);
  orc::run_forward_source(hh->m, s, phase_mask);
  return 0;
}

double orc_source_z(void* h, int slot) { return H(h)->slot(slot).z; }

int orc_field(void* h, int slot, int tf, double* T, double* gx, double* gz) {
  orc::Source& s = H(h)->slot(slot);
  const orc::TField& t = s.tf[tf];
  const int nn = (int)t.T.size() - 1;
  for (int n = 1; n <= nn; ++n) {
    if (T) T[n - 1] = t.T[n];
    if (gx) gx[n - 1] = t.gx[n];
    if (gz) gz[n - 1] = t.gz[n];
  }
  return t.solved ? nn : -1;
}

int orc_set_field(void* h, int slot, int tf, const double* T, const double* gx,
                  const double* gz) {
  static const int tf_reg[13] = {0, 5, 2, 2, 6, 6, 1, 1, 1, 1, 1, 5, 1};
  Handle* hh = H(h);
  orc::Source& s = hh->slot(slot);
  orc::TField& t = s.tf[tf];
  t.reg = tf_reg[tf];
  const int nn = hh->m.reg[t.reg].nnode;
  t.T.assign(nn + 1, orc::kHugeTime);
  t.gx.assign(nn + 1, 0.0);
  t.gz.assign(nn + 1, 0.0);
  for (int n = 1; n <= nn; ++n) { t.T[n] = T[n - 1]; t.gx[n] = gx[n - 1]; t.gz[n] = gz[n - 1]; }
  t.solved = true;
  return nn;
}

int orc_propagate(void* h, int reg, int* status, double* T, double* gx, double* gz) {
  Handle* hh = H(h);
  orc::Region& r = hh->m.reg[reg];
  for (int n = 1; n <= r.nnode; ++n) {
    r.status[n] = status[n - 1];
    r.T[n] = T[n - 1];
    r.gx[n] = gx[n - 1];
    r.gz[n] = gz[n - 1];
  }
  orc::propagate2d(hh->m, r);
  for (int n = 1; n <= r.nnode; ++n) {
    status[n - 1] = r.status[n];
    T[n - 1] = r.T[n];
    gx[n - 1] = r.gx[n];
    gz[n - 1] = r.gz[n];
  }
  return 0;
}

int orc_trace(void* h, int slot, int phase, double rx, double rz, double* t_out, int* valid,
              int* nnz, int* idx_out, double* val_out, int cap, int* npts, double* pts,
              int pts_cap, int* nsec) {
  Handle* hh = H(h);
  orc::Model& m = hh->m;
  orc::Source& s = hh->slot(slot);
  // invert2d_main.f90:517-537: a receiver above the seafloor is in water.
  const double zsf = seafloor_z(m, rx);
  const bool in_water = rz < zsf;
  double recx = rx, recz = in_water ? zsf : rz, wt = 0.0;
  if (in_water) {
    if (phase == 4 || phase == 5) {
      recx = rx; recz = rz; wt = 0.0;
    } else {
      const int itf = m.path[phase].tf_sequence[m.path[phase].n_tf];
      orc::find_optimal_entry(m, s, itf, rx, rz, recx, recz, wt);
    }
  }
  orc::Ray ray;
  ray.raypath_id = phase;
  orc::trace_ray_from_receiver2d(m, s, recx, recz, ray);
  if (ray.valid) ray.receiver_time = ray.receiver_time + wt;
  *t_out = ray.receiver_time;
  *valid = ray.valid ? 1 : 0;
  *nnz = 0;
  if (npts) *npts = 0;
  if (nsec) *nsec = ray.nsections;
  if (!ray.valid) return 0;
  orc::compute_frechet_for_ray2d(m, s, ray);
  const int k = (int)ray.pdev.size();
  *nnz = k;
  for (int i = 0; i < k && i < cap; ++i) { idx_out[i] = ray.pdev_indx[i]; val_out[i] = ray.pdev[i]; }
  if (npts && pts) {
    int c = 0;
    for (int sct = 1; sct <= ray.nsections; ++sct) {
      const orc::RaySection& rs = ray.sec[sct];
      for (size_t p = 0; p < rs.px.size(); ++p) {
        if (c < pts_cap) { pts[2 * c] = rs.px[p]; pts[2 * c + 1] = rs.pz[p]; }
        ++c;
      }
    }
    *npts = c;
  }
  return 0;
}

int orc_lsqr(void* h, int ndata, int nparm, const int* gindx, const double* gval,
             const int* row_ptr, const double* residual, const double* gtg_diag,
             const double* dm_sum, double eps_min, double wdv, double wdv_iface,
             double w_smooth, double w_smooth_iface, int max_iter, double* dm, int* iters,
             double* rnorm, double* test2) {
  const orc::Model& m = H(h)->m;
  orc::LsqrGeom G;
  G.nx = m.grid.nx; G.nz = m.grid.nz; G.inv_idx = m.inv_idx.data();
  if (m.iface_inv > 0) { G.iface_start = m.iface_start; G.iface_nx = m.isec[m.iface_inv].nnode; }
  orc::LsqrInput in;
  in.ndata = ndata; in.nparm = nparm; in.n_vel_parms = m.n_vel_parms; in.max_iter = max_iter;
  in.gindx = gindx; in.gval = gval; in.row_ptr = row_ptr; in.residual = residual;
  in.gtg_diag = gtg_diag; in.dm_sum = dm_sum; in.eps_min = eps_min; in.wdv = wdv;
  in.wdv_iface = wdv_iface; in.w_smooth = w_smooth; in.w_smooth_iface = w_smooth_iface;
  const orc::LsqrResult r = orc::run_lsqr_laplacian(G, in, dm);
  if (iters) *iters = r.iters;
  if (rnorm) *rnorm = r.rnorm;
  if (test2) *test2 = r.test2;
  return 0;
}

void orc_spmv(int ndata, int nparm, const int* gindx, const double* gval, const int* row_ptr,
              int transpose, const double* x, double* y) {
  if (transpose) orc::sparse_ATx(ndata, nparm, gindx, gval, row_ptr, x, y);
  else orc::sparse_Ax(ndata, nparm, gindx, gval, row_ptr, x, y);
}

void orc_laplacian(void* h, int nparm, const double* vin, double* vout) {
  const orc::Model& m = H(h)->m;
  orc::LsqrGeom G;
  G.nx = m.grid.nx; G.nz = m.grid.nz; G.inv_idx = m.inv_idx.data();
  if (m.iface_inv > 0) { G.iface_start = m.iface_start; G.iface_nx = m.isec[m.iface_inv].nnode; }
  orc::laplacian(G, nparm, vin, vout);
}

// run_lsqr for smooth_type 1, 2 or 3 (inversion2d.f90:6578-7167); the
// Gaussian matrices are built here from corr_x / corr_z / corr_x_iface and
// mvscale as lsqr_inversion2d builds them.
int orc_lsqr_smooth(void* h, int smooth_type, int ndata, int nparm, const int* gindx,
                    const double* gval, const int* row_ptr, const double* residual,
                    const double* gtg_diag, const double* dm_sum, const double* mvscale,
                    double corr_x, double corr_z, double corr_x_iface, double eps_min,
                    double wdv, double wdv_iface, double w_smooth, double w_smooth_iface,
                    int max_iter, double* dm, int* iters, double* rnorm, double* test2) {
  const orc::Model& m = H(h)->m;
  orc::LsqrGeom G;
  G.nx = m.grid.nx; G.nz = m.grid.nz; G.inv_idx = m.inv_idx.data();
  if (m.iface_inv > 0) { G.iface_start = m.iface_start; G.iface_nx = m.isec[m.iface_inv].nnode; }
  orc::LsqrInput in;
  in.ndata = ndata; in.nparm = nparm; in.n_vel_parms = m.n_vel_parms; in.max_iter = max_iter;
  in.gindx = gindx; in.gval = gval; in.row_ptr = row_ptr; in.residual = residual;
  in.gtg_diag = gtg_diag; in.dm_sum = dm_sum; in.eps_min = eps_min; in.wdv = wdv;
  in.wdv_iface = wdv_iface; in.w_smooth = w_smooth; in.w_smooth_iface = w_smooth_iface;
  orc::Csr rh, rv, ri;
  if (smooth_type == 2) orc::gauss_smooth_matrices(m, nparm, corr_x, corr_z, mvscale, rh, rv);
  if (smooth_type >= 2) orc::iface_gauss_smooth_matrix(m, nparm, corr_x_iface, mvscale, ri);
  const orc::LsqrResult r = orc::run_lsqr_general(G, in, smooth_type, &rh, &rv, &ri, dm);
  *iters = r.iters; *rnorm = r.rnorm; *test2 = r.test2;
  return 0;
}

// run_lsqr (smooth_type 1) with the Laplacian on an explicit parameter grid:
// inv_idx over nz x nx (ix fastest, 0 unused) numbers n_vel_parms velocity
// parameters, and iface_nx interface parameters follow them (a coarse
// inversion grid of the projection, or the propagation grid itself).
int orc_lsqr_geom(int gnx, int gnz, const int* inv_idx, int n_vel_parms, int iface_nx,
                  int ndata, int nparm, const int* gindx, const double* gval,
                  const int* row_ptr, const double* residual, const double* gtg_diag,
                  const double* dm_sum, double eps_min, double wdv, double wdv_iface,
                  double w_smooth, double w_smooth_iface, int max_iter, double* dm, int* iters,
                  double* rnorm, double* test2) {
  orc::LsqrGeom G;
  G.nx = gnx; G.nz = gnz; G.inv_idx = inv_idx;
  if (iface_nx > 0) { G.iface_start = n_vel_parms; G.iface_nx = iface_nx; }
  orc::LsqrInput in;
  in.ndata = ndata; in.nparm = nparm; in.n_vel_parms = n_vel_parms; in.max_iter = max_iter;
  in.gindx = gindx; in.gval = gval; in.row_ptr = row_ptr; in.residual = residual;
  in.gtg_diag = gtg_diag; in.dm_sum = dm_sum; in.eps_min = eps_min; in.wdv = wdv;
  in.wdv_iface = wdv_iface; in.w_smooth = w_smooth; in.w_smooth_iface = w_smooth_iface;
  const orc::LsqrResult r = orc::run_lsqr_laplacian(G, in, dm);
  *iters = r.iters; *rnorm = r.rnorm; *test2 = r.test2;
  return 0;
}

// Gaussian smoothing matrices: which 0 = R_h, 1 = R_v (velocity parameters),
// 2 = interface R_h.  Writes the 1-based CSR (rp[nparm+1], col/val up to cap)
// and returns nnz.
int orc_gauss_smooth(void* h, double corr_x, double corr_z, double corr_x_iface,
                     const double* mvscale, int which, int* rp, int* col, double* val, int cap) {
  const orc::Model& m = H(h)->m;
  const int nparm = m.n_inv_parms;
  orc::Csr a, b;
  if (which == 2) orc::iface_gauss_smooth_matrix(m, nparm, corr_x_iface, mvscale, a);
  else orc::gauss_smooth_matrices(m, nparm, corr_x, corr_z, mvscale, a, b);
  const orc::Csr& r = which == 1 ? b : a;
  const int nnz = (int)r.col.size();
  if (rp) std::copy(r.rp.begin(), r.rp.end(), rp);
  for (int k = 0; k < nnz && k < cap; ++k) { col[k] = r.col[k]; val[k] = r.val[k]; }
  return nnz;
}

}  // extern "C"
