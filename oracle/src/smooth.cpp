// Oracle Gaussian smoothing matrices of the smooth_type 2/3 LSQR layouts.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <algorithm>
#include <cmath>
#include "oracle.hpp"
#include "smooth.hpp"

namespace orc {

namespace {

// Counts per row, then 1-based row pointers (rows of parameters the loop
// does not visit stay empty).
void counts_to_rowptr(std::vector<int>& rp, int nparm) {
  rp[0] = 1;
  for (int i = 1; i <= nparm; ++i) rp[i] = rp[i - 1] + rp[i];
}

}  // namespace

// build_gauss_smooth_matrix (src/inversion2d.f90:1252-1402): per velocity
// parameter of the (propagation) grid, R_h holds exp(-dx^2/cx^2) * mvscale(j)
// for the active nodes of its row within 3 cx (+1 column) and R_v the same
// along its column within 3 cz, each row followed by its diagonal
// -sum(beta) * mvscale(i).
void gauss_smooth_matrices(const Model& m, int nparm, double corr_x, double corr_z,
                           const double* mvscale, Csr& rh, Csr& rv) {
  const Grid& g = m.grid;
  rh.rp.assign(nparm + 1, 0);
  rv.rp.assign(nparm + 1, 0);
  const int kx_min = -(int)(3.0 * corr_x / g.dx) - 1;
  const int kx_max = (int)(3.0 * corr_x / g.dx) + 1;
  auto idx_at = [&](int ix, int iz) { return m.inv_idx[g.g(ix, iz)]; };
  // pass 1: counts
  for (int iz = 1; iz <= g.nz; ++iz)
    for (int ix = 1; ix <= g.nx; ++ix) {
      const int idx = idx_at(ix, iz);
      if (idx <= 0) continue;
      int n = 1;
      for (int jx = std::max(1, ix + kx_min); jx <= std::min(g.nx, ix + kx_max); ++jx)
        if (jx != ix && idx_at(jx, iz) > 0) ++n;
      rh.rp[idx] = n;
      n = 1;
      for (int jz = 1; jz <= g.nz; ++jz) {
        if (jz == iz) continue;
        if (std::fabs(g.z[jz] - g.z[iz]) > 3.0 * corr_z) continue;
        if (idx_at(ix, jz) > 0) ++n;
      }
      rv.rp[idx] = n;
    }
  counts_to_rowptr(rh.rp, nparm);
  counts_to_rowptr(rv.rp, nparm);
  rh.col.assign(rh.rp[nparm] - 1, 0);
  rh.val.assign(rh.rp[nparm] - 1, 0.0);
  rv.col.assign(rv.rp[nparm] - 1, 0);
  rv.val.assign(rv.rp[nparm] - 1, 0.0);
  // pass 2: values
  for (int iz = 1; iz <= g.nz; ++iz)
    for (int ix = 1; ix <= g.nx; ++ix) {
      const int idx = idx_at(ix, iz);
      if (idx <= 0) continue;
      int k = rh.rp[idx - 1] - 1;
      double bsum = 0.0;
      for (int jx = std::max(1, ix + kx_min); jx <= std::min(g.nx, ix + kx_max); ++jx) {
        if (jx == ix) continue;
        const int jdx = idx_at(jx, iz);
        if (jdx <= 0) continue;
        const double d = g.x[jx] - g.x[ix];
        const double beta = std::exp(-(d * d) / (corr_x * corr_x));
        bsum = bsum + beta;
        rh.col[k] = jdx;
        rh.val[k] = beta * mvscale[jdx - 1];
        ++k;
      }
      rh.col[k] = idx;
      rh.val[k] = -bsum * mvscale[idx - 1];
      k = rv.rp[idx - 1] - 1;
      bsum = 0.0;
      for (int jz = 1; jz <= g.nz; ++jz) {
        if (jz == iz) continue;
        const double d = g.z[jz] - g.z[iz];
        if (std::fabs(d) > 3.0 * corr_z) continue;
        const int jdx = idx_at(ix, jz);
        if (jdx <= 0) continue;
        const double beta = std::exp(-(d * d) / (corr_z * corr_z));
        bsum = bsum + beta;
        rv.col[k] = jdx;
        rv.val[k] = beta * mvscale[jdx - 1];
        ++k;
      }
      rv.col[k] = idx;
      rv.val[k] = -bsum * mvscale[idx - 1];
    }
}

// build_iface_gauss_smooth_matrix (src/inversion2d.f90:1524-1616): the same
// 1-D Gaussian over the nodes of the inverted interface (parameters
// start_index + 1 .. start_index + nx), within 3 cx (+1 node).
void iface_gauss_smooth_matrix(const Model& m, int nparm, double corr_x_iface,
                               const double* mvscale, Csr& ri) {
  ri.rp.assign(nparm + 1, 0);
  ri.col.clear();
  ri.val.clear();
  if (corr_x_iface <= 0.0 || m.iface_inv <= 0) {
    counts_to_rowptr(ri.rp, nparm);
    return;
  }
  const int nx_if = std::min(m.isec[m.iface_inv].nnode, (int)m.vgx.size() - 1);
  const std::vector<double>& x = m.vgx;   // interface node x (1-based): velocity-grid x
  const double dx_if = x[2] - x[1];
  const int kx_min = -(int)(3.0 * corr_x_iface / dx_if) - 1;
  const int kx_max = (int)(3.0 * corr_x_iface / dx_if) + 1;
  const int start = m.iface_start;
  for (int ix = 1; ix <= nx_if; ++ix) {
    const int idx = start + ix;
    if (idx < 1 || idx > nparm) continue;
    int n = 1;
    for (int jx = std::max(1, ix + kx_min); jx <= std::min(nx_if, ix + kx_max); ++jx) {
      const int jdx = start + jx;
      if (jx != ix && jdx >= 1 && jdx <= nparm) ++n;
    }
    ri.rp[idx] = n;
  }
  counts_to_rowptr(ri.rp, nparm);
  ri.col.assign(ri.rp[nparm] - 1, 0);
  ri.val.assign(ri.rp[nparm] - 1, 0.0);
  for (int ix = 1; ix <= nx_if; ++ix) {
    const int idx = start + ix;
    if (idx < 1 || idx > nparm) continue;
    int k = ri.rp[idx - 1] - 1;
    double bsum = 0.0;
    for (int jx = std::max(1, ix + kx_min); jx <= std::min(nx_if, ix + kx_max); ++jx) {
      if (jx == ix) continue;
      const int jdx = start + jx;
      if (jdx < 1 || jdx > nparm) continue;
      const double d = x[jx] - x[ix];
      const double beta = std::exp(-(d * d) / (corr_x_iface * corr_x_iface));
      bsum = bsum + beta;
      ri.col[k] = jdx;
      ri.val[k] = beta * mvscale[jdx - 1];
      ++k;
    }
    ri.col[k] = idx;
    ri.val[k] = -bsum * mvscale[idx - 1];
  }
}

// apply_gauss_smooth_h / _v / iface_h (:1446-1482, :1619-1636): y = R x, and
// the transposes (:1484-1521): y = R^T x.
void csr_apply(const Csr& r, int nparm, const double* x, double* y, bool transpose) {
  for (int i = 0; i < nparm; ++i) y[i] = 0.0;
  for (int i = 1; i <= nparm; ++i)
    for (int k = r.rp[i - 1]; k < r.rp[i]; ++k) {
      if (transpose) y[r.col[k - 1] - 1] += r.val[k - 1] * x[i - 1];
      else y[i - 1] += r.val[k - 1] * x[r.col[k - 1] - 1];
    }
}

}  // namespace orc
