// Oracle LSQR interfaces.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#pragma once

namespace orc {

struct LsqrGeom {
  int nx = 0, nz = 0;
  const int* inv_idx = nullptr;   // nx*nz, ix fastest, 1-based ids, 0 inactive
  int iface_start = 0, iface_nx = 0;
};

struct LsqrInput {
  int ndata = 0, nparm = 0, n_vel_parms = 0, max_iter = 0;
  const int* gindx = nullptr;     // 1-based column ids
  const double* gval = nullptr;
  const int* row_ptr = nullptr;   // 1-based, ndata+1 entries
  const double* residual = nullptr;
  const double* gtg_diag = nullptr;
  const double* dm_sum = nullptr;
  double eps_min = 0, wdv = 0, wdv_iface = 0, w_smooth = 0, w_smooth_iface = 0;
};

struct LsqrResult {
  int iters = 0;
  double rnorm = 0, bnorm = 0, test2 = 0;
};

void sparse_Ax(int ndata, int nparm, const int* gindx, const double* gval, const int* row_ptr,
               const double* x, double* y);
void sparse_ATx(int ndata, int nparm, const int* gindx, const double* gval, const int* row_ptr,
                const double* y, double* x);
void laplacian(const LsqrGeom& G, int nparm, const double* vin, double* vout);
LsqrResult run_lsqr_laplacian(const LsqrGeom& G, const LsqrInput& in, double* dm);

struct Csr;
// run_lsqr for every smooth_type: 1 = [G; w_s L; w_d I], 2 = [G; w_s R_h;
// w_s R_v; w_d I] with the interface Gaussian ri in the R_h block's interface
// rows, 3 = [G; w_s L (velocity) + w_si ri (interface); w_d I].  rh / rv / ri
// are the 1-based CSRs of the Gaussian matrices (ri may be empty: not built).
LsqrResult run_lsqr_general(const LsqrGeom& G, const LsqrInput& in, int smooth_type,
                            const Csr* rh, const Csr* rv, const Csr* ri, double* dm);

}  // namespace orc
