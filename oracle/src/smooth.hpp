// Oracle Gaussian smoothing matrices.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#pragma once
#include <vector>

namespace orc {

struct Model;

// 1-based CSR: rp[nparm + 1] (rp[0] = 1), col 1-based parameter ids.
struct Csr {
  std::vector<int> rp, col;
  std::vector<double> val;
};

void gauss_smooth_matrices(const Model& m, int nparm, double corr_x, double corr_z,
                           const double* mvscale, Csr& rh, Csr& rv);
void iface_gauss_smooth_matrix(const Model& m, int nparm, double corr_x_iface,
                               const double* mvscale, Csr& ri);
void csr_apply(const Csr& r, int nparm, const double* x, double* y, bool transpose);

}  // namespace orc
