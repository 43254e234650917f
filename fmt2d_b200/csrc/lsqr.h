// Device LSQR on the augmented system of the reference's run_lsqr
// (src/inversion2d.f90:6578-7167) and the raw G / G^T products
// (sparse_Ax / sparse_ATx, src/inversion2d.f90:2997-3042).
//
// G is held twice in HBM, as CSR (rows = picks) and as CSC (columns =
// inversion parameters, entries of a column in ascending row order), so both
// products are gathers with a fixed summation order: results are
// deterministic run to run.  All vectors and scalars are FP64.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "engine.h"

namespace fmt2d {

struct LsqrParams {
  int smooth_type = 1;          // 1: Laplacian; 2: Gaussian R_h, R_v; 3: Laplacian + interface R_h
  double wdv = 0, wdv_iface = 0, w_smooth = 0, w_smooth_iface = 0, eps_min = 0;
  int max_iter = 2000;
};

struct LsqrOut {
  int iters = 0;
  double rnorm = 0, bnorm = 0, test2 = 0;
};

// Scalars of the iteration, kept on the device between kernels.
struct LsqrScalars {
  double alpha, beta;          // norms of the current v and u (their stored scale)
  double rhobar, phibar, anorm2, rnorm, test2, bnorm;
  double t_r, p_r;             // pending w / dm update: theta/rho, phi/rho
  int iter, iters_out;
  int state;                   // kLsInit, kLsRun, kLsFinal, kLsDone
  int pending;                 // kPendNone, kPendInitW, kPendUpdate
  unsigned count;              // blocks finished (last-block reductions)
  unsigned pad;
};

enum { kLsInit = 0, kLsRun = 1, kLsFinal = 2, kLsDone = 3 };
enum { kPendNone = 0, kPendInitW = 1, kPendUpdate = 2 };

// A sparse matrix over the inversion parameters (0-based CSR, np rows; rows
// the matrix does not cover are empty).  rp == nullptr: no matrix (all rows
// empty).
struct SpRows {
  const int* rp = nullptr;
  const int* col = nullptr;
  const double* val = nullptr;
};

// Kernel view of one solve.
struct LsqrDev {
  int nd = 0, np = 0, nvp = 0;
  const int* rp = nullptr;      // CSR row pointer (nd+1), 0-based
  const int* col = nullptr;     // CSR column (np = out of range, skipped)
  const double* val = nullptr;
  const int* cp = nullptr;      // CSC column pointer (np+1)
  const int* crow = nullptr;    // CSC row
  const double* cval = nullptr;
  const int4* nb = nullptr;     // per velocity parameter: left, right, up, down (-1 none)
  int if_start = 0, if_n = 0;   // inverted interface parameters [if_start, if_start+if_n)
  const uint8_t* mask = nullptr;// 1: velocity column masked (gtg < 0.01 eps_min)
  double ws_v = 0, ws_i = 0, wd_v = 0, wd_i = 0;
  // smooth_type and, for 2 and 3, the Gaussian operators: R_h, R_v and their
  // transposes, the interface R_h (applied as its own adjoint, as the
  // reference does)
  int stype = 1;
  SpRows rh, rht, rv, rvt, ri;
  const double* residual = nullptr;
  const double* dm_sum = nullptr;
  double* u = nullptr;          // [data | smoothing (np; 2 np for smooth_type 2) | damping],
                                // scale 1/beta
  double* v = nullptr;          // np, scale 1/alpha
  double* w = nullptr;          // np
  double* dm = nullptr;         // np
  double* part = nullptr;       // per-block partial sums
  LsqrScalars* sc = nullptr;
  int max_iter = 0;
};

// Launch shape shared by every kernel of a solve (the last-block reductions
// need one fixed grid).
constexpr int kLsThreads = 256;

// smooth_type 1 uses the Laplacian kernels, 2 and 3 the general ones (same
// scalar recurrences); the launch functions pick by d.stype.
void lsqr_launch_init_u(const LsqrDev& d, int grid, cudaStream_t st);
void lsqr_launch_adj(const LsqrDev& d, int grid, cudaStream_t st);
void lsqr_launch_fwd(const LsqrDev& d, int grid, cudaStream_t st);
void lsqr_launch_spmv(const LsqrDev& d, int transpose, const double* x, double* y, int grid,
                      cudaStream_t st);
void lsqr_launch_gtg(const LsqrDev& d, double* out, int grid, cudaStream_t st);
void lsqr_launch_mask(const LsqrDev& d, const double* gtg, double thr, uint8_t* mask, int grid,
                      cudaStream_t st);

class Lsqr {
 public:
  Lsqr(int device, cudaStream_t st);
  ~Lsqr();
  // Laplacian neighbour table of the model's inversion numbering.
  std::string set_geometry(const Model& m);
  // The same for an explicit parameter grid: idx[nz*nx] (ix fastest) holds
  // 1-based velocity parameter ids (0: none), nvp of them, followed by if_n
  // interface parameters (a coarse inversion grid, fmt2d_projection).
  std::string set_param_grid(int nx, int nz, const int* idx, int nvp, int if_n);
  // Gaussian smoothing operators of the smooth_type 2/3 layouts
  // (build_gauss_smooth_matrix / build_iface_gauss_smooth_matrix with the
  // column scaling mvscale folded in): R_h if corr_x > 0, R_v if corr_z > 0,
  // the interface R_h if corr_x_iface > 0 and an interface is inverted.
  std::string set_smoothing(const Model& m, double corr_x, double corr_z, double corr_x_iface,
                            const double* mvscale);
  // G from a host CSR (index base 0 or 1, as read_frechet_data2d's 1-based
  // arrays).  Builds the device CSR and CSC.
  std::string set_matrix(int ndata, int nparm, const int* row_ptr, const int* col,
                         const double* val, int base);
  std::string spmv(int transpose, const double* x, double* y);
  std::string gtg_diag(double* out);
  std::string solve(const LsqrParams& p, const double* residual, const double* gtg,
                    const double* dm_sum, double* dm, LsqrOut* out);
  // The same solve with every work vector in a file-scope device array
  // (nothing allocated); residual, gtg, dm_sum and dm are device pointers.
  std::string solve_noalloc(const LsqrParams& p, const double* residual, const double* gtg,
                            const double* dm_sum, double* dm, LsqrOut* out);
  int ndata() const { return nd_; }
  int nparm() const { return np_; }
  long long nnz() const { return nnz_; }
  double last_ms() const { return last_ms_; }
  int last_launches() const { return last_launches_; }

 private:
  std::string build_csc();
  LsqrDev view() const;
  int device_;
  cudaStream_t st_;
  int nd_ = 0, np_ = 0, nvp_ = 0, if_start_ = 0, if_n_ = 0;
  long long nnz_ = 0;
  int grid_ = 0;
  DevBuf rp_, col_, val_, cp_, crow_, cval_, nb_, mask_, res_, dms_, gtg_, u_, v_, w_, dm_,
      part_, sc_, x_, y_;
  // smoothing matrices: R_h, R_h^T, R_v, R_v^T, interface R_h
  DevBuf sm_rp_[5], sm_col_[5], sm_val_[5];
  bool have_sm_[5] = {false, false, false, false, false};
  int sm_np_ = -1;           // parameters the smoothing matrices were built for
  LsqrScalars* h_sc_ = nullptr;
  double last_ms_ = 0;
  int last_launches_ = 0;
  bool have_geom_ = false;
};

}  // namespace fmt2d
