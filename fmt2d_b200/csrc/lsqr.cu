// Device LSQR (src/inversion2d.f90:6578-7167, smooth_type 1) and the G / G^T
// products (src/inversion2d.f90:2997-3042).
//
// One LSQR iteration is two kernels:
//   k_ls_fwd : u <- [G v; w_s L v; w_d v] - alpha u      (warp per CSR row for
//              the data rows, thread per parameter for the smoothing and damping
//              rows) and the pending w / dm update of the previous iteration;
//   k_ls_adj : v <- [G^T u_G + w_s L u_L + w_d u_D] - beta v   (warp per CSC
//              column), masked, plus the scalar recurrences of the rotation.
// u and v are stored unnormalised together with their norms (beta, alpha):
// readers divide on load, which removes the two normalisation passes of the
// reference.  Every norm is a deterministic reduction: per-block partials
// summed in a fixed order by the last block to finish (no spin-waits).  The
// iteration loop runs as a captured CUDA graph of kIterPerGraph iterations;
// after convergence the kernels return at their first instruction.
#include "lsqr.h"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <algorithm>
#include <cmath>
#include <mutex>

namespace fmt2d {

#define LCK(x)                                                                \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_); \
  } while (0)

namespace {

constexpr int kIterPerGraph = 8;
constexpr double kAtol = 1.0e-4;   // inversion2d.f90:6868

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Sum over the block; the result is valid in thread 0.
__device__ double block_sum(double x) {
  __shared__ double sh[32];
  x = warp_sum(x);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    x = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
    x = warp_sum(x);
  }
  __syncthreads();
  return x;
}

// Publishes this block's partial sum; in the last block to finish returns
// true (in every thread) with the grid total in *total (thread 0 only).
__device__ bool last_block_total(const LsqrDev& d, double partial, double* total) {
  __shared__ bool last;
  partial = block_sum(partial);
  if (threadIdx.x == 0) {
    d.part[blockIdx.x] = partial;
    __threadfence();
    const unsigned t = atomicAdd(&d.sc->count, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(d.part + i);
  s = block_sum(s);
  if (threadIdx.x == 0) {
    *total = s;
    d.sc->count = 0u;
  }
  return true;
}

__device__ __forceinline__ bool masked(const LsqrDev& d, int j) { return j < d.nvp && d.mask[j]; }
__device__ __forceinline__ double w_smooth(const LsqrDev& d, int j) {
  return j < d.nvp ? (d.mask[j] ? 0.0 : d.ws_v) : d.ws_i;
}
__device__ __forceinline__ double w_damp(const LsqrDev& d, int j) {
  return j < d.nvp ? (d.mask[j] ? 0.0 : d.wd_v) : d.wd_i;
}

// apply_laplacian_smooth_2d (inversion2d.f90:1161-1249) at parameter j of the
// vector x (stride-free accessor): 5-point Laplacian over the existing
// neighbours of a velocity node (left, right, up, down, then -k centre), the
// 1-D interface Laplacian with one-sided ends.
__device__ __forceinline__ double lap_at(const LsqrDev& d, const double* x, int j) {
  if (j < d.nvp) {
    const int4 n = d.nb[j];
    double acc = 0.0;
    int k = 0;
    if (n.x >= 0) { acc += x[n.x]; ++k; }
    if (n.y >= 0) { acc += x[n.y]; ++k; }
    if (n.z >= 0) { acc += x[n.z]; ++k; }
    if (n.w >= 0) { acc += x[n.w]; ++k; }
    return acc - (double)k * x[j];
  }
  const int ix = j - d.if_start + 1;   // 1-based node of the interface
  if (ix < 1 || ix > d.if_n) return 0.0;
  if (ix == 1) return (j + 1 < d.np) ? (0.0 + x[j + 1]) - x[j] : 0.0;
  if (ix == d.if_n) return (0.0 + x[j - 1]) - x[j];
  return ((0.0 + x[j - 1]) + x[j + 1]) - 2.0 * x[j];
}

// sum_k val[k] * x[idx[k]] over [k0, k1), lanes strided, warp-reduced.
__device__ __forceinline__ double warp_dot(const int* __restrict__ idx,
                                           const double* __restrict__ val, int k0, int k1,
                                           const double* __restrict__ x, int lim) {
  const int lane = threadIdx.x & 31;
  double a0 = 0.0, a1 = 0.0;
  int k = k0 + lane;
  for (; k + 32 < k1; k += 64) {
    const int j0 = __ldg(idx + k), j1 = __ldg(idx + k + 32);
    const double g0 = __ldg(val + k), g1 = __ldg(val + k + 32);
    if (j0 < lim) a0 += g0 * x[j0];
    if (j1 < lim) a1 += g1 * x[j1];
  }
  if (k < k1) {
    const int j0 = __ldg(idx + k);
    if (j0 < lim) a0 += __ldg(val + k) * x[j0];
  }
  return warp_sum(a0 + a1);
}

// The right-hand side's norm (every block passes its partial sum of squares):
// beta, and the early exit of a zero right-hand side.
__device__ void init_u_tail(const LsqrDev& d, double ss) {
  double tot = 0.0;
  if (last_block_total(d, ss, &tot) && threadIdx.x == 0) {
    LsqrScalars& S = *d.sc;
    const double bnorm = sqrt(tot);
    S.bnorm = bnorm;
    S.beta = bnorm;
    S.alpha = 1.0;
    S.iter = 0;
    S.pending = kPendNone;
    if (bnorm < 1.0e-30) {   // inversion2d.f90:6739-6745
      S.state = kLsDone;
      S.iters_out = 0;
      S.rnorm = 0.0;
      S.test2 = 0.0;
    } else {
      S.state = kLsInit;
    }
  }
}

// v's norm alpha, then either the start of the iteration (after the first
// A^T u) or the rotation of one LSQR step.
__device__ void adj_tail(const LsqrDev& d, double ss, bool init) {
  double tot = 0.0;
  if (last_block_total(d, ss, &tot) && threadIdx.x == 0) {
    LsqrScalars& S = *d.sc;
    const double a = sqrt(tot);
    if (init) {
      if (a < 1.0e-30) {   // inversion2d.f90:6853-6860
        S.state = kLsDone;
        S.iters_out = 0;
        S.rnorm = S.bnorm;
        S.test2 = 0.0;
        return;
      }
      S.alpha = a;
      S.phibar = S.beta;
      S.rhobar = a;
      S.anorm2 = a * a + S.beta * S.beta;
      S.pending = kPendInitW;
      S.state = kLsRun;
      S.iter = 0;
      return;
    }
    // inversion2d.f90:7122-7157
    const double b = S.beta;
    S.alpha = a;
    S.anorm2 = S.anorm2 + a * a + b * b;
    const double rho = sqrt(S.rhobar * S.rhobar + b * b);
    const double c = S.rhobar / rho, s = b / rho;
    const double theta = s * a;
    S.rhobar = -c * a;
    const double phi = c * S.phibar;
    S.phibar = s * S.phibar;
    S.t_r = theta / rho;
    S.p_r = phi / rho;
    S.pending = kPendUpdate;
    S.rnorm = fabs(S.phibar);
    const double arnorm = S.phibar * a * fabs(c);
    S.test2 = arnorm / (sqrt(S.anorm2) * S.rnorm + 1.0e-30);
    S.iter += 1;
    if (S.test2 < kAtol || 1.0 + S.test2 <= 1.0) {
      S.state = kLsFinal;
      S.iters_out = S.iter;
    } else if (S.iter >= d.max_iter) {
      S.state = kLsFinal;
      S.iters_out = d.max_iter + 1;   // a Fortran DO index after the last trip
    }
  }
}

// u's norm beta; the pending w / dm update is done.
__device__ void fwd_tail(const LsqrDev& d, double ss, bool run, int state) {
  double tot = 0.0;
  if (last_block_total(d, ss, &tot) && threadIdx.x == 0) {
    LsqrScalars& S = *d.sc;
    if (run) S.beta = sqrt(tot);
    S.pending = kPendNone;
    if (state == kLsFinal) S.state = kLsDone;
  }
}

// The pending w / dm update of the previous step at parameter j (vn: v_j
// normalised).
__device__ __forceinline__ void w_dm_update(const LsqrDev& d, int j, double vn, int pending,
                                            double t_r, double p_r) {
  if (pending == kPendInitW) {
    d.w[j] = vn;
  } else if (pending == kPendUpdate) {
    const bool m = masked(d, j);
    const double wo = d.w[j];
    const double z = m ? 0.0 : wo;
    double wn = vn - t_r * wo;
    if (m) wn = 0.0;
    d.w[j] = wn;
    d.dm[j] = d.dm[j] + p_r * z;
  }
}

__global__ void __launch_bounds__(kLsThreads) k_ls_init_u(LsqrDev d) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  double ss = 0.0;
  for (int i = tid; i < d.nd; i += nth) {
    const double r = d.residual[i];
    d.u[i] = r;
    ss += r * r;
  }
  for (int j = tid; j < d.np; j += nth) {
    const double s = -(w_smooth(d, j) * lap_at(d, d.dm_sum, j));
    const double t = -(w_damp(d, j) * d.dm_sum[j]);
    d.u[d.nd + j] = s;
    d.u[d.nd + d.np + j] = t;
    ss += s * s + t * t;
  }
  init_u_tail(d, ss);
}

// v <- A^T u (- beta v), masked; then the rotation of one LSQR step.
__global__ void __launch_bounds__(kLsThreads) k_ls_adj(LsqrDev d) {
  const int state = d.sc->state;
  if (state != kLsInit && state != kLsRun) return;
  const bool init = state == kLsInit;
  const double beta = d.sc->beta, alpha = d.sc->alpha;
  const double bsc = beta > 0.0 ? beta : 1.0, asc = alpha > 0.0 ? alpha : 1.0;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  const double* uL = d.u + d.nd;
  const double* uD = d.u + d.nd + d.np;
  double ss = 0.0;
  for (int j = warp; j < d.np; j += nwarp) {
    const double g = warp_dot(d.crow, d.cval, d.cp[j], d.cp[j + 1], d.u, d.nd);
    if (lane == 0) {
      double atu = g / bsc;
      atu = atu + (w_smooth(d, j) * lap_at(d, uL, j)) / bsc;
      atu = atu + (w_damp(d, j) * uD[j]) / bsc;
      double vn = init ? atu : atu - beta * (d.v[j] / asc);
      if (masked(d, j)) vn = 0.0;
      d.v[j] = vn;
      ss += vn * vn;
    }
  }
  adj_tail(d, ss, init);
}

// u <- A v - alpha u, and the pending w / dm update of the previous step.
__global__ void __launch_bounds__(kLsThreads) k_ls_fwd(LsqrDev d) {
  const int state = d.sc->state;
  if (state != kLsRun && state != kLsFinal) return;
  const bool run = state == kLsRun;
  const int pending = d.sc->pending;
  const double alpha = d.sc->alpha, beta = d.sc->beta;
  const double t_r = d.sc->t_r, p_r = d.sc->p_r;
  const double bsc = beta > 0.0 ? beta : 1.0, asc = alpha > 0.0 ? alpha : 1.0;
  const int lane = threadIdx.x & 31;
  double ss = 0.0;
  if (run) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarp = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < d.nd; i += nwarp) {
      const double g = warp_dot(d.col, d.val, d.rp[i], d.rp[i + 1], d.v, d.np);
      if (lane == 0) {
        const double un = g / asc - alpha * (d.u[i] / bsc);
        d.u[i] = un;
        ss += un * un;
      }
    }
  }
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  double* uL = d.u + d.nd;
  double* uD = d.u + d.nd + d.np;
  for (int j = tid; j < d.np; j += nth) {
    const double vn = d.v[j] / asc;
    if (run) {
      const double s = (w_smooth(d, j) * lap_at(d, d.v, j)) / asc - alpha * (uL[j] / bsc);
      const double t = w_damp(d, j) * vn - alpha * (uD[j] / bsc);
      uL[j] = s;
      uD[j] = t;
      ss += s * s + t * t;
    }
    w_dm_update(d, j, vn, pending, t_r, p_r);
  }
  fwd_tail(d, ss, run, state);
}

// ---------------------------------------------------------------- Gaussian layouts
// smooth_type 2: u = [data | w_s R_h | w_s R_v | damping], the interface rows
// of the R_h block holding w_si R_i instead; adjoint R_h^T, R_v^T, R_i.
// smooth_type 3: u = [data | w_s L (velocity rows), w_si R_i (interface
// rows) | damping]; adjoint L and R_i.  Masked velocity rows are zero in
// every block (inversion2d.f90:6608-6736, 6753-6851, 6883-7120).

// Row j of A times x, warp-cooperative (every lane gets the sum).
__device__ __forceinline__ double row_dot(const SpRows& A, int j, const double* x, int np) {
  if (!A.rp) return 0.0;
  return warp_dot(A.col, A.val, A.rp[j], A.rp[j + 1], x, np);
}

__device__ __forceinline__ double* damp_block(const LsqrDev& d) {
  return d.u + d.nd + (d.stype == 2 ? 2 : 1) * (size_t)d.np;
}

// Rows j of the smoothing blocks applied to x (unweighted by a scale):
// s1 (the first block), s2 (the R_v block of smooth_type 2).  Warp-uniform j.
__device__ __forceinline__ void smooth_rows(const LsqrDev& d, const double* x, int j, double* s1,
                                            double* s2) {
  *s2 = 0.0;
  if (d.stype == 3) {
    if (j < d.nvp) {
      *s1 = w_smooth(d, j) * lap_at(d, x, j);
    } else {
      const double h = row_dot(d.ri, j, x, d.np);
      *s1 = d.ws_i > 0.0 ? d.ws_i * h : 0.0;
    }
    return;
  }
  const double h = row_dot(d.rh, j, x, d.np), v = row_dot(d.rv, j, x, d.np);
  if (j < d.nvp) {
    const bool m = d.mask[j];
    *s1 = d.ws_v * (m ? 0.0 : h);
    *s2 = d.ws_v * (m ? 0.0 : v);
  } else {
    const bool ri = d.ws_i > 0.0 && d.ri.rp;
    const double hi = ri ? row_dot(d.ri, j, x, d.np) : 0.0;
    *s1 = ri ? d.ws_i * hi : 0.0;
    *s2 = d.ws_v * v;
  }
}

__global__ void __launch_bounds__(kLsThreads) k_ls_init_u_g(LsqrDev d) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31, warp = tid >> 5, nwarp = nth >> 5;
  double ss = 0.0;
  for (int i = tid; i < d.nd; i += nth) {
    const double r = d.residual[i];
    d.u[i] = r;
    ss += r * r;
  }
  double* u1 = d.u + d.nd;
  double* u2 = u1 + d.np;
  for (int j = warp; j < d.np; j += nwarp) {
    double s1, s2;
    smooth_rows(d, d.dm_sum, j, &s1, &s2);
    if (lane == 0) {
      u1[j] = -s1;
      ss += s1 * s1;
      if (d.stype == 2) {
        u2[j] = -s2;
        ss += s2 * s2;
      }
    }
  }
  double* uD = damp_block(d);
  for (int j = tid; j < d.np; j += nth) {
    const double t = -(w_damp(d, j) * d.dm_sum[j]);
    uD[j] = t;
    ss += t * t;
  }
  init_u_tail(d, ss);
}

__global__ void __launch_bounds__(kLsThreads) k_ls_adj_g(LsqrDev d) {
  const int state = d.sc->state;
  if (state != kLsInit && state != kLsRun) return;
  const bool init = state == kLsInit;
  const double beta = d.sc->beta, alpha = d.sc->alpha;
  const double bsc = beta > 0.0 ? beta : 1.0, asc = alpha > 0.0 ? alpha : 1.0;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  const double* u1 = d.u + d.nd;
  const double* u2 = u1 + d.np;
  const double* uD = damp_block(d);
  double ss = 0.0;
  for (int j = warp; j < d.np; j += nwarp) {
    const double g = warp_dot(d.crow, d.cval, d.cp[j], d.cp[j + 1], d.u, d.nd);
    double a1, a2 = 0.0, ai = 0.0;
    bool has_i = false;
    if (d.stype == 3) {
      if (j < d.nvp) {
        a1 = w_smooth(d, j) * lap_at(d, u1, j);
      } else {
        const double h = row_dot(d.ri, j, u1, d.np);
        a1 = d.ws_i > 0.0 ? d.ws_i * h : 0.0;
      }
    } else {
      const double h = row_dot(d.rht, j, u1, d.np), v = row_dot(d.rvt, j, u2, d.np);
      const bool m = masked(d, j);
      a1 = d.ws_v * (m ? 0.0 : h);
      a2 = d.ws_v * (m ? 0.0 : v);
      if (j >= d.nvp && d.ws_i > 0.0 && d.ri.rp) {
        ai = d.ws_i * row_dot(d.ri, j, u1, d.np);
        has_i = true;
      }
    }
    if (lane == 0) {
      double atu = g / bsc;
      atu = atu + a1 / bsc;
      if (d.stype == 2) {
        atu = atu + a2 / bsc;
        if (has_i) atu = atu + ai / bsc;
      }
      atu = atu + (w_damp(d, j) * uD[j]) / bsc;
      double vn = init ? atu : atu - beta * (d.v[j] / asc);
      if (masked(d, j)) vn = 0.0;
      d.v[j] = vn;
      ss += vn * vn;
    }
  }
  adj_tail(d, ss, init);
}

__global__ void __launch_bounds__(kLsThreads) k_ls_fwd_g(LsqrDev d) {
  const int state = d.sc->state;
  if (state != kLsRun && state != kLsFinal) return;
  const bool run = state == kLsRun;
  const int pending = d.sc->pending;
  const double alpha = d.sc->alpha, beta = d.sc->beta;
  const double t_r = d.sc->t_r, p_r = d.sc->p_r;
  const double bsc = beta > 0.0 ? beta : 1.0, asc = alpha > 0.0 ? alpha : 1.0;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  double ss = 0.0;
  double* u1 = d.u + d.nd;
  double* u2 = u1 + d.np;
  double* uD = damp_block(d);
  if (run) {
    for (int i = warp; i < d.nd; i += nwarp) {
      const double g = warp_dot(d.col, d.val, d.rp[i], d.rp[i + 1], d.v, d.np);
      if (lane == 0) {
        const double un = g / asc - alpha * (d.u[i] / bsc);
        d.u[i] = un;
        ss += un * un;
      }
    }
    for (int j = warp; j < d.np; j += nwarp) {
      double s1, s2;
      smooth_rows(d, d.v, j, &s1, &s2);
      if (lane == 0) {
        const double a = s1 / asc - alpha * (u1[j] / bsc);
        u1[j] = a;
        ss += a * a;
        if (d.stype == 2) {
          const double b = s2 / asc - alpha * (u2[j] / bsc);
          u2[j] = b;
          ss += b * b;
        }
      }
    }
  }
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int j = tid; j < d.np; j += nth) {
    const double vn = d.v[j] / asc;
    if (run) {
      const double t = w_damp(d, j) * vn - alpha * (uD[j] / bsc);
      uD[j] = t;
      ss += t * t;
    }
    w_dm_update(d, j, vn, pending, t_r, p_r);
  }
  fwd_tail(d, ss, run, state);
}

__global__ void k_spmv_rows(LsqrDev d, const double* __restrict__ x, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < d.nd; i += nwarp) {
    const double g = warp_dot(d.col, d.val, d.rp[i], d.rp[i + 1], x, d.np);
    if (lane == 0) y[i] = g;
  }
}

__global__ void k_spmv_cols(LsqrDev d, const double* __restrict__ x, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int j = warp; j < d.np; j += nwarp) {
    const double g = warp_dot(d.crow, d.cval, d.cp[j], d.cp[j + 1], x, d.nd);
    if (lane == 0) y[j] = g;
  }
}

// Column sums of squares (inversion2d.f90:466-475).
__global__ void k_gtg(LsqrDev d, double* out) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int j = warp; j < d.np; j += nwarp) {
    double a = 0.0;
    for (int k = d.cp[j] + lane; k < d.cp[j + 1]; k += 32) {
      const double g = d.cval[k];
      a += g * g;
    }
    a = warp_sum(a);
    if (lane == 0) out[j] = a;
  }
}

__global__ void k_mask(LsqrDev d, const double* gtg, double thr, uint8_t* mask) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int j = tid; j < d.np; j += nth) mask[j] = (j < d.nvp && gtg[j] < thr) ? 1 : 0;
}

// ---------------------------------------------------------------- CSR / CSC build
__global__ void k_csr_rebase(int* rp, int nrp, int* col, long long nnz, int base, int np) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < nrp; k += nth) rp[k] -= base;
  for (long long k = tid; k < nnz; k += nth) {
    const int c = col[k] - base;
    col[k] = (c >= 0 && c < np) ? c : np;   // out of range: skipped (sparse_Ax/ATx)
  }
}

__global__ void k_row_of(const int* rp, int nd, int* row_of, int* iota) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < nd; i += nwarp)
    for (int k = rp[i] + lane; k < rp[i + 1]; k += 32) {
      row_of[k] = i;
      iota[k] = k;
    }
}

__global__ void k_count_cols(const int* col, long long nnz, int np, int* cnt) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < nnz; k += nth)
    if (col[k] < np) atomicAdd(cnt + col[k], 1);
}

__global__ void k_csc_fill(const int* perm, const int* row_of, const double* val, int nvalid,
                           int* crow, double* cval) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int k = tid; k < nvalid; k += nth) {
    const int p = perm[k];
    crow[k] = row_of[p];
    cval[k] = val[p];
  }
}

}  // namespace

void lsqr_launch_init_u(const LsqrDev& d, int grid, cudaStream_t st) {
  if (d.stype == 1) k_ls_init_u<<<grid, kLsThreads, 0, st>>>(d);
  else k_ls_init_u_g<<<grid, kLsThreads, 0, st>>>(d);
}
void lsqr_launch_adj(const LsqrDev& d, int grid, cudaStream_t st) {
  if (d.stype == 1) k_ls_adj<<<grid, kLsThreads, 0, st>>>(d);
  else k_ls_adj_g<<<grid, kLsThreads, 0, st>>>(d);
}
void lsqr_launch_fwd(const LsqrDev& d, int grid, cudaStream_t st) {
  if (d.stype == 1) k_ls_fwd<<<grid, kLsThreads, 0, st>>>(d);
  else k_ls_fwd_g<<<grid, kLsThreads, 0, st>>>(d);
}
void lsqr_launch_spmv(const LsqrDev& d, int transpose, const double* x, double* y, int grid,
                      cudaStream_t st) {
  if (transpose) k_spmv_cols<<<grid, kLsThreads, 0, st>>>(d, x, y);
  else k_spmv_rows<<<grid, kLsThreads, 0, st>>>(d, x, y);
}
void lsqr_launch_gtg(const LsqrDev& d, double* out, int grid, cudaStream_t st) {
  k_gtg<<<grid, kLsThreads, 0, st>>>(d, out);
}
void lsqr_launch_mask(const LsqrDev& d, const double* gtg, double thr, uint8_t* mask, int grid,
                      cudaStream_t st) {
  k_mask<<<grid, kLsThreads, 0, st>>>(d, gtg, thr, mask);
}

// ---------------------------------------------------------------- host
Lsqr::Lsqr(int device, cudaStream_t st) : device_(device), st_(st) {
  cudaSetDevice(device_);
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ls_adj, kLsThreads, 0);
  grid_ = std::max(1, nsm) * std::max(1, std::min(per_sm, 8));
  cudaMallocHost(&h_sc_, sizeof(LsqrScalars));
}

Lsqr::~Lsqr() {
  cudaSetDevice(device_);
  if (h_sc_) cudaFreeHost(h_sc_);
}

std::string Lsqr::set_geometry(const Model& m) {
  return set_param_grid(m.nx, m.nz, m.inv_idx.data(), m.n_vel_parms,
                        m.iface_inv > 0 ? m.nx : 0);
}

std::string Lsqr::set_param_grid(int nx, int nz, const int* idx, int nvp, int if_n) {
  if (nx < 1 || nz < 1 || !idx || nvp < 0 || if_n < 0) return "bad parameter grid";
  for (size_t k = 0; k < (size_t)nx * nz; ++k)
    if (idx[k] < 0 || idx[k] > nvp) return "parameter grid ids must be 0..n_vel_parms";
  // a new parameter grid: smoothing matrices built for another no longer apply
  for (bool& h : have_sm_) h = false;
  sm_np_ = -1;
  nvp_ = nvp;
  if_start_ = nvp;
  if_n_ = if_n;
  std::vector<int4> nb((size_t)std::max(nvp_, 1), make_int4(-1, -1, -1, -1));
  auto id = [&](int ix, int iz) { return idx[(size_t)iz * nx + ix]; };
  for (int iz = 0; iz < nz; ++iz)
    for (int ix = 0; ix < nx; ++ix) {
      const int k = id(ix, iz);
      if (k <= 0) continue;
      int4 n = make_int4(-1, -1, -1, -1);
      if (ix > 0 && id(ix - 1, iz) > 0) n.x = id(ix - 1, iz) - 1;
      if (ix < nx - 1 && id(ix + 1, iz) > 0) n.y = id(ix + 1, iz) - 1;
      if (iz > 0 && id(ix, iz - 1) > 0) n.z = id(ix, iz - 1) - 1;
      if (iz < nz - 1 && id(ix, iz + 1) > 0) n.w = id(ix, iz + 1) - 1;
      nb[k - 1] = n;
    }
  cudaSetDevice(device_);
  nb_.alloc(nb.size() * sizeof(int4));
  if (!nb_.p) return "device allocation failed (Laplacian table)";
  LCK(cudaMemcpyAsync(nb_.p, nb.data(), nb.size() * sizeof(int4), cudaMemcpyHostToDevice, st_));
  LCK(cudaStreamSynchronize(st_));
  have_geom_ = true;
  return std::string();
}

LsqrDev Lsqr::view() const {
  LsqrDev d;
  d.nd = nd_;
  d.np = np_;
  d.nvp = std::min(nvp_, np_);
  d.rp = rp_.as<int>();
  d.col = col_.as<int>();
  d.val = val_.as<double>();
  d.cp = cp_.as<int>();
  d.crow = crow_.as<int>();
  d.cval = cval_.as<double>();
  d.nb = nb_.as<int4>();
  d.if_start = if_start_;
  d.if_n = if_n_;
  d.mask = mask_.as<uint8_t>();
  d.residual = res_.as<double>();
  d.dm_sum = dms_.as<double>();
  d.u = u_.as<double>();
  d.v = v_.as<double>();
  d.w = w_.as<double>();
  d.dm = dm_.as<double>();
  d.part = part_.as<double>();
  d.sc = sc_.as<LsqrScalars>();
  return d;
}

std::string Lsqr::set_matrix(int ndata, int nparm, const int* row_ptr, const int* col,
                             const double* val, int base) {
  if (ndata < 0 || nparm <= 0 || !row_ptr || (base != 0 && base != 1))
    return "bad matrix dimensions";
  const long long nnz = (long long)row_ptr[ndata] - base;
  if (row_ptr[0] != base || nnz < 0 || nnz > 0x7fffffffLL) return "bad row pointer";
  for (int i = 0; i < ndata; ++i)
    if (row_ptr[i + 1] < row_ptr[i]) return "row pointer not monotone";
  if (nnz > 0 && (!col || !val)) return "null column or value array";
  cudaSetDevice(device_);
  nd_ = ndata;
  np_ = nparm;
  nnz_ = nnz;
  rp_.alloc((size_t)(ndata + 1) * 4);
  col_.alloc((size_t)nnz * 4);
  val_.alloc((size_t)nnz * 8);
  if (!rp_.p || !col_.p || !val_.p) return "device allocation failed (CSR)";
  LCK(cudaMemcpyAsync(rp_.p, row_ptr, (size_t)(ndata + 1) * 4, cudaMemcpyHostToDevice, st_));
  if (nnz) {
    LCK(cudaMemcpyAsync(col_.p, col, (size_t)nnz * 4, cudaMemcpyHostToDevice, st_));
    LCK(cudaMemcpyAsync(val_.p, val, (size_t)nnz * 8, cudaMemcpyHostToDevice, st_));
  }
  k_csr_rebase<<<grid_, kLsThreads, 0, st_>>>(rp_.as<int>(), ndata + 1, col_.as<int>(), nnz, base,
                                              nparm);
  LCK(cudaGetLastError());
  return build_csc();
}

std::string Lsqr::build_csc() {
  const int nnz = (int)nnz_;
  cp_.alloc((size_t)(np_ + 1) * 4);
  crow_.alloc((size_t)nnz * 4);
  cval_.alloc((size_t)nnz * 8);
  part_.alloc((size_t)grid_ * 8);
  sc_.alloc(sizeof(LsqrScalars));
  if (!cp_.p || !crow_.p || !cval_.p || !part_.p || !sc_.p) return "device allocation failed (CSC)";
  DevBuf row_of, iota, keys, perm, cnt, tmp;
  row_of.alloc((size_t)nnz * 4);
  iota.alloc((size_t)nnz * 4);
  keys.alloc((size_t)nnz * 4);
  perm.alloc((size_t)nnz * 4);
  cnt.alloc((size_t)(np_ + 1) * 4);
  if (!row_of.p || !iota.p || !keys.p || !perm.p || !cnt.p) return "device allocation failed (CSC build)";
  LCK(cudaMemsetAsync(cnt.p, 0, (size_t)(np_ + 1) * 4, st_));
  k_row_of<<<grid_, kLsThreads, 0, st_>>>(rp_.as<int>(), nd_, row_of.as<int>(), iota.as<int>());
  k_count_cols<<<grid_, kLsThreads, 0, st_>>>(col_.as<int>(), nnz, np_, cnt.as<int>());
  LCK(cudaGetLastError());
  int end_bit = 1;
  while (end_bit < 31 && (1LL << end_bit) <= np_) ++end_bit;
  size_t sort_bytes = 0, scan_bytes = 0;
  LCK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, col_.as<int>(), keys.as<int>(),
                                      iota.as<int>(), perm.as<int>(), nnz, 0, end_bit, st_));
  LCK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt.as<int>(), cp_.as<int>(), np_ + 1,
                                    st_));
  tmp.alloc(std::max(sort_bytes, scan_bytes));
  if (!tmp.p) return "device allocation failed (sort workspace)";
  if (nnz)
    LCK(cub::DeviceRadixSort::SortPairs(tmp.p, sort_bytes, col_.as<int>(), keys.as<int>(),
                                        iota.as<int>(), perm.as<int>(), nnz, 0, end_bit, st_));
  LCK(cub::DeviceScan::ExclusiveSum(tmp.p, scan_bytes, cnt.as<int>(), cp_.as<int>(), np_ + 1, st_));
  int nvalid = 0;
  LCK(cudaMemcpyAsync(&nvalid, cp_.as<int>() + np_, 4, cudaMemcpyDeviceToHost, st_));
  LCK(cudaStreamSynchronize(st_));
  if (nvalid > 0)
    k_csc_fill<<<grid_, kLsThreads, 0, st_>>>(perm.as<int>(), row_of.as<int>(), val_.as<double>(),
                                              nvalid, crow_.as<int>(), cval_.as<double>());
  LCK(cudaGetLastError());
  LCK(cudaStreamSynchronize(st_));
  return std::string();
}

std::string Lsqr::spmv(int transpose, const double* x, double* y) {
  if (!rp_.p) return "no matrix set";
  cudaSetDevice(device_);
  const int nin = transpose ? nd_ : np_, nout = transpose ? np_ : nd_;
  x_.alloc((size_t)std::max(nin, 1) * 8);
  y_.alloc((size_t)std::max(nout, 1) * 8);
  if (!x_.p || !y_.p) return "device allocation failed";
  if (nin) LCK(cudaMemcpyAsync(x_.p, x, (size_t)nin * 8, cudaMemcpyHostToDevice, st_));
  lsqr_launch_spmv(view(), transpose, x_.as<double>(), y_.as<double>(), grid_, st_);
  LCK(cudaGetLastError());
  if (nout) LCK(cudaMemcpyAsync(y, y_.p, (size_t)nout * 8, cudaMemcpyDeviceToHost, st_));
  LCK(cudaStreamSynchronize(st_));
  return std::string();
}

std::string Lsqr::gtg_diag(double* out) {
  if (!rp_.p) return "no matrix set";
  cudaSetDevice(device_);
  y_.alloc((size_t)np_ * 8);
  if (!y_.p) return "device allocation failed";
  lsqr_launch_gtg(view(), y_.as<double>(), grid_, st_);
  LCK(cudaGetLastError());
  LCK(cudaMemcpyAsync(out, y_.p, (size_t)np_ * 8, cudaMemcpyDeviceToHost, st_));
  LCK(cudaStreamSynchronize(st_));
  return std::string();
}

namespace {

// 1-based host CSR (np rows) -> 0-based device CSR; with transpose, the CSR of
// the transpose (entries of a row of A^T in ascending row order of A).
std::string upload_csr(const std::vector<int>& rp1, const std::vector<int>& col1,
                       const std::vector<double>& val, bool transpose, int np, DevBuf& rp_d,
                       DevBuf& col_d, DevBuf& val_d, cudaStream_t st) {
  const size_t nnz = col1.size();
  std::vector<int> rp(np + 1, 0), col(nnz);
  std::vector<double> v(nnz);
  if (!transpose) {
    for (int i = 0; i <= np; ++i) rp[i] = rp1[i] - 1;
    for (size_t k = 0; k < nnz; ++k) col[k] = col1[k] - 1;
    v = val;
  } else {
    for (size_t k = 0; k < nnz; ++k) ++rp[col1[k]];   // counts at (col - 1) + 1
    for (int i = 0; i < np; ++i) rp[i + 1] += rp[i];
    std::vector<int> next(rp.begin(), rp.end() - 1);
    for (int i = 0; i < np; ++i)
      for (int k = rp1[i] - 1; k < rp1[i + 1] - 1; ++k) {
        const int q = next[col1[k] - 1]++;
        col[q] = i;
        v[q] = val[k];
      }
  }
  rp_d.alloc((size_t)(np + 1) * 4);
  col_d.alloc(std::max<size_t>(nnz, 1) * 4);
  val_d.alloc(std::max<size_t>(nnz, 1) * 8);
  if (!rp_d.p || !col_d.p || !val_d.p) return "device allocation failed (smoothing matrix)";
  LCK(cudaMemcpyAsync(rp_d.p, rp.data(), (size_t)(np + 1) * 4, cudaMemcpyHostToDevice, st));
  if (nnz) {
    LCK(cudaMemcpyAsync(col_d.p, col.data(), nnz * 4, cudaMemcpyHostToDevice, st));
    LCK(cudaMemcpyAsync(val_d.p, v.data(), nnz * 8, cudaMemcpyHostToDevice, st));
  }
  LCK(cudaStreamSynchronize(st));
  return std::string();
}

}  // namespace

std::string Lsqr::set_smoothing(const Model& m, double corr_x, double corr_z, double corr_x_iface,
                                const double* mvscale) {
  if (!mvscale) return "null mvscale";
  cudaSetDevice(device_);
  const int np = m.n_inv_parms;
  for (bool& h : have_sm_) h = false;
  sm_np_ = np;
  std::vector<int> rp, col;
  std::vector<double> val;
  // R_h -> slots 0 (R_h) and 1 (R_h^T), R_v -> 2 and 3, interface R_h -> 4
  const struct { int which; double c; int slot; } mats[3] = {
      {0, corr_x, 0}, {1, corr_z, 2}, {2, corr_x_iface, 4}};
  for (const auto& q : mats) {
    if (!(q.c > 0.0)) continue;
    if (q.which == 2 && m.iface_inv <= 0) continue;
    std::string e = gauss_smooth_csr(m, q.which, corr_x, corr_z, corr_x_iface, mvscale, rp, col, val);
    if (!e.empty()) return e;
    e = upload_csr(rp, col, val, false, np, sm_rp_[q.slot], sm_col_[q.slot], sm_val_[q.slot], st_);
    if (!e.empty()) return e;
    have_sm_[q.slot] = true;
    if (q.which < 2) {
      e = upload_csr(rp, col, val, true, np, sm_rp_[q.slot + 1], sm_col_[q.slot + 1],
                     sm_val_[q.slot + 1], st_);
      if (!e.empty()) return e;
      have_sm_[q.slot + 1] = true;
    }
  }
  return std::string();
}

std::string Lsqr::solve(const LsqrParams& p, const double* residual, const double* gtg,
                        const double* dm_sum, double* dm, LsqrOut* out) {
  if (!rp_.p) return "no matrix set";
  if (!have_geom_) return "no model geometry for the smoothing operator";
  if (p.smooth_type < 1 || p.smooth_type > 3) return "smooth_type must be 1, 2 or 3";
  if (p.max_iter < 1) return "max_iter must be >= 1";
  if (np_ != if_start_ + if_n_) return "matrix columns differ from the model's inversion parameters";
  if (!dm) return "null output";
  if (p.smooth_type != 1 && sm_np_ != np_)
    return "smooth_type 2 and 3 need the Gaussian matrices of this model (set_smoothing)";
  if (p.smooth_type == 2 && p.w_smooth > 0.0 && !(have_sm_[0] && have_sm_[2]))
    return "smooth_type 2 with w_smooth > 0 needs R_h and R_v (corr_x, corr_z > 0)";
  cudaSetDevice(device_);
  const size_t na = (size_t)nd_ + (p.smooth_type == 2 ? 3 : 2) * (size_t)np_;
  res_.alloc((size_t)std::max(nd_, 1) * 8);
  dms_.alloc((size_t)np_ * 8);
  gtg_.alloc((size_t)np_ * 8);
  mask_.alloc((size_t)np_);
  u_.alloc(na * 8);
  v_.alloc((size_t)np_ * 8);
  w_.alloc((size_t)np_ * 8);
  dm_.alloc((size_t)np_ * 8);
  if (!res_.p || !dms_.p || !gtg_.p || !mask_.p || !u_.p || !v_.p || !w_.p || !dm_.p)
    return "device allocation failed (LSQR vectors)";
  if (nd_ && !residual) return "null residual";
  // events and the iteration graph are released on every return path
  struct Res {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~Res() {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } r;
  LCK(cudaEventCreate(&r.e0));
  LCK(cudaEventCreate(&r.e1));
  cudaEvent_t e0 = r.e0, e1 = r.e1;
  cudaEventRecord(e0, st_);
  if (nd_) LCK(cudaMemcpyAsync(res_.p, residual, (size_t)nd_ * 8, cudaMemcpyHostToDevice, st_));
  if (dm_sum) LCK(cudaMemcpyAsync(dms_.p, dm_sum, (size_t)np_ * 8, cudaMemcpyHostToDevice, st_));
  else LCK(cudaMemsetAsync(dms_.p, 0, (size_t)np_ * 8, st_));
  LsqrDev d = view();
  d.ws_v = p.w_smooth;
  d.ws_i = p.w_smooth_iface;
  d.wd_v = p.wdv;
  d.wd_i = p.wdv_iface;
  d.max_iter = p.max_iter;
  d.stype = p.smooth_type;
  if (d.stype != 1) {
    auto rows = [&](int k) {
      SpRows r;
      if (have_sm_[k]) {
        r.rp = sm_rp_[k].as<int>();
        r.col = sm_col_[k].as<int>();
        r.val = sm_val_[k].as<double>();
      }
      return r;
    };
    d.rh = rows(0);
    d.rht = rows(1);
    d.rv = rows(2);
    d.rvt = rows(3);
    d.ri = rows(4);
  }
  int launches = 0;
  if (gtg) {
    LCK(cudaMemcpyAsync(gtg_.p, gtg, (size_t)np_ * 8, cudaMemcpyHostToDevice, st_));
  } else {
    lsqr_launch_gtg(d, gtg_.as<double>(), grid_, st_);
    ++launches;
  }
  lsqr_launch_mask(d, gtg_.as<double>(), p.eps_min * 0.01, mask_.as<uint8_t>(), grid_, st_);
  LCK(cudaMemsetAsync(dm_.p, 0, (size_t)np_ * 8, st_));
  LCK(cudaMemsetAsync(sc_.p, 0, sizeof(LsqrScalars), st_));
  lsqr_launch_init_u(d, grid_, st_);
  lsqr_launch_adj(d, grid_, st_);
  lsqr_launch_fwd(d, grid_, st_);
  launches += 4;
  LCK(cudaGetLastError());
  // the iteration loop: a graph of kIterPerGraph (adj, fwd) pairs
  LCK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < kIterPerGraph; ++k) {
    lsqr_launch_adj(d, grid_, st_);
    lsqr_launch_fwd(d, grid_, st_);
  }
  LCK(cudaStreamEndCapture(st_, &r.graph));
  LCK(cudaGraphInstantiate(&r.exec, r.graph, 0));
  cudaGraphExec_t exec = r.exec;
  const int max_graphs = p.max_iter / kIterPerGraph + 2;
  std::string err;
  for (int gi = 0; gi <= max_graphs; ++gi) {
    LCK(cudaMemcpyAsync(h_sc_, sc_.p, sizeof(LsqrScalars), cudaMemcpyDeviceToHost, st_));
    LCK(cudaStreamSynchronize(st_));
    if (h_sc_->state == kLsDone) break;
    if (gi == max_graphs) { err = "LSQR did not terminate"; break; }
    LCK(cudaGraphLaunch(exec, st_));
    launches += 2 * kIterPerGraph;
  }
  cudaEventRecord(e1, st_);
  LCK(cudaMemcpyAsync(dm, dm_.p, (size_t)np_ * 8, cudaMemcpyDeviceToHost, st_));
  LCK(cudaStreamSynchronize(st_));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  last_ms_ = ms;
  last_launches_ = launches;
  if (!err.empty()) return err;
  if (out) {
    out->iters = h_sc_->iters_out;
    out->rnorm = h_sc_->rnorm;
    out->bnorm = h_sc_->bnorm;
    out->test2 = h_sc_->test2;
  }
  return std::string();
}


// ---------------------------------------------------------------- no-alloc solve
// LSQR for callers that cannot allocate device memory while they solve: a
// driver that overlaps this solve with work on other streams (cudaMalloc and
// cudaFree can synchronise the whole device and stall those streams), or a
// host program whose device memory is all reserved up front by its own pool
// allocator (a caching allocator or a Fortran driver's fixed arena), where a
// new cudaMalloc fails or fragments that reserve.  The work vectors live in
// one file-scope device array of kNoAllocBytes, which every GPU that loads
// the library holds until the process exits.  Every call shares it, so calls
// that overlap on the GPU (other host threads, other contexts of the same
// device) race on it; each call clears what has to start at zero.
namespace {

constexpr size_t kNoAllocDoubles = size_t(1) << 22;   // 32 MiB
constexpr size_t kNoAllocAlign = 32;                  // doubles (256 bytes)
constexpr size_t kNoAllocPart = 2048;                 // per-block partial sums

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {

std::mutex g_noalloc_mu;
struct NoAllocAddr {
  void* ctx = nullptr;    // CUcontext the address was looked up in
  void* ptr = nullptr;
};
NoAllocAddr g_noalloc_addr[256];

// CUcontext current on this thread (the driver call is reached through the
// runtime's entry-point query, so the library need not link the driver).
void* current_context() {
  typedef int (*CtxGetCurrent)(void**);
  static CtxGetCurrent fn = nullptr;
  static bool looked = false;
  if (!looked) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrent>(f);
    looked = true;
  }
  void* c = nullptr;
  if (fn) fn(&c);
  return c;
}

// Device address of the scratch array on `device` (which must be current).
// It is looked up with cudaGetSymbolAddress on the first call in a CUDA
// context of the device (in host code the array's name is only a host-side
// stand-in, so kernels must be given this address) and again whenever the
// device's context changed since (after cudaDeviceReset the module is loaded
// anew and the array may sit elsewhere).
std::string noalloc_scratch(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= 256) return "device ordinal out of range";
  void* ctx = current_context();
  NoAllocAddr& a = g_noalloc_addr[device];
  if (!a.ptr || ctx != a.ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e);
    a.ptr = p;
    a.ctx = current_context();
  }
  *out = static_cast<double*>(a.ptr);
  return std::string();
}

size_t round_up(size_t n) { return (n + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign; }

}  // namespace

std::string Lsqr::solve_noalloc(const LsqrParams& p, const double* residual, const double* gtg,
                                const double* dm_sum, double* dm, LsqrOut* out) {
  if (!rp_.p) return "no matrix set";
  if (!have_geom_) return "no model geometry for the smoothing operator";
  if (p.smooth_type != 1) return "smooth_type must be 1 (Laplacian)";
  if (p.max_iter < 1) return "max_iter must be >= 1";
  if (np_ != if_start_ + if_n_) return "matrix columns differ from the model's inversion parameters";
  if (!dm || (nd_ > 0 && !residual)) return "null device vector";
  if (grid_ > (int)kNoAllocPart) return "launch grid larger than the scratch partial-sum area";
  // scratch layout (doubles): scalars | partials | u | v | w | gtg | zeros | mask bytes
  const size_t o_sc = 0, o_part = kNoAllocAlign;
  const size_t o_u = o_part + kNoAllocPart;
  const size_t o_v = o_u + round_up((size_t)nd_ + 2 * (size_t)np_);
  const size_t o_w = o_v + round_up(np_);
  const size_t o_g = o_w + round_up(np_);
  const size_t o_z = o_g + round_up(np_);
  const size_t o_m = o_z + round_up(np_);
  const size_t need = o_m + round_up(((size_t)np_ + 7) / 8);
  if (need > kNoAllocDoubles)
    return "problem too large for the no-alloc scratch: needs " + std::to_string(need * 8) +
           " bytes (ndata + 6.125 nparm doubles plus 16.6 KB), the array holds " +
           std::to_string(kNoAllocDoubles * 8) + " bytes";
  cudaSetDevice(device_);
  double* S = nullptr;
  std::string e = noalloc_scratch(device_, &S);
  if (!e.empty()) return e;
  LsqrDev d = view();
  d.sc = reinterpret_cast<LsqrScalars*>(S + o_sc);
  d.part = S + o_part;
  d.u = S + o_u;
  d.v = S + o_v;
  d.w = S + o_w;
  d.dm = dm;
  d.mask = reinterpret_cast<uint8_t*>(S + o_m);
  d.residual = residual;
  d.ws_v = p.w_smooth;
  d.ws_i = p.w_smooth_iface;
  d.wd_v = p.wdv;
  d.wd_i = p.wdv_iface;
  d.max_iter = p.max_iter;
  if (!dm_sum) {
    LCK(cudaMemsetAsync(S + o_z, 0, (size_t)np_ * 8, st_));
    dm_sum = S + o_z;
  }
  d.dm_sum = dm_sum;
  if (!gtg) {
    lsqr_launch_gtg(d, S + o_g, grid_, st_);
    gtg = S + o_g;
  }
  lsqr_launch_mask(d, gtg, p.eps_min * 0.01, reinterpret_cast<uint8_t*>(S + o_m), grid_, st_);
  LCK(cudaMemsetAsync(dm, 0, (size_t)np_ * 8, st_));
  LCK(cudaMemsetAsync(d.sc, 0, sizeof(LsqrScalars), st_));
  lsqr_launch_init_u(d, grid_, st_);
  lsqr_launch_adj(d, grid_, st_);
  lsqr_launch_fwd(d, grid_, st_);
  LCK(cudaGetLastError());
  LsqrScalars hs;
  const int max_rounds = p.max_iter / kIterPerGraph + 2;
  for (int r = 0;; ++r) {
    LCK(cudaMemcpyAsync(&hs, d.sc, sizeof(LsqrScalars), cudaMemcpyDeviceToHost, st_));
    LCK(cudaStreamSynchronize(st_));
    if (hs.state == kLsDone) break;
    if (r == max_rounds) return "LSQR did not terminate";
    for (int k = 0; k < kIterPerGraph; ++k) {
      lsqr_launch_adj(d, grid_, st_);
      lsqr_launch_fwd(d, grid_, st_);
    }
    LCK(cudaGetLastError());
  }
  if (out) {
    out->iters = hs.iters_out;
    out->rnorm = hs.rnorm;
    out->bnorm = hs.bnorm;
    out->test2 = hs.test2;
  }
  return std::string();
}

}  // namespace fmt2d
