// Oracle LSQR products and solver (Laplacian smoothing variant).
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle.hpp"
#include "lsqr.hpp"
#include "smooth.hpp"
#include <algorithm>

namespace orc {

// inversion2d.f90:2997-3018 — y = G x over 1-based CSR.
void sparse_Ax(int ndata, int nparm, const int* gindx, const double* gval, const int* row_ptr,
               const double* x, double* y) {
  for (int i = 1; i <= ndata; ++i) {
    double acc = 0.0;
    for (int k = row_ptr[i - 1]; k <= row_ptr[i] - 1; ++k) {
      const int j = gindx[k - 1];
      if (j >= 1 && j <= nparm) acc = acc + gval[k - 1] * x[j - 1];
    }
    y[i - 1] = acc;
  }
}

// inversion2d.f90:3021-3042 — x = G^T y.
void sparse_ATx(int ndata, int nparm, const int* gindx, const double* gval, const int* row_ptr,
                const double* y, double* x) {
  for (int j = 0; j < nparm; ++j) x[j] = 0.0;
  for (int i = 1; i <= ndata; ++i)
    for (int k = row_ptr[i - 1]; k <= row_ptr[i] - 1; ++k) {
      const int j = gindx[k - 1];
      if (j >= 1 && j <= nparm) x[j - 1] = x[j - 1] + gval[k - 1] * y[i - 1];
    }
}

// inversion2d.f90:1161-1249 — 5-point Laplacian on the active velocity nodes
// plus the 1-D interface Laplacian (one-sided at the ends).
void laplacian(const LsqrGeom& G, int nparm, const double* vin, double* vout) {
  for (int j = 0; j < nparm; ++j) vout[j] = 0.0;
  auto I = [&](int ix, int iz) { return G.inv_idx[(ix - 1) + (size_t)(iz - 1) * G.nx]; };
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int ix = 1; ix <= G.nx; ++ix) {
      const int idx = I(ix, iz);
      if (idx <= 0) continue;
      int nb = 0;
      double acc = vout[idx - 1];
      if (ix > 1) { const int j = I(ix - 1, iz); if (j > 0) { acc += vin[j - 1]; ++nb; } }
      if (ix < G.nx) { const int j = I(ix + 1, iz); if (j > 0) { acc += vin[j - 1]; ++nb; } }
      if (iz > 1) { const int j = I(ix, iz - 1); if (j > 0) { acc += vin[j - 1]; ++nb; } }
      if (iz < G.nz) { const int j = I(ix, iz + 1); if (j > 0) { acc += vin[j - 1]; ++nb; } }
      vout[idx - 1] = acc - double(nb) * vin[idx - 1];
    }
  if (G.iface_nx > 0) {
    const int st = G.iface_start, nxi = G.iface_nx;
    for (int ix = 1; ix <= nxi; ++ix) {
      const int idx = st + ix;
      if (idx < 1 || idx > nparm) continue;
      if (ix == 1) {
        const int j = st + ix + 1;
        if (j <= nparm) vout[idx - 1] = vout[idx - 1] + vin[j - 1] - vin[idx - 1];
      } else if (ix == nxi) {
        const int j = st + ix - 1;
        if (j >= 1) vout[idx - 1] = vout[idx - 1] + vin[j - 1] - vin[idx - 1];
      } else {
        vout[idx - 1] = vout[idx - 1] + vin[st + ix - 2];
        vout[idx - 1] = vout[idx - 1] + vin[st + ix];
        vout[idx - 1] = vout[idx - 1] - 2.0 * vin[idx - 1];
      }
    }
  }
}

static double dot(const std::vector<double>& a) {
  double s = 0.0;
  for (double v : a) s += v * v;
  return s;
}

// inversion2d.f90:6578-7167, smooth_type = 1: LSQR on
// [G; w_s L; w_d I] dm = [r; -w_s L dm_sum; -w_d dm_sum] with inactive
// velocity columns (gtg < 0.01 eps_min) masked out.
LsqrResult run_lsqr_laplacian(const LsqrGeom& G, const LsqrInput& in, double* dm) {
  const int nd = in.ndata, np = in.nparm, nvp = in.n_vel_parms;
  const double thr = in.eps_min * 0.01;
  auto masked = [&](int j1) { return j1 <= nvp && in.gtg_diag[j1 - 1] < thr; };
  const bool smooth = in.w_smooth > 0.0 || in.w_smooth_iface > 0.0;
  const bool damp = in.wdv > 0.0 || in.wdv_iface > 0.0;
  const int na = nd + 2 * np;
  std::vector<double> u(na, 0.0), v(np), w(np), z(np), Av(na), Atu(np), so(np), sw(np);
  LsqrResult res{};
  for (int i = 0; i < nd; ++i) u[i] = in.residual[i];
  auto smooth_scale = [&](std::vector<double>& o) {
    for (int j = 1; j <= np; ++j) {
      if (j <= nvp) o[j - 1] = masked(j) ? 0.0 : in.w_smooth * o[j - 1];
      else o[j - 1] = in.w_smooth_iface * o[j - 1];
    }
  };
  if (smooth) {
    laplacian(G, np, in.dm_sum, so.data());
    smooth_scale(so);
    for (int j = 0; j < np; ++j) u[nd + j] = -so[j];
  }
  if (damp) {
    for (int j = 1; j <= np; ++j) {
      if (j <= nvp) u[nd + np + j - 1] = masked(j) ? 0.0 : -in.wdv * in.dm_sum[j - 1];
      else u[nd + np + j - 1] = -in.wdv_iface * in.dm_sum[j - 1];
    }
  }
  const double bnorm = std::sqrt(dot(u));
  res.bnorm = bnorm;
  for (int j = 0; j < np; ++j) dm[j] = 0.0;
  if (bnorm < 1.0e-30) return res;
  double beta = bnorm;
  for (double& x : u) x = x / beta;
  auto At = [&](const std::vector<double>& uu, std::vector<double>& out) {
    sparse_ATx(nd, np, in.gindx, in.gval, in.row_ptr, uu.data(), out.data());
    if (smooth) {
      for (int j = 0; j < np; ++j) sw[j] = uu[nd + j];
      laplacian(G, np, sw.data(), so.data());
      smooth_scale(so);
      for (int j = 0; j < np; ++j) out[j] = out[j] + so[j];
    }
    if (damp) {
      for (int j = 1; j <= np; ++j) {
        if (j <= nvp) { if (!masked(j)) out[j - 1] = out[j - 1] + in.wdv * uu[nd + np + j - 1]; }
        else out[j - 1] = out[j - 1] + in.wdv_iface * uu[nd + np + j - 1];
      }
    }
  };
  At(u, v);
  for (int j = 1; j <= np; ++j) if (masked(j)) v[j - 1] = 0.0;
  double alpha = std::sqrt(dot(v));
  if (alpha < 1.0e-30) { res.rnorm = bnorm; return res; }
  for (double& x : v) x = x / alpha;
  w = v;
  double phibar = beta, rhobar = alpha, anorm2 = alpha * alpha + beta * beta;
  const double atol = 1.0e-4;
  int it;
  for (it = 1; it <= in.max_iter; ++it) {
    for (int j = 1; j <= np; ++j) if (masked(j)) v[j - 1] = 0.0;
    sparse_Ax(nd, np, in.gindx, in.gval, in.row_ptr, v.data(), Av.data());
    if (smooth) {
      laplacian(G, np, v.data(), so.data());
      smooth_scale(so);
      for (int j = 0; j < np; ++j) Av[nd + j] = so[j];
    } else {
      for (int j = 0; j < np; ++j) Av[nd + j] = 0.0;
    }
    for (int j = 1; j <= np; ++j) {
      double val = 0.0;
      if (damp) {
        if (j <= nvp) val = masked(j) ? 0.0 : in.wdv * v[j - 1];
        else val = in.wdv_iface * v[j - 1];
      }
      Av[nd + np + j - 1] = val;
    }
    for (int i = 0; i < na; ++i) u[i] = Av[i] - alpha * u[i];
    beta = std::sqrt(dot(u));
    if (beta > 0.0) for (double& x : u) x = x / beta;
    At(u, Atu);
    for (int j = 0; j < np; ++j) v[j] = Atu[j] - beta * v[j];
    for (int j = 1; j <= np; ++j) if (masked(j)) v[j - 1] = 0.0;
    alpha = std::sqrt(dot(v));
    if (alpha > 0.0) for (double& x : v) x = x / alpha;
    anorm2 = anorm2 + alpha * alpha + beta * beta;
    const double rho = std::sqrt(rhobar * rhobar + beta * beta);
    const double c = rhobar / rho, s = beta / rho;
    const double theta = s * alpha;
    rhobar = -c * alpha;
    const double phi = c * phibar;
    phibar = s * phibar;
    z = w;
    for (int j = 1; j <= np; ++j) if (masked(j)) z[j - 1] = 0.0;
    for (int j = 0; j < np; ++j) w[j] = v[j] - (theta / rho) * w[j];
    for (int j = 1; j <= np; ++j) if (masked(j)) w[j - 1] = 0.0;
    for (int j = 0; j < np; ++j) dm[j] = dm[j] + (phi / rho) * z[j];
    res.rnorm = std::fabs(phibar);
    const double arnorm = phibar * alpha * std::fabs(c);
    res.test2 = arnorm / (std::sqrt(anorm2) * res.rnorm + 1.0e-30);
    if (res.test2 < atol) break;
    if (1.0 + res.test2 <= 1.0) break;
  }
  res.iters = it;  // like a Fortran DO index: max_iter+1 when no exit
  return res;
}

// inversion2d.f90:6578-7167 for smooth_type 1, 2 and 3: the same
// Golub-Kahan iteration as run_lsqr_laplacian over the augmented operator of
// the chosen layout.  The interface Gaussian's adjoint is the matrix itself,
// as the reference applies it (:6826-6833, :7100-7106).
LsqrResult run_lsqr_general(const LsqrGeom& G, const LsqrInput& in, int smooth_type,
                            const Csr* rh, const Csr* rv, const Csr* ri, double* dm) {
  const int nd = in.ndata, np = in.nparm, nvp = in.n_vel_parms;
  const double thr = in.eps_min * 0.01;
  auto masked = [&](int j1) { return j1 <= nvp && in.gtg_diag[j1 - 1] < thr; };
  const bool gauss = smooth_type == 2;
  const bool smooth = gauss ? in.w_smooth > 0.0 : (in.w_smooth > 0.0 || in.w_smooth_iface > 0.0);
  const bool ri_built = ri && !ri->col.empty();
  const bool damp = in.wdv > 0.0 || in.wdv_iface > 0.0;
  const int db = gauss ? nd + 2 * np : nd + np;        // damping block
  const int na = db + np;
  std::vector<double> u(na, 0.0), v(np), w(np), z(np), Av(na), Atu(np), so(np), sw(np),
      sh(np), sv(np);
  LsqrResult res{};
  // the smoothing block(s) of A x, written into out[nd ..]
  auto smooth_fwd = [&](const double* x, std::vector<double>& out) {
    if (smooth_type == 2) {
      if (smooth) {
        csr_apply(*rh, np, x, sh.data(), false);
        csr_apply(*rv, np, x, sv.data(), false);
        for (int j = 1; j <= np; ++j)
          if (masked(j)) { sh[j - 1] = 0.0; sv[j - 1] = 0.0; }
        for (int j = 0; j < np; ++j) { out[nd + j] = in.w_smooth * sh[j]; out[nd + np + j] = in.w_smooth * sv[j]; }
      } else {
        for (int j = 0; j < 2 * np; ++j) out[nd + j] = 0.0;
      }
      if (in.w_smooth_iface > 0.0 && ri_built) {
        csr_apply(*ri, np, x, sh.data(), false);
        for (int j = nvp + 1; j <= np; ++j) out[nd + j - 1] = in.w_smooth_iface * sh[j - 1];
      } else {
        for (int j = nvp + 1; j <= np; ++j) out[nd + j - 1] = 0.0;
      }
      return;
    }
    if (!smooth) { for (int j = 0; j < np; ++j) out[nd + j] = 0.0; return; }
    laplacian(G, np, x, so.data());
    for (int j = 1; j <= nvp; ++j) so[j - 1] = masked(j) ? 0.0 : in.w_smooth * so[j - 1];
    if (smooth_type == 1) {
      for (int j = nvp + 1; j <= np; ++j) so[j - 1] = in.w_smooth_iface * so[j - 1];
    } else if (in.w_smooth_iface > 0.0) {
      csr_apply(*ri, np, x, sh.data(), false);
      for (int j = nvp + 1; j <= np; ++j) so[j - 1] = in.w_smooth_iface * sh[j - 1];
    } else {
      for (int j = nvp + 1; j <= np; ++j) so[j - 1] = 0.0;
    }
    for (int j = 0; j < np; ++j) out[nd + j] = so[j];
  };
  // right-hand side: residual, minus the smoothing of dm_sum, minus the damping
  for (int i = 0; i < nd; ++i) u[i] = in.residual[i];
  smooth_fwd(in.dm_sum, u);
  for (int j = nd; j < db; ++j) u[j] = -u[j];
  if (damp) {
    for (int j = 1; j <= np; ++j) {
      if (j <= nvp) u[db + j - 1] = masked(j) ? 0.0 : -in.wdv * in.dm_sum[j - 1];
      else u[db + j - 1] = -in.wdv_iface * in.dm_sum[j - 1];
    }
  }
  const double bnorm = std::sqrt(dot(u));
  res.bnorm = bnorm;
  for (int j = 0; j < np; ++j) dm[j] = 0.0;
  if (bnorm < 1.0e-30) return res;
  double beta = bnorm;
  for (double& x : u) x = x / beta;
  auto At = [&](const std::vector<double>& uu, std::vector<double>& out) {
    sparse_ATx(nd, np, in.gindx, in.gval, in.row_ptr, uu.data(), out.data());
    if (smooth_type == 2) {
      if (smooth) {
        csr_apply(*rh, np, uu.data() + nd, sh.data(), true);
        csr_apply(*rv, np, uu.data() + nd + np, sv.data(), true);
        for (int j = 1; j <= np; ++j)
          if (masked(j)) { sh[j - 1] = 0.0; sv[j - 1] = 0.0; }
        for (int j = 0; j < np; ++j) out[j] = out[j] + in.w_smooth * sh[j] + in.w_smooth * sv[j];
      }
      if (in.w_smooth_iface > 0.0 && ri_built) {
        csr_apply(*ri, np, uu.data() + nd, so.data(), false);
        for (int j = nvp + 1; j <= np; ++j) out[j - 1] = out[j - 1] + in.w_smooth_iface * so[j - 1];
      }
    } else if (smooth) {
      for (int j = 0; j < np; ++j) sw[j] = uu[nd + j];
      laplacian(G, np, sw.data(), so.data());
      for (int j = 1; j <= nvp; ++j) so[j - 1] = masked(j) ? 0.0 : in.w_smooth * so[j - 1];
      if (smooth_type == 1) {
        for (int j = nvp + 1; j <= np; ++j) so[j - 1] = in.w_smooth_iface * so[j - 1];
      } else if (in.w_smooth_iface > 0.0) {
        csr_apply(*ri, np, sw.data(), sh.data(), false);
        for (int j = nvp + 1; j <= np; ++j) so[j - 1] = in.w_smooth_iface * sh[j - 1];
      } else {
        for (int j = nvp + 1; j <= np; ++j) so[j - 1] = 0.0;
      }
      for (int j = 0; j < np; ++j) out[j] = out[j] + so[j];
    }
    if (damp) {
      for (int j = 1; j <= np; ++j) {
        if (j <= nvp) { if (!masked(j)) out[j - 1] = out[j - 1] + in.wdv * uu[db + j - 1]; }
        else out[j - 1] = out[j - 1] + in.wdv_iface * uu[db + j - 1];
      }
    }
  };
  At(u, v);
  for (int j = 1; j <= np; ++j) if (masked(j)) v[j - 1] = 0.0;
  double alpha = std::sqrt(dot(v));
  if (alpha < 1.0e-30) { res.rnorm = bnorm; return res; }
  for (double& x : v) x = x / alpha;
  w = v;
  double phibar = beta, rhobar = alpha, anorm2 = alpha * alpha + beta * beta;
  const double atol = 1.0e-4;
  int it;
  for (it = 1; it <= in.max_iter; ++it) {
    for (int j = 1; j <= np; ++j) if (masked(j)) v[j - 1] = 0.0;
    sparse_Ax(nd, np, in.gindx, in.gval, in.row_ptr, v.data(), Av.data());
    smooth_fwd(v.data(), Av);
    for (int j = 1; j <= np; ++j) {
      double val = 0.0;
      if (damp) {
        if (j <= nvp) val = masked(j) ? 0.0 : in.wdv * v[j - 1];
        else val = in.wdv_iface * v[j - 1];
      }
      Av[db + j - 1] = val;
    }
    for (int i = 0; i < na; ++i) u[i] = Av[i] - alpha * u[i];
    beta = std::sqrt(dot(u));
    if (beta > 0.0) for (double& x : u) x = x / beta;
    At(u, Atu);
    for (int j = 0; j < np; ++j) v[j] = Atu[j] - beta * v[j];
    for (int j = 1; j <= np; ++j) if (masked(j)) v[j - 1] = 0.0;
    alpha = std::sqrt(dot(v));
    if (alpha > 0.0) for (double& x : v) x = x / alpha;
    anorm2 = anorm2 + alpha * alpha + beta * beta;
    const double rho = std::sqrt(rhobar * rhobar + beta * beta);
    const double c = rhobar / rho, s = beta / rho;
    const double theta = s * alpha;
    rhobar = -c * alpha;
    const double phi = c * phibar;
    phibar = s * phibar;
    z = w;
    for (int j = 1; j <= np; ++j) if (masked(j)) z[j - 1] = 0.0;
    for (int j = 0; j < np; ++j) w[j] = v[j] - (theta / rho) * w[j];
    for (int j = 1; j <= np; ++j) if (masked(j)) w[j - 1] = 0.0;
    for (int j = 0; j < np; ++j) dm[j] = dm[j] + (phi / rho) * z[j];
    res.rnorm = std::fabs(phibar);
    const double arnorm = phibar * alpha * std::fabs(c);
    res.test2 = arnorm / (std::sqrt(anorm2) * res.rnorm + 1.0e-30);
    if (res.test2 < atol) break;
    if (1.0 + res.test2 <= 1.0) break;
  }
  res.iters = it;
  return res;
}

}  // namespace orc
