// Oracle ray backtrace, water-leg entry search and Frechet rows.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle.hpp"
#include <algorithm>

namespace orc {

// rays2d.f90:1222-1257
double interpolate_interface2d(const Model& m, double px, const Isec& is) {
  if (is.nnode < 1) return 0.0;
  if (is.nnode < 2) return is.z[1];
  const int ix = (int)std::floor((px - is.x[1]) / m.grid.dx) + 1;
  if (ix < 1) return is.z[1];
  if (ix >= is.nnode) return is.z[is.nnode];
  double w = (px - is.x[ix]) / m.grid.dx;
  w = std::min(1.0, std::max(0.0, w));
  return (1.0 - w) * is.z[ix] + w * is.z[ix + 1];
}

// rays2d.f90:1261-1306
void interface_normal2d(const Model& m, double px, const Isec& is, double& nx, double& nz,
                        double& h) {
  const double dx = m.grid.dx;
  if (is.nnode < 2) { nx = 0.0; nz = 1.0; h = is.z[1]; return; }
  int ix = (int)std::floor((px - is.x[1]) / dx) + 1;
  if (ix < 1) ix = 1;
  if (ix >= is.nnode) ix = is.nnode - 1;
  double w = std::min(1.0, std::max(0.0, (px - is.x[ix]) / dx));
  h = (1.0 - w) * is.z[ix] + w * is.z[ix + 1];
  double dzdx;
  if (ix > 1 && ix < is.nnode - 1) dzdx = (is.z[ix + 1] - is.z[ix - 1]) / (2.0 * dx);
  else if (ix == 1 && is.nnode >= 3) dzdx = (is.z[ix + 1] - is.z[ix]) / dx;
  else if (ix == is.nnode - 1 && is.nnode >= 3) dzdx = (is.z[ix + 1] - is.z[ix - 1]) / (2.0 * dx);
  else dzdx = 0.0;
  const double l = std::sqrt(1.0 + dzdx * dzdx);
  nx = -dzdx / l;
  nz = 1.0 / l;
}

static int find_region_node(const Model& m, const Region& r, int ix, int iz) {
  if (ix >= 1 && ix <= m.grid.nx && iz >= 1 && iz <= m.grid.nz) {
    const int n = r.rid[m.grid.g(ix, iz)];
    return (n <= 0 || n > r.nnode) ? 0 : n;
  }
  return 0;
}

// rays2d.f90:996-1020 — the nearest region node in the same column, up to
// five rows away (below first).
static int find_nearby_region_node(const Model& m, const Region& r, int ix, int iz) {
  for (int d = 1; d <= 5; ++d) {
    int iz2 = iz + d;
    if (iz2 >= 1 && iz2 <= m.grid.nz && ix >= 1 && ix <= m.grid.nx) {
      const int n = r.rid[m.grid.g(ix, iz2)];
      if (n > 0 && n <= r.nnode) return n;
    }
    iz2 = iz - d;
    if (iz2 >= 1 && iz2 <= m.grid.nz && ix >= 1 && ix <= m.grid.nx) {
      const int n = r.rid[m.grid.g(ix, iz2)];
      if (n > 0 && n <= r.nnode) return n;
    }
  }
  return 0;
}

// rays2d.f90:1070-1131
static int find_position_in_region2d(const Model& m, const Region& r, double px, double pz) {
  const Grid& g = m.grid;
  int ix = (int)std::floor((px - g.x0) / g.dx) + 1;
  int iz = (int)std::floor((pz - g.z0) / g.dz) + 1;
  ix = std::max(1, std::min(g.nx - 1, ix));
  iz = std::max(1, std::min(g.nz - 1, iz));
  double dmin = 1.0e100;
  int best = 0;
  for (int ii = ix; ii <= ix + 1; ++ii)
    for (int jj = iz; jj <= iz + 1; ++jj) {
      const int mm = r.rid[g.g(ii, jj)];
      if (mm > 0 && mm <= r.nnode) {
        const double d = (px - r.x[mm]) * (px - r.x[mm]) + (pz - r.z[mm]) * (pz - r.z[mm]);
        if (d < dmin) { best = mm; dmin = d; }
      }
    }
  if (best == 0) {
    dmin = 1.0e100;
    for (int mm = 1; mm <= r.nnode; ++mm) {
      const double d = (px - r.x[mm]) * (px - r.x[mm]) + (pz - r.z[mm]) * (pz - r.z[mm]);
      if (d < dmin) { best = mm; dmin = d; }
    }
  }
  return best;
}

// rays2d.f90:825-894 (+ interpolate_gradient_reg :1037-1066)
void interpolate_time_gradient2d(const Model& m, const Region& r, const double* gxv,
                                 const double* gzv, double px, double pz, double& dtdx,
                                 double& dtdz) {
  const Grid& g = m.grid;
  int ix = (int)std::floor((px - g.x0) / g.dx) + 1;
  int iz = (int)std::floor((pz - g.z0) / g.dz) + 1;
  ix = std::max(1, std::min(g.nx - 1, ix));
  iz = std::max(1, std::min(g.nz - 1, iz));
  const double w1 = std::min(1.0, std::max(0.0, (px - g.x[ix]) / g.dx));
  const double w2 = std::min(1.0, std::max(0.0, (pz - g.z[iz]) / g.dz));
  int n1 = find_region_node(m, r, ix, iz), n2 = find_region_node(m, r, ix + 1, iz);
  int n3 = find_region_node(m, r, ix, iz + 1), n4 = find_region_node(m, r, ix + 1, iz + 1);
  if (n1 == 0) n1 = find_nearby_region_node(m, r, ix, iz);
  if (n2 == 0) n2 = find_nearby_region_node(m, r, ix + 1, iz);
  if (n3 == 0) n3 = find_nearby_region_node(m, r, ix, iz + 1);
  if (n4 == 0) n4 = find_nearby_region_node(m, r, ix + 1, iz + 1);
  double g1x = 0, g2x = 0, g3x = 0, g4x = 0, g1z = 0, g2z = 0, g3z = 0, g4z = 0;
  if (n1 > 0) { g1x = gxv[n1]; g1z = gzv[n1]; }
  if (n2 > 0) { g2x = gxv[n2]; g2z = gzv[n2]; }
  if (n3 > 0) { g3x = gxv[n3]; g3z = gzv[n3]; }
  if (n4 > 0) { g4x = gxv[n4]; g4z = gzv[n4]; }
  double gx = (1.0 - w1) * (1.0 - w2) * g1x + w1 * (1.0 - w2) * g2x + (1.0 - w1) * w2 * g3x +
              w1 * w2 * g4x;
  double gz = (1.0 - w1) * (1.0 - w2) * g1z + w1 * (1.0 - w2) * g2z + (1.0 - w1) * w2 * g3z +
              w1 * w2 * g4z;
  if (std::sqrt(gx * gx + gz * gz) < 0.01) {
    const int nm = find_position_in_region2d(m, r, px, pz);
    gx = 0.0; gz = 0.0;
    if (nm > 0) { gx = gxv[nm]; gz = gzv[nm]; }
  }
  dtdx = gx;
  dtdz = gz;
}

// rays2d.f90:898-975
double interpolate_arrivaltime2d(const Model& m, const Region& r, const double* T, double px,
                                 double pz) {
  const Grid& g = m.grid;
  int ix = (int)std::floor((px - g.x0) / g.dx) + 1;
  int iz = (int)std::floor((pz - g.z0) / g.dz) + 1;
  ix = std::max(1, std::min(g.nx - 1, ix));
  iz = std::max(1, std::min(g.nz - 1, iz));
  const double w1 = std::min(1.0, std::max(0.0, (px - g.x[ix]) / g.dx));
  const double w2 = std::min(1.0, std::max(0.0, (pz - g.z[iz]) / g.dz));
  const int n1 = find_region_node(m, r, ix, iz), n2 = find_region_node(m, r, ix + 1, iz);
  const int n3 = find_region_node(m, r, ix, iz + 1), n4 = find_region_node(m, r, ix + 1, iz + 1);
  auto tn = [&](int n, int a, int b) {
    if (n > 0) return T[n];
    const int q = find_nearby_region_node(m, r, a, b);
    return (q > 0 && q <= r.nnode) ? T[q] : kHugeTime;
  };
  const double t1 = tn(n1, ix, iz), t2 = tn(n2, ix + 1, iz);
  const double t3 = tn(n3, ix, iz + 1), t4 = tn(n4, ix + 1, iz + 1);
  const double hh = kHugeTime * 0.5;
  if (t1 < hh && t2 < hh && t3 < hh && t4 < hh)
    return (1.0 - w1) * (1.0 - w2) * t1 + w1 * (1.0 - w2) * t2 + (1.0 - w1) * w2 * t3 +
           w1 * w2 * t4;
  double t = kHugeTime, dmin = kHugeTime;
  for (int n = 1; n <= r.nnode; ++n) {
    const double d = (px - r.x[n]) * (px - r.x[n]) + (pz - r.z[n]) * (pz - r.z[n]);
    if (d < dmin) { dmin = d; t = T[n]; }
  }
  return t;
}

// rays2d.f90:1310-1350 (grid velocity is associated, so it is bilinear on it)
static double get_velocity_at2d(const Model& m, double px, double pz) {
  const Grid& g = m.grid;
  int ix = (int)std::floor((px - g.x0) / g.dx) + 1;
  int iz = (int)std::floor((pz - g.z0) / g.dz) + 1;
  ix = std::max(1, std::min(g.nx - 1, ix));
  iz = std::max(1, std::min(g.nz - 1, iz));
  const double w1 = std::min(1.0, std::max(0.0, (px - g.x[ix]) / g.dx));
  const double w2 = std::min(1.0, std::max(0.0, (pz - g.z[iz]) / g.dz));
  auto V = [&](int a, int b) { return g.vel[g.g(a, b)]; };
  return (1.0 - w1) * (1.0 - w2) * V(ix, iz) + w1 * (1.0 - w2) * V(ix + 1, iz) +
         (1.0 - w1) * w2 * V(ix, iz + 1) + w1 * w2 * V(ix + 1, iz + 1);
}

namespace {

struct SecCtx {
  Model* m;
  Source* s;
  Ray* ray;
  int seqnum;
};

// rays2d.f90:764-821
static bool find_interface_crossing2d(const Model& m, std::vector<double>& X,
                                      std::vector<double>& Z, int n, double ppx, double ppz,
                                      const Isec& ie, double g0x, double g0z, double dl) {
  const double tol = 0.01 * m.grid.tolerance;
  const double zi = interpolate_interface2d(m, ppx, ie);
  const double x1 = 0.0, x2 = dl;
  const double f = Z[n - 1] - interpolate_interface2d(m, X[n - 1], ie);
  double fmid = ppz - zi;
  if (f * fmid > tol) return false;
  if (std::fabs(f * fmid) <= tol) {
    X[n] = X[n - 1];
    Z[n] = interpolate_interface2d(m, X[n], ie);
    return true;
  }
  if (f * fmid < -tol) {
    double rtbis, dx;
    if (f < 0.0) { rtbis = x1; dx = x2 - x1; }
    else { rtbis = x2; dx = x1 - x2; }
    for (int k = 1; k <= 10; ++k) {
      dx *= 0.5;
      const double xm = rtbis + dx;
      X[n] = X[n - 1] - xm * g0x;
      Z[n] = Z[n - 1] - xm * g0z;
      fmid = Z[n] - interpolate_interface2d(m, X[n], ie);
      if (fmid <= 0.0) rtbis = xm;
    }
    X[n] = X[n - 1] - rtbis * g0x;
    Z[n] = Z[n - 1] - rtbis * g0z;
    Z[n] = interpolate_interface2d(m, X[n], ie);
  }
  return true;
}

// rays2d.f90:157-720
static void trace_ray_section2d(Model& m, Source& s, Ray& ray, int seqnum, double x_in,
                                double z_in, double& x_out, double& z_out) {
  RaySection& rs = ray.sec[seqnum];
  const TField& tf = s.tf[rs.tf];
  const Region& reg = m.reg[tf.reg];
  const Isec& iftop = m.isec[reg.itop];
  const Isec& ifbot = m.isec[reg.ibot];
  const Grid& g = m.grid;
  const double v_average = 5.0;
  const int maxpoints = 5000;
  bool refraction = false;
  int start_direction = 0;
  const Isec* ifend = nullptr;
  int ifend_id = 0;
  const TField* tf_next = nullptr;
  const int nsec = ray.nsections;
  if (seqnum < nsec && seqnum > 1) {
    ifend_id = rs.iend;
    ifend = &m.isec[ifend_id];
    tf_next = &s.tf[ray.sec[seqnum - 1].tf];
    start_direction = reg.id - m.reg[s.tf[ray.sec[seqnum + 1].tf].reg].id;
    refraction = m.reg[tf_next->reg].id != reg.id;
  }
  if (seqnum == nsec && seqnum > 1) {
    ifend_id = rs.iend;
    ifend = &m.isec[ifend_id];
    tf_next = &s.tf[ray.sec[seqnum - 1].tf];
    start_direction = 0;
    refraction = m.reg[tf_next->reg].id != reg.id;
  }
  if (seqnum == 1) {
    ifend = nullptr;
    ifend_id = 0;
    tf_next = nullptr;
    start_direction = (seqnum + 1 <= nsec) ? reg.id - m.reg[s.tf[ray.sec[seqnum + 1].tf].reg].id : 0;
  }
  bool same_internal = false, left_start = true;
  if (ifend && rs.istart) {
    same_internal = (ifend->id == rs.istart && ifend->id != iftop.id && ifend->id != ifbot.id);
    if (same_internal) left_start = false;
  }
  const double dlmax = 0.1 * g.dx * v_average;
  const double p_tol = 5.0e-4 * g.dx;
  const double s_tol = 2.5 * g.dx;
  std::vector<double> X(maxpoints + 2), Z(maxpoints + 2);  // 1-based
  int n = 1;
  X[1] = x_in;
  Z[1] = z_in;
  double dist_hw = 0.0;
  const bool on_bot = std::fabs(z_in - interpolate_interface2d(m, x_in, ifbot)) < 0.1 * g.dz;
  const bool on_top = std::fabs(z_in - interpolate_interface2d(m, x_in, iftop)) < 0.1 * g.dz;
  const Region* nreg = tf_next ? &m.reg[tf_next->reg] : nullptr;
  auto grad_at = [&](double px, double pz, double& gx, double& gz) {
    interpolate_time_gradient2d(m, reg, tf.gx.data(), tf.gz.data(), px, pz, gx, gz);
  };
  auto grad_next = [&](double px, double pz, double& gx, double& gz) {
    interpolate_time_gradient2d(m, *nreg, tf_next->gx.data(), tf_next->gz.data(), px, pz, gx, gz);
  };
  auto finish = [&](int npts) {
    rs.px.assign(X.begin() + 1, X.begin() + 1 + npts);
    rs.pz.assign(Z.begin() + 1, Z.begin() + 1 + npts);
  };
  auto near_src = [&](int k) {
    const double dx = X[k] - s.x, dz = Z[k] - s.z;
    return std::sqrt(dx * dx + dz * dz) < s_tol;
  };
  // refraction test at an interface point: true = refract (end section)
  auto refracts = [&](double px, double zi, double& g0x, double& g0z) {
    double nx, nz, h;
    interface_normal2d(m, px, m.isec[ifend_id], nx, nz, h);
    double g1x, g1z;
    grad_at(px, zi, g0x, g0z);
    grad_next(px, zi, g1x, g1z);
    const double d = nx * g1x + nz * g1z;
    const double tx = g1x - d * nx, tz = g1z - d * nz;
    return std::sqrt(tx * tx + tz * tz) <= std::sqrt(g0x * g0x + g0z * g0z);
  };
  double g0x = 0, g0z = 0, g1x = 0, g1z = 0, ppx = 0, ppz = 0, dl = dlmax;
  for (;;) {  // ploop
    ++n;
    if (n > maxpoints) { ray.valid = false; return; }
    if (seqnum == 1 && n > 2 && near_src(n - 1)) {
      X[n] = s.x; Z[n] = s.z; finish(n); return;
    }
    if (ray.headwave || ray.diffracted) {
      if (n > 2) {
        const double ddx = X[n - 1] - X[n - 2], ddz = Z[n - 1] - Z[n - 2];
        dist_hw += std::sqrt(ddx * ddx + ddz * ddz);
      }
      if (dist_hw > 200.0) { ray.valid = false; return; }
    }
    dl = dlmax;
    if (n == 2 && (on_bot || on_top)) dl = 10.0 * dlmax;
    grad_at(X[n - 1], Z[n - 1], g0x, g0z);
    ppx = X[n - 1] - dl * g0x;
    ppz = Z[n - 1] - dl * g0z;
    if (on_bot && ppz > Z[n - 1]) ppz = 2.0 * Z[n - 1] - ppz;
    if (on_top && ppz < Z[n - 1]) ppz = 2.0 * Z[n - 1] - ppz;
    if (n == 2 && start_direction != 0 && !refraction && seqnum != 1) {
      double nx, nz, h;
      interface_normal2d(m, x_in, m.isec[rs.istart], nx, nz, h);
      if (g0x * start_direction * nx + g0z * start_direction * nz > 0.0) { ray.valid = false; return; }
    }
    if (ifend && ifend->id != iftop.id && ifend->id != ifbot.id) {
      const double fp = Z[n - 1] - interpolate_interface2d(m, X[n - 1], *ifend);
      const double fn = ppz - interpolate_interface2d(m, ppx, *ifend);
      if (same_internal && !left_start) {
        if (std::fabs(fn) > 0.5 * g.dz) left_start = true;
      } else if (std::fabs(fp) > 1.0e-3) {
        if (fp * fn <= 0.0) {
          double fr = std::fabs(fp - fn) > 1.0e-12 ? fp / (fp - fn) : 1.0;
          fr = std::min(1.0, std::max(0.0, fr));
          X[n] = X[n - 1] + fr * (ppx - X[n - 1]);
          Z[n] = interpolate_interface2d(m, X[n], *ifend);
          if (seqnum == 1 && near_src(n)) { X[n] = s.x; Z[n] = s.z; }
          finish(n);
          return;
        }
      }
    }
    bool exit_ploop = false, cycle_ploop = false;
    // top interface against the straight step
    {
      const double zi = interpolate_interface2d(m, ppx, iftop);
      if (ppz <= zi) {
        if (iftop.id == ifend_id) {
          if (refraction) {
            if (refracts(ppx, zi, g0x, g0z)) {
              exit_ploop = true;
            } else {
              X[n] = ppx; Z[n] = zi;
              rs.headwave = true; ray.headwave = true;
              if (seqnum == 1 && near_src(n)) { X[n] = s.x; Z[n] = s.z; finish(n); return; }
              cycle_ploop = true;
            }
          } else {
            exit_ploop = true;
          }
        } else if (n == 2 && on_top && rs.istart && rs.istart == iftop.id) {
          // no-op: fall through to the bottom test
        } else {
          X[n] = ppx; Z[n] = zi;
          rs.diffracted = true; ray.diffracted = true;
          if (seqnum == 1 && near_src(n)) { X[n] = s.x; Z[n] = s.z; finish(n); return; }
          cycle_ploop = true;
        }
      }
    }
    if (exit_ploop) break;
    if (cycle_ploop) continue;
    {
      const double zi = interpolate_interface2d(m, ppx, ifbot);
      if (ppz >= zi) {
        if (ifbot.id == ifend_id) {
          if (refraction) {
            if (ray.raypath_id == 4 && seqnum == 2) {
              exit_ploop = true;
            } else if (refracts(ppx, zi, g0x, g0z)) {
              exit_ploop = true;
            } else {
              X[n] = ppx; Z[n] = zi;
              rs.headwave = true; ray.headwave = true;
              if (seqnum == 1 && near_src(n)) { X[n] = s.x; Z[n] = s.z; finish(n); return; }
              cycle_ploop = true;
            }
          } else {
            exit_ploop = true;
          }
        } else if (n == 2 && on_bot && rs.istart && rs.istart == ifbot.id) {
        } else {
          X[n] = ppx; Z[n] = zi;
          rs.diffracted = true; ray.diffracted = true;
          if (seqnum == 1 && near_src(n)) { X[n] = s.x; Z[n] = s.z; finish(n); return; }
          cycle_ploop = true;
        }
      }
    }
    if (exit_ploop) break;
    if (cycle_ploop) continue;
    int iter = 1;
    for (;;) {  // itloop: Heun step with step halving
      ppx = X[n - 1] - dl * g0x;
      ppz = Z[n - 1] - dl * g0z;
      grad_at(ppx, ppz, g1x, g1z);
      X[n] = X[n - 1] - dl * (g0x + g1x) * 0.5;
      Z[n] = Z[n - 1] - dl * (g0z + g1z) * 0.5;
      {
        const double zi = interpolate_interface2d(m, X[n], iftop);
        if (Z[n] <= zi) {
          if (iftop.id == ifend_id) {
            if (refraction) {
              if (refracts(X[n], zi, g0x, g0z)) {
                ppx = X[n]; ppz = Z[n];
                exit_ploop = true;
              } else {
                Z[n] = zi;
                rs.headwave = true; ray.headwave = true;
                cycle_ploop = true;
              }
            } else {
              ppx = X[n]; ppz = Z[n];
              exit_ploop = true;
            }
          } else if (n == 2 && on_top && rs.istart && rs.istart == iftop.id) {
          } else {
            Z[n] = zi;
            rs.diffracted = true; ray.diffracted = true;
            cycle_ploop = true;
          }
        }
      }
      if (exit_ploop || cycle_ploop) break;
      {
        const double zi = interpolate_interface2d(m, X[n], ifbot);
        if (Z[n] >= zi) {
          if (ifbot.id == ifend_id) {
            if (refraction) {
              if (ray.raypath_id == 4 && seqnum == 2) {
                ppx = X[n]; ppz = Z[n];
                exit_ploop = true;
              } else if (refracts(X[n], zi, g0x, g0z)) {
                ppx = X[n]; ppz = Z[n];
                exit_ploop = true;
              } else {
                Z[n] = zi;
                rs.headwave = true; ray.headwave = true;
                cycle_ploop = true;
              }
            } else {
              ppx = X[n]; ppz = Z[n];
              exit_ploop = true;
            }
          } else if (n == 2 && on_bot && rs.istart && rs.istart == ifbot.id) {
          } else {
            Z[n] = zi;
            rs.diffracted = true; ray.diffracted = true;
            cycle_ploop = true;
          }
        }
      }
      if (exit_ploop || cycle_ploop) break;
      const double ex = X[n] - ppx, ez = Z[n] - ppz;
      if (std::sqrt(ex * ex + ez * ez) < p_tol) break;
      ++iter;
      if (iter > 10) { ray.valid = false; return; }
      dl = 0.5 * dl;
    }
    if (exit_ploop) break;
    if (cycle_ploop) continue;
    if (seqnum == 1 && near_src(n)) { X[n] = s.x; Z[n] = s.z; finish(n); return; }
  }
  if (seqnum == 1) { ray.valid = false; return; }
  if (ifend) {
    if (!find_interface_crossing2d(m, X, Z, n, ppx, ppz, *ifend, g0x, g0z, dl)) {
      ray.valid = false;
      return;
    }
  }
  x_out = X[n];
  z_out = Z[n];
  finish(n);
}

}  // namespace

// rays2d.f90:7-153
void trace_ray_from_receiver2d(Model& m, Source& s, double rx, double rz, Ray& ray) {
  const Path& P = m.path[ray.raypath_id];
  const int ns = P.n_tf;
  ray.nsections = ns;
  ray.sec.assign(ns + 1, RaySection());
  for (int n = ns; n >= 1; --n) {
    RaySection& rs = ray.sec[n];
    rs.place = n;
    rs.tf = P.tf_sequence[n];
    if (!s.tf[rs.tf].solved) { ray.valid = false; return; }
    rs.reg = s.tf[rs.tf].reg;
    rs.istart = (n < ns) ? P.sequence[2 * n] : 0;
    rs.iend = (n > 1) ? P.sequence[2 * n - 1] : 0;
  }
  double x_in = rx, z_in = rz, x_out = 0, z_out = 0;
  for (int n = ns; n >= 1; --n) {
    if (n == ns) {
      const TField& tf = s.tf[ray.sec[n].tf];
      const Region& r = m.reg[tf.reg];
      ray.receiver_time = interpolate_arrivaltime2d(m, r, tf.T.data(), rx, rz);
      interpolate_time_gradient2d(m, r, tf.gx.data(), tf.gz.data(), rx, rz, ray.rgx, ray.rgz);
      if (ray.receiver_time > 1.0e10) { ray.valid = false; return; }
      if (ray.rgx == 0.0 && ray.rgz == 0.0) { ray.valid = false; return; }
    }
    trace_ray_section2d(m, s, ray, n, x_in, z_in, x_out, z_out);
    if (!ray.valid) break;
    if (n > 1) { x_in = x_out; z_in = z_out; }
  }
}

// inversion2d.f90:6344-6438 — best seafloor entry point of an in-water pick.
void find_optimal_entry(Model& m, Source& s, int itf, double rx, double rz, double& ex,
                        double& ez, double& wt) {
  const TField& tf = s.tf[itf];
  const Region& r = m.reg[tf.reg];
  const Isec& sf = m.isec[2];
  const int nsf = sf.nnode;
  const double dxs = sf.x[2] - sf.x[1];
  auto sf_z = [&](double px) {
    if (nsf < 2) return sf.z[1];
    const int ixx = (int)std::floor((px - sf.x[1]) / dxs) + 1;
    if (ixx < 1) return sf.z[1];
    if (ixx >= nsf) return sf.z[nsf];
    double w = std::min(1.0, std::max(0.0, (px - sf.x[ixx]) / dxs));
    return (1.0 - w) * sf.z[ixx] + w * sf.z[ixx + 1];
  };
  double tbest = kHugeTime;
  const double z0 = sf_z(rx);
  double xb = rx, zb = z0, wb = (z0 - rz) / m.vwater;
  for (int i = 1; i <= nsf; ++i) {
    const double xt = sf.x[i], zs = sf.z[i];
    const double tf_ = interpolate_arrivaltime2d(m, r, tf.T.data(), xt, zs);
    if (tf_ > kHugeTime * 0.5) continue;
    const double tw = std::sqrt((xt - rx) * (xt - rx) + (zs - rz) * (zs - rz)) / m.vwater;
    if (tf_ + tw < tbest) { tbest = tf_ + tw; xb = xt; zb = zs; wb = tw; }
  }
  if (xb <= sf.x[1] || xb >= sf.x[nsf]) { ex = xb; ez = zb; wt = wb; return; }
  double xl = 0, xr = 0;
  for (int i = 1; i <= nsf - 1; ++i)
    if (xb >= sf.x[i] && xb <= sf.x[i + 1]) { xl = sf.x[i]; xr = sf.x[i + 1]; break; }
  const int nref = 10;
  const double dr = (xr - xl) / double(nref);
  for (int k = 1; k <= nref - 1; ++k) {
    const double xt = xl + double(k) * dr;
    const double zs = sf_z(xt);
    const double tf_ = interpolate_arrivaltime2d(m, r, tf.T.data(), xt, zs);
    if (tf_ > kHugeTime * 0.5) continue;
    const double tw = std::sqrt((xt - rx) * (xt - rx) + (zs - rz) * (zs - rz)) / m.vwater;
    if (tf_ + tw < tbest) { tbest = tf_ + tw; xb = xt; zb = zs; wb = tw; }
  }
  ex = xb; ez = zb; wt = wb;
}

// inversion2d.f90:4548-4787 — slowness row by midpoint bilinear splat of each
// segment length, plus the interface-depth entries of a reflection.
void compute_frechet_for_ray2d(Model& m, Source& s, Ray& ray) {
  const Grid& g = m.grid;
  const int np = m.n_inv_parms;
  std::vector<double> cd(np + 2, 0.0);
  for (int k = 1; k <= ray.nsections; ++k) {
    const RaySection& rs = ray.sec[k];
    const int npts = (int)rs.px.size();
    if (npts <= 1) continue;
    if (rs.reg == 1) continue;
    for (int p = 0; p < npts - 1; ++p) {
      const double px = 0.5 * (rs.px[p] + rs.px[p + 1]);
      const double pz = 0.5 * (rs.pz[p] + rs.pz[p + 1]);
      const double ddx = rs.px[p + 1] - rs.px[p], ddz = rs.pz[p + 1] - rs.pz[p];
      const double sl = std::sqrt(ddx * ddx + ddz * ddz);
      if (sl < 1.0e-10) continue;
      const double vdx = m.vgx[2] - m.vgx[1];
      int ivx = (int)std::floor((px - m.vgx[1]) / vdx) + 1;
      ivx = std::max(1, std::min(g.nx - 1, ivx));
      int ivz;
      double wz;
      if (pz < g.z[1]) continue;
      if (pz >= g.z[g.nz]) { ivz = g.nz - 1; wz = 1.0; }
      else {
        ivz = (int)std::floor((pz - g.z[1]) / g.dz) + 1;
        ivz = std::max(1, std::min(g.nz - 1, ivz));
        wz = (pz - g.z[ivz]) / g.dz;
      }
      double wx = std::min(1.0, std::max(0.0, (px - m.vgx[ivx]) / vdx));
      wz = std::min(1.0, std::max(0.0, wz));
      auto add = [&](int a, int b, double w) {
        const int idx = m.inv_idx[g.g(a, b)];
        if (idx > 0) cd[idx] += w * sl;
      };
      add(ivx, ivz, (1.0 - wx) * (1.0 - wz));
      add(ivx + 1, ivz, wx * (1.0 - wz));
      add(ivx, ivz + 1, (1.0 - wx) * wz);
      add(ivx + 1, ivz + 1, wx * wz);
    }
  }
  if (m.iface_inv > 0) {
    bool done_rec = false, do_if = false;
    int prev = 0;
    for (int k = ray.nsections; k >= 1; --k) {
      const RaySection& rs = ray.sec[k];
      if ((int)rs.px.size() <= 2) continue;
      if (!done_rec) { prev = k; done_rec = true; }
      else do_if = true;
      if (do_if) {
        if (rs.istart == 0) { prev = k; continue; }
        if (rs.istart == m.iface_inv) {
          const Isec& is = m.isec[rs.istart];
          const double px = rs.px[0], pz = rs.pz[0];
          const TField& tf = s.tf[rs.tf];
          double gx, gz;
          interpolate_time_gradient2d(m, m.reg[rs.reg], tf.gx.data(), tf.gz.data(), px, pz, gx, gz);
          const double vin = get_velocity_at2d(m, px, pz);
          const double nl = std::sqrt(gx * gx + gz * gz);
          if (nl > 0.0) { gx = gx / (vin * nl); gz = gz / (vin * nl); }
          double nx, nz, h;
          interface_normal2d(m, px, is, nx, nz, h);
          const double gin = gx * nx + gz * nz;
          double gout;
          if (rs.reg == ray.sec[prev].reg) {
            gout = -gin;
          } else {
            const double tx = gx - gin * nx, tz = gz - gin * nz;
            const double par = std::sqrt(tx * tx + tz * tz);
            const double vout = get_velocity_at2d(m, px, pz);
            double det = 1.0 / (vout * vout) - par * par;
            if (det < 0.0) det = 0.0;
            gout = std::copysign(std::sqrt(det), gin);
          }
          const double geo = (gin - gout) * nz;
          const double dxi = is.x[2] - is.x[1];
          int ivx = (int)std::floor((px - is.x[1]) / dxi) + 1;
          ivx = std::max(1, std::min(is.nnode - 1, ivx));
          const double wx = std::min(1.0, std::max(0.0, (px - is.x[ivx]) / dxi));
          int idx = m.iface_start + ivx - 1;
          if (idx >= 1 && idx <= np) cd[idx + 1] += (1.0 - wx) * geo;
          idx = m.iface_start + ivx;
          if (idx >= 1 && idx <= np) cd[idx + 1] += wx * geo;
        }
      }
      prev = k;
    }
  }
  ray.pdev_indx.clear();
  ray.pdev.clear();
  for (int n = 1; n <= np; ++n)
    if (std::fabs(cd[n]) > 1.0e-30) { ray.pdev_indx.push_back(n); ray.pdev.push_back(cd[n]); }
}

}  // namespace orc
