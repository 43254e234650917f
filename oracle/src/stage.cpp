// Oracle stage coupling and the per-source phase recipe.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle.hpp"
#include <algorithm>

namespace orc {

// propagate2d.f90:2307-2411
void initialize_region_from_source2d(Model& m, Region& r, double sx, double sz, double t0) {
  const Grid& g = m.grid;
  std::fill(r.status.begin(), r.status.end(), -1);
  std::fill(r.T.begin(), r.T.end(), kHugeTime);
  std::fill(r.gx.begin(), r.gx.end(), 0.0);
  std::fill(r.gz.begin(), r.gz.end(), 0.0);
  int ix0 = (int)std::floor((sx - g.x0) / g.dx) + 1;
  int iz0 = (int)std::floor((sz - g.z0) / g.dz) + 1;
  if (ix0 < 1) ix0 = 1;
  if (ix0 >= g.nx) ix0 = g.nx - 1;
  if (iz0 < 1) iz0 = 1;
  if (iz0 >= g.nz) iz0 = g.nz - 1;
  for (int ix = ix0; ix <= ix0 + 1; ++ix) {
    for (int iz = iz0; iz <= iz0 + 1; ++iz) {
      if (ix < 1 || ix > g.nx || iz < 1 || iz > g.nz) continue;
      const int mm = r.rid[g.g(ix, iz)];
      if (mm <= 0 || mm > r.nnode) continue;
      const double ddx = g.x[ix] - sx, ddz = g.z[iz] - sz;
      const double dist = std::sqrt(ddx * ddx + ddz * ddz);
      double v = r.vel[mm];
      if (v < 0.01) v = 0.01;
      if (dist < 0.01 * g.tolerance) {
        r.T[mm] = t0;
        r.status[mm] = 0;
        r.gx[mm] = 0.0;
        r.gz[mm] = 0.0;
      } else {
        r.T[mm] = t0 + dist / v;
        r.status[mm] = 1;
        r.gx[mm] = ddx / (dist * v);
        r.gz[mm] = ddz / (dist * v);
      }
    }
  }
  for (int n = 1; n <= r.nnode; ++n) {
    if (r.status[n] != 0) continue;
    const int i1 = r.i1[n], i2 = r.i2[n];
    if (i1 == 0) continue;
    for (int dx = -1; dx <= 1; dx += 2)
      for (int dz = -1; dz <= 1; dz += 2) {
        const int a = i1 + dx, b = i2 + dz;
        if (a < 1 || a > g.nx || b < 1 || b > g.nz) continue;
        const int mm = r.rid[g.g(a, b)];
        if (mm > 0 && mm <= r.nnode && r.status[mm] == -1) r.status[mm] = 1;
      }
  }
}

// propagate2d.f90:2414-2554
void transfer_times_to_intersection(Model& m, Isec& is, const TField& tf) {
  const Grid& g = m.grid;
  is.T.assign(is.nnode + 1, kHugeTime);
  is.gx.assign(is.nnode + 1, 0.0);
  is.gz.assign(is.nnode + 1, 0.0);
  is.has_T = true;
  if (tf.reg == 0) return;
  const Region& r = m.reg[tf.reg];
  const std::vector<int>* ids = nullptr;
  if (is.id == r.ibot) ids = &r.ibot_rid;
  else if (is.id == r.itop) ids = &r.itop_rid;
  if (ids) {
    for (int n = 1; n <= is.nnode; ++n) {
      const int mm = (*ids)[n];
      if (mm > 0 && mm <= r.nnode) {
        is.T[n] = tf.T[mm];
        is.gx[n] = tf.gx[mm];
        is.gz[n] = tf.gz[mm];
      }
    }
    return;
  }
  // sample_region_time: bilinear on the loaded field, nearest node otherwise
  for (int n = 1; n <= is.nnode; ++n) {
    const double px = is.x[n], pz = is.z[n];
    int ix = (int)std::floor((px - g.x0) / g.dx) + 1;
    int iz = (int)std::floor((pz - g.z0) / g.dz) + 1;
    ix = std::max(1, std::min(g.nx - 1, ix));
    iz = std::max(1, std::min(g.nz - 1, iz));
    double w1 = std::min(1.0, std::max(0.0, (px - g.x[ix]) / g.dx));
    double w2 = std::min(1.0, std::max(0.0, (pz - g.z[iz]) / g.dz));
    const int n1 = r.rid[g.g(ix, iz)], n2 = r.rid[g.g(ix + 1, iz)];
    const int n3 = r.rid[g.g(ix, iz + 1)], n4 = r.rid[g.g(ix + 1, iz + 1)];
    if (n1 > 0 && n2 > 0 && n3 > 0 && n4 > 0) {
      auto bl = [&](const std::vector<double>& a) {
        return (1.0 - w1) * (1.0 - w2) * a[n1] + w1 * (1.0 - w2) * a[n2] +
               (1.0 - w1) * w2 * a[n3] + w1 * w2 * a[n4];
      };
      is.T[n] = bl(tf.T);
      is.gx[n] = bl(tf.gx);
      is.gz[n] = bl(tf.gz);
    } else {
      int nn = 0;
      double dmin = 1.0e100;
      for (int i = 1; i <= r.nnode; ++i) {
        const double d = (px - r.x[i]) * (px - r.x[i]) + (pz - r.z[i]) * (pz - r.z[i]);
        if (d < dmin) { dmin = d; nn = i; }
      }
      if (nn > 0) { is.T[n] = tf.T[nn]; is.gx[n] = tf.gx[nn]; is.gz[n] = tf.gz[nn]; }
    }
  }
}

// propagate2d.f90:2632-2741 — keep the tangential slowness, rebuild the
// normal component on the target side with the target-side velocity.
void reflect_gradient_at_interface(Model& m, Isec& is, const Region& target) {
  for (int n = 1; n <= is.nnode; ++n) {
    const double nx = is.nx_[n], nz = is.nz_[n];
    if (is.T[n] >= kHugeTime * 0.5) { is.gx[n] = 0.0; is.gz[n] = 0.0; continue; }
    const double gp = is.gx[n] * nx + is.gz[n] * nz;
    const double px = is.gx[n] - gp * nx, pz = is.gz[n] - gp * nz;
    int side;
    if (target.itop == is.id) side = 1;
    else if (target.ibot == is.id) side = -1;
    else side = gp < 0.0 ? -1 : 1;
    double v = side > 0 ? is.vel_bot[n] : is.vel_top[n];
    if (!(v > 0.01)) {
      int mm = 0;
      if (target.itop == is.id) mm = target.itop_rid[n];
      if (mm == 0 && target.ibot == is.id) mm = target.ibot_rid[n];
      if (mm > 0 && mm <= target.nnode) v = target.vel[mm];
    }
    if (v <= 0.01) { is.T[n] = kHugeTime; is.gx[n] = 0.0; is.gz[n] = 0.0; continue; }
    const double pt = 1.0 / v;
    const double pn2 = pt * pt - (px * px + pz * pz);
    if (pn2 < -1.0e-10) {
      is.T[n] = kHugeTime; is.gx[n] = 0.0; is.gz[n] = 0.0;
    } else {
      const double pn = std::sqrt(pn2 < 0.0 ? 0.0 : pn2);
      is.gx[n] = px + side * pn * nx;
      is.gz[n] = pz + side * pn * nz;
    }
  }
}

// propagate2d.f90:1982-2304 (mapped-interface branch; every stage of the
// phase recipe starts from the top or bottom interface of its own region).
void sweep_region_from_interface2d(Model& m, Region& r, const Isec& is) {
  const Grid& g = m.grid;
  std::fill(r.status.begin(), r.status.end(), -1);
  std::fill(r.T.begin(), r.T.end(), kHugeTime);
  std::fill(r.gx.begin(), r.gx.end(), 0.0);
  std::fill(r.gz.begin(), r.gz.end(), 0.0);
  const std::vector<int>* ids = nullptr;
  if (is.id == r.itop) ids = &r.itop_rid;
  else if (is.id == r.ibot) ids = &r.ibot_rid;
  if (!ids) return;  // unmapped branch is never reached by the recipe
  for (int n = 1; n <= is.nnode; ++n) {
    const int mm = (*ids)[n];
    if (mm > 0 && mm <= r.nnode) {
      r.status[mm] = 1;
      r.T[mm] = is.has_T ? is.T[n] : 0.0;
      r.gx[mm] = is.has_T ? is.gx[n] : 0.0;
      r.gz[mm] = is.has_T ? is.gz[n] : 0.0;
    }
  }
  const bool is_bottom = (is.id == r.ibot);
  for (int n = 1; n <= is.nnode; ++n) {
    const int mm = (*ids)[n];
    if (mm <= 0 || mm > r.nnode) continue;
    if (r.status[mm] != 1) continue;
    if (r.i1[mm] != 0) continue;
    int ix = (int)std::lround((r.x[mm] - g.x0) / g.dx) + 1;
    ix = std::max(1, std::min(g.nx, ix));
    int izf = 0;
    for (int iz = 1; iz <= g.nz - 1; ++iz)
      if (g.z[iz] <= r.z[mm] && r.z[mm] < g.z[iz + 1]) { izf = iz; break; }
    if (izf == 0) {
      if (r.z[mm] <= g.z[1]) izf = 1;
      if (r.z[mm] >= g.z[g.nz]) izf = g.nz - 1;
    }
    if (izf == 0) continue;
    int iz0, iz1, st;
    if (is_bottom) { iz0 = izf; iz1 = std::max(1, izf - 2); st = -1; }
    else { iz0 = izf + 1; iz1 = std::min(g.nz, izf + 3); st = 1; }
    for (int iz = iz0; st > 0 ? iz <= iz1 : iz >= iz1; iz += st) {
      for (int ixx = std::max(1, ix - 1); ixx <= std::min(g.nx, ix + 1); ++ixx) {
        const int nt = r.rid[g.g(ixx, iz)];
        if (nt <= 0 || nt > r.nnode) continue;
        if (r.status[nt] != -1) continue;
        r.status[nt] = 1;
        const double ddx = r.x[nt] - r.x[mm], ddz = r.z[nt] - r.z[mm];
        const double dist = std::sqrt(ddx * ddx + ddz * ddz);
        double v = r.vel[nt];
        if (v < 0.01) v = 0.01;
        r.T[nt] = r.T[mm] + dist / v;
        r.gx[nt] = ddx / (dist * v);
        r.gz[nt] = ddz / (dist * v);
      }
    }
  }
}

// inversion2d.f90:4264-4292 — top-row gradient fix of the water-layer fields.
static void water_top_fix(Model& m, Region& r, bool upward) {
  const Grid& g = m.grid;
  for (int ix = 1; ix <= g.nx; ++ix) {
    const int mt = r.rid[g.g(ix, 1)], mb = r.rid[g.g(ix, 2)];
    if (mt > 0 && mb > 0) {
      const double gz = r.gz[mt];
      const bool bad = upward ? (gz > 0.0 || std::fabs(gz) < 0.01)
                              : (gz < 0.0 || std::fabs(gz) < 0.01);
      if (bad) { r.gx[mt] = r.gx[mb]; r.gz[mt] = r.gz[mb]; }
    }
  }
}

// inversion2d.f90:4294-4409 — min-plus head-wave sweep along the Moho after
// the up-going PmP stage.  The node mapping is the intersection's
// rright/rleft table as the reference leaves it after all regions are
// defined (rright of the Moho intersection is numbered in region 4 while the
// sweep indexes region 6); it is reproduced unchanged.
static void pmp_headwave(Model& m, Region& r, Isec& is) {
  const Grid& g = m.grid;
  const int nn = is.nnode;
  if (nn <= 0) return;
  std::vector<double> th(nn + 1), vh(nn + 1);
  auto map_node = [&](int n) {
    int mm = 0;
    if (is.has_rright) mm = is.rright[n];
    if (mm == 0 && is.has_rleft) mm = is.rleft[n];
    return mm;
  };
  for (int n = 1; n <= nn; ++n) {
    const int mm = map_node(n);
    th[n] = (mm > 0 && mm <= r.nnode) ? r.T[mm] : kHugeTime;
    vh[n] = 0.0;
    if (mm > 0 && mm <= r.nnode) {
      if (r.i1[mm] == 0) {
        const int i3 = r.i3[mm];
        for (int k = 1; k <= 4; ++k) {
          const int c = is.ccfi(k, i3);
          if (c <= 0) continue;
          for (int ii = 0; ii <= 1; ++ii)
            for (int jj = 0; jj <= 1; ++jj) {
              const int ixx = is.cc_ix[c] + ii, izz = is.cc_iz[c] + jj;
              if (ixx < 1 || ixx > g.nx || izz < 1 || izz > g.nz) continue;
              if (g.node_region[g.g(ixx, izz)] != r.id) continue;
              const int q = g.rnode_id[g.g(ixx, izz)];
              if (q > 0 && q <= r.nnode && r.i1[q] > 0 && r.z[q] > is.z[n] + 0.5 * g.dz)
                vh[n] = std::max(vh[n], r.vel[q]);
            }
        }
      } else {
        vh[n] = r.vel[mm];
      }
    }
  }
  const double dxi = is.x[2] - is.x[1];
  for (int n = 2; n <= nn; ++n)
    if (vh[n] > 0.0) th[n] = std::min(th[n], th[n - 1] + dxi / vh[n]);
  for (int n = nn - 1; n >= 1; --n)
    if (vh[n] > 0.0) th[n] = std::min(th[n], th[n + 1] + dxi / vh[n]);
  for (int n = 1; n <= nn; ++n) {
    const int mm = map_node(n);
    if (mm > 0 && mm <= r.nnode && th[n] < r.T[mm] - 1.0e-10) r.T[mm] = th[n];
  }
  for (int n = 1; n <= nn; ++n) {
    const int mm = map_node(n);
    if (!(mm > 0 && mm <= r.nnode) || r.status[mm] != 0) continue;
    if (r.i1[mm] > 0) {
      fit_gradient_at_node2d(m, r, mm, r.gx[mm], r.gz[mm]);
    } else {
      double dtdx;
      if (n > 1 && n < nn) dtdx = (th[n + 1] - th[n - 1]) / (2.0 * dxi);
      else if (n == 1 && nn > 1) dtdx = (th[2] - th[1]) / dxi;
      else if (n == nn && nn > 1) dtdx = (th[nn] - th[nn - 1]) / dxi;
      else dtdx = 0.0;
      double dtdz = 0.0;
      if (vh[n] > 0.0) {
        const double s2 = 1.0 / (vh[n] * vh[n]) - dtdx * dtdx;
        dtdz = s2 > 0.0 ? std::sqrt(s2) : 0.0;
      }
      r.gx[mm] = dtdx;
      r.gz[mm] = dtdz;
    }
  }
}

// inversion2d.f90:4214-4476 — every phase's stage chain for one source.
void run_forward_source(Model& m, Source& s, int phase_mask) {
  static const int tf_reg[13] = {0, 5, 2, 2, 6, 6, 1, 1, 1, 1, 1, 5, 1};
  static const int tf_istart[13] = {0, 2, 2, 3, 2, 4, 2, 1, 2, 2, 1, 2, 2};
  for (int k = 1; k <= 12; ++k) {
    TField& t = s.tf[k];
    t.reg = tf_reg[k];
    t.istart = tf_istart[k];
    const int nn = m.reg[t.reg].nnode;
    t.T.assign(nn + 1, kHugeTime);
    t.gx.assign(nn + 1, 0.0);
    t.gz.assign(nn + 1, 0.0);
    t.solved = false;
  }
  for (int ip = 1; ip <= 5; ++ip) {
    if (!(phase_mask & (1 << (ip - 1)))) continue;
    const Path& P = m.path[ip];
    for (int k = 1; k <= P.n_tf; ++k) {
      const int itf = P.tf_sequence[k];
      TField& tf = s.tf[itf];
      Region& r = m.reg[tf.reg];
      if (k == 1) {
        initialize_region_from_source2d(m, r, s.x, s.z, 0.0);
      } else {
        const TField& prev = s.tf[P.tf_sequence[k - 1]];
        Isec& is = m.isec[tf.istart];
        transfer_times_to_intersection(m, is, prev);
        const bool refl = (ip == 2 && k == 2) || (ip == 3 && k == 2) || (ip == 4 && k >= 2) ||
                          (ip == 5 && k >= 2);
        if (refl) reflect_gradient_at_interface(m, is, r);
        sweep_region_from_interface2d(m, r, is);
      }
      propagate2d(m, r);
      if (r.id == 1) {
        if ((ip == 4 && (k == 2 || k == 4)) || (ip == 5 && (k == 1 || k == 4)))
          water_top_fix(m, r, true);
        else if ((ip == 4 && k == 3) || (ip == 5 && k == 2))
          water_top_fix(m, r, false);
      }
      if (ip == 3 && k == 2) pmp_headwave(m, r, m.isec[tf.istart]);
      tf.T = r.T;
      tf.gx = r.gx;
      tf.gz = r.gz;
      tf.solved = true;
      if (ip == 3 && k == 2) transfer_times_to_intersection(m, m.isec[tf.istart], tf);
    }
  }
}

}  // namespace orc
