// Oracle model build: smesh resampling, intersections (cut cells), regions,
// fully-regular tagging, velocity sampling, inversion numbering and phases.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle.hpp"
#include <algorithm>
#include <stdexcept>

namespace orc {

// invert2d_main.f90:279-340 — resample the smesh (depth relative to the
// seafloor) onto the uniform propagation grid with dz = dx.
void resample_smesh(int nx, int nzs, const double* xpos, const double* topo,
                    const double* zrel, const double* vel, double vwater,
                    int* nz_out, std::vector<double>& vel_out, double* zmax_out) {
  const double dz = xpos[1] - xpos[0];
  double maxtopo = topo[0];
  for (int i = 1; i < nx; ++i) maxtopo = std::max(maxtopo, topo[i]);
  const double zmax = zrel[nzs - 1] + maxtopo + 5.0;
  const int nz = (int)std::lround((zmax - 0.0) / dz) + 1;
  *nz_out = nz;
  *zmax_out = zmax;
  vel_out.assign((size_t)nx * nz, 0.0);
  for (int ix = 1; ix <= nx; ++ix) {
    int iv = ix;
    if (iv < 1) iv = 1;
    if (iv >= nx) iv = nx - 1;
    double wx = double(ix - iv);
    wx = std::min(1.0, std::max(0.0, wx));
    const double zsf = (1.0 - wx) * topo[iv - 1] + wx * topo[iv];
    for (int iz = 1; iz <= nz; ++iz) {
      const double zval = (iz - 1) * dz;
      const double pz = zval - zsf;
      double v;
      if (pz < 0.0) {
        v = vwater;
      } else if (pz >= zrel[nzs - 1]) {
        v = vel[(ix - 1) + (size_t)(nzs - 1) * nx];
      } else {
        int io = 1;
        for (io = 1; io <= nzs - 1; ++io)
          if (pz >= zrel[io - 1] && pz < zrel[io]) break;
        if (io >= nzs) io = nzs - 1;
        const double wz = (pz - zrel[io - 1]) / (zrel[io] - zrel[io - 1]);
        v = (1.0 - wz) * vel[(ix - 1) + (size_t)(io - 1) * nx] +
            wz * vel[(ix - 1) + (size_t)io * nx];
      }
      vel_out[(ix - 1) + (size_t)(iz - 1) * nx] = v;
    }
  }
}

// propagate2d.f90:1335-1502 — normals, one cut cell per interface node (the
// interface index doubles as the grid column), inode lists, ccind_from_2dc.
static void find_intersection2d(Model& m, Isec& is, const double* xs, const double* zs,
                                int nn) {
  Grid& g = m.grid;
  is.nnode = nn;
  is.x.assign(nn + 1, 0.0);
  is.z.assign(nn + 1, 0.0);
  is.nx_.assign(nn + 1, 0.0);
  is.nz_.assign(nn + 1, 0.0);
  for (int i = 1; i <= nn; ++i) { is.x[i] = xs[i - 1]; is.z[i] = zs[i - 1]; }
  for (int ix = 1; ix <= nn; ++ix) {
    double dzdx;
    if (ix > 1 && ix < nn) dzdx = (is.z[ix + 1] - is.z[ix - 1]) / (is.x[ix + 1] - is.x[ix - 1]);
    else if (ix == 1 && nn >= 2) dzdx = (is.z[ix + 1] - is.z[ix]) / (is.x[ix + 1] - is.x[ix]);
    else if (ix == nn && nn >= 2) dzdx = (is.z[ix] - is.z[ix - 1]) / (is.x[ix] - is.x[ix - 1]);
    else dzdx = 0.0;
    const double len = std::sqrt(1.0 + dzdx * dzdx);
    is.nx_[ix] = -dzdx / len;
    is.nz_[ix] = 1.0 / len;
  }
  std::vector<int> tix, tiz;
  for (int ix = 1; ix <= nn; ++ix) {
    const double zv = is.z[ix];
    int izc = 0;
    for (int iz = 1; iz <= g.nz - 1; ++iz)
      if (g.z[iz] <= zv && zv < g.z[iz + 1]) { izc = iz; break; }
    if (izc == 0) {
      if (zv <= g.z[1]) izc = 1;
      if (zv >= g.z[g.nz]) izc = g.nz - 1;
    }
    if (izc > 0) { tix.push_back(ix); tiz.push_back(izc); }
  }
  const int ncc = (int)tix.size();
  is.n_ccells = ncc;
  is.cc_ix.assign(std::max(ncc, 1) + 1, 0);
  is.cc_iz.assign(std::max(ncc, 1) + 1, 0);
  is.n_inodes.assign(std::max(ncc, 1) + 1, 0);
  is.inodes.assign((size_t)std::max(ncc, 1) * 4, 0);
  for (int c = 1; c <= ncc; ++c) { is.cc_ix[c] = tix[c - 1]; is.cc_iz[c] = tiz[c - 1]; }
  // cut cells are created in ascending ix, one per ix: the cell of node ix
  // is the only one with cc_ix == ix.
  for (int ix = 1; ix <= nn; ++ix) {
    const double zv = is.z[ix];
    for (int c = 1; c <= ncc; ++c) {
      if (is.cc_ix[c] != ix) continue;
      const int izc = is.cc_iz[c];
      if (g.z[izc] <= zv && zv <= g.z[izc + 1]) {
        is.n_inodes[c] += 1;
        if (is.n_inodes[c] > 4) throw std::runtime_error("find_intersection2d: too many inodes");
        is.inodes[(c - 1) * 4 + is.n_inodes[c] - 1] = ix;
      }
    }
  }
  is.ccell_from_inode.assign((size_t)nn * 4, 0);
  for (int ix = 1; ix <= nn; ++ix) {
    int cnt = 0;
    for (int c = 1; c <= ncc; ++c) {
      if (is.cc_ix[c] == ix) {
        ++cnt;
        if (cnt <= 4) is.ccell_from_inode[(ix - 1) * 4 + cnt - 1] = c;
      }
    }
  }
  for (int c = 1; c <= ncc; ++c) {
    const int ix = is.cc_ix[c], iz = is.cc_iz[c];
    if (ix >= 1 && ix < g.nx && iz >= 1 && iz < g.nz) {
      const int gi = g.g(ix, iz);
      if (!g.cc_assoc[gi]) {
        g.cc_assoc[gi] = 1;
        for (int k = 0; k < 6; ++k) g.cc_idx[(size_t)gi * 6 + k] = 0;
      }
      g.cc_idx[(size_t)gi * 6 + is.id] = c;
    }
  }
}

// propagate2d.f90:1623-1645 (internal interpolate_iface_z2d)
static double iface_z_at(const Model& m, const Isec& is, double px) {
  if (is.nnode < 2) return is.z[1];
  const int ixx = (int)std::floor((px - is.x[1]) / m.grid.dx) + 1;
  if (ixx < 1) return is.z[1];
  if (ixx >= is.nnode) return is.z[is.nnode];
  double w = (px - is.x[ixx]) / m.grid.dx;
  w = std::min(1.0, std::max(0.0, w));
  return (1.0 - w) * is.z[ixx] + w * is.z[ixx + 1];
}

// propagate2d.f90:1505-1621 — node numbering: grid nodes with
// z_top <= z <= z_bot, ix outer / iz inner, then top then bottom interface.
static void define_region2d(Model& m, Region& r, int itop, int ibot) {
  Grid& g = m.grid;
  Isec& it = m.isec[itop];
  Isec& ib = m.isec[ibot];
  r.itop = itop;
  r.ibot = ibot;
  int ng = 0;
  for (int ix = 1; ix <= g.nx; ++ix) {
    const double zt = iface_z_at(m, it, g.x[ix]);
    const double zb = iface_z_at(m, ib, g.x[ix]);
    for (int iz = 1; iz <= g.nz; ++iz)
      if (zt <= g.z[iz] && g.z[iz] <= zb) ++ng;
  }
  r.ngnode = ng;
  r.nnode = ng + it.nnode + ib.nnode;
  const int nn = r.nnode;
  r.i1.assign(nn + 1, 0); r.i2.assign(nn + 1, 0); r.i3.assign(nn + 1, 0);
  r.x.assign(nn + 1, 0.0); r.z.assign(nn + 1, 0.0); r.vel.assign(nn + 1, 0.0);
  r.status.assign(nn + 1, -1);
  r.T.assign(nn + 1, kHugeTime); r.gx.assign(nn + 1, 0.0); r.gz.assign(nn + 1, 0.0);
  r.rid.assign((size_t)g.nx * g.nz, 0);
  int n = 0;
  for (int ix = 1; ix <= g.nx; ++ix) {
    const double zt = iface_z_at(m, it, g.x[ix]);
    const double zb = iface_z_at(m, ib, g.x[ix]);
    for (int iz = 1; iz <= g.nz; ++iz) {
      const int gi = g.g(ix, iz);
      if (zt <= g.z[iz] && g.z[iz] <= zb) {
        ++n;
        r.i1[n] = ix; r.i2[n] = iz; r.i3[n] = 0;
        r.x[n] = g.x[ix]; r.z[n] = g.z[iz];
        g.rnode_id[gi] = n;
        g.node_region[gi] = r.id;
        r.rid[gi] = n;
      } else if (g.node_region[gi] == 0) {
        g.node_region[gi] = -1;
      }
    }
  }
  it.rright.assign(it.nnode + 1, 0); it.has_rright = true;
  r.itop_rid.assign(it.nnode + 1, 0);
  for (int k = 1; k <= it.nnode; ++k) {
    ++n;
    r.i1[n] = 0; r.i2[n] = itop; r.i3[n] = k;
    r.x[n] = it.x[k]; r.z[n] = it.z[k];
    it.rright[k] = n; r.itop_rid[k] = n;
  }
  ib.rleft.assign(ib.nnode + 1, 0); ib.has_rleft = true;
  r.ibot_rid.assign(ib.nnode + 1, 0);
  for (int k = 1; k <= ib.nnode; ++k) {
    ++n;
    r.i1[n] = 0; r.i2[n] = ibot; r.i3[n] = k;
    r.x[n] = ib.x[k]; r.z[n] = ib.z[k];
    ib.rleft[k] = n; r.ibot_rid[k] = n;
  }
}

// propagate2d.f90:1941-1979
static void tag_regular_nodes2d(Model& m) {
  Grid& g = m.grid;
  g.fully_regular.assign((size_t)g.nx * g.nz, 1);
  for (int ix = 1; ix <= g.nx; ++ix) {
    for (int iz = 1; iz <= g.nz; ++iz) {
      const int gi = g.g(ix, iz);
      if (g.node_region[gi] <= 0) { g.fully_regular[gi] = 0; continue; }
      bool reg = true;
      for (int i = 0; i <= 1; ++i)
        for (int j = 0; j <= 1; ++j)
          if (ix - i > 0 && ix - i < g.nx && iz - j > 0 && iz - j < g.nz)
            if (g.cc_assoc[g.g(ix - i, iz - j)]) reg = false;
      if (ix == 1 || ix == g.nx) reg = false;
      if (iz == 1 || iz == g.nz) reg = false;
      g.fully_regular[gi] = reg ? 1 : 0;
    }
  }
}

// propagate2d.f90:1695-1797 — bilinear velocity one grid step above / below
// every interface node.  The velocity grid is the resampled propagation grid.
static double vel_side(const Model& m, const std::vector<double>& vx, double px, double pzoff) {
  const Grid& g = m.grid;
  const int nxv = g.nx, nzv = g.nz;
  const double dxv = vx[2] - vx[1];
  int ivx = (int)std::floor((px - vx[1]) / dxv) + 1;
  if (ivx < 1) ivx = 1;
  if (ivx >= nxv) ivx = nxv - 1;
  double wx = (px - vx[ivx]) / dxv;
  wx = std::min(1.0, std::max(0.0, wx));
  int ivz;
  double wz;
  if (pzoff < g.z[1]) { ivz = 1; wz = 0.0; }
  else if (pzoff >= g.z[nzv]) { ivz = nzv - 1; wz = 1.0; }
  else {
    for (ivz = 1; ivz <= nzv - 1; ++ivz)
      if (pzoff >= g.z[ivz] && pzoff < g.z[ivz + 1]) break;
    if (ivz >= nzv) ivz = nzv - 1;
    const double lo = pzoff - g.z[ivz];
    const double up = g.z[ivz + 1] - g.z[ivz];
    wz = up > 0.0 ? lo / up : 0.0;
  }
  wz = std::min(1.0, std::max(0.0, wz));
  auto V = [&](int ix, int iz) { return g.vel[g.g(ix, iz)]; };
  return (1.0 - wx) * (1.0 - wz) * V(ivx, ivz) + wx * (1.0 - wz) * V(ivx + 1, ivz) +
         (1.0 - wx) * wz * V(ivx, ivz + 1) + wx * wz * V(ivx + 1, ivz + 1);
}

// propagate2d.f90:1800-1938
static void velocities_to_region2d(Model& m, Region& r) {
  const Grid& g = m.grid;
  for (int n = 1; n <= r.nnode; ++n) {
    if (r.i1[n] != 0) r.vel[n] = g.vel[g.g(r.i1[n], r.i2[n])];
    else if (r.i2[n] == r.itop) r.vel[n] = m.isec[r.itop].vel_bot[r.i3[n]];
    else if (r.i2[n] == r.ibot) r.vel[n] = m.isec[r.ibot].vel_top[r.i3[n]];
  }
  for (int n = 1; n <= r.nnode; ++n) {
    const int i1 = r.i1[n];
    if (i1 == 0) continue;
    const int i2 = r.i2[n];
    if (i2 < g.nz && r.rid[g.g(i1, i2 + 1)] <= 0) {
      const Isec& ib = m.isec[r.ibot];
      int i3 = (int)std::lround((r.x[n] - ib.x[1]) / g.dx) + 1;
      i3 = std::max(1, std::min(ib.nnode, i3));
      r.vel[n] = ib.vel_top[i3];
    }
    if (i2 > 1 && r.rid[g.g(i1, i2 - 1)] <= 0) {
      const Isec& it = m.isec[r.itop];
      int i3 = (int)std::lround((r.x[n] - it.x[1]) / g.dx) + 1;
      i3 = std::max(1, std::min(it.nnode, i3));
      r.vel[n] = it.vel_bot[i3];
    }
  }
}

void build_model(Model& m, int nx, int nz, double dx, const double* xpos,
                 const double* vel_pgrid, const double* iface_z, double vwater, int iface_inv) {
  Grid& g = m.grid;
  g.nx = nx; g.nz = nz; g.dx = dx; g.dz = dx; g.x0 = xpos[0]; g.z0 = 0.0;
  g.tolerance = std::min(g.dx, g.dz) * 0.01;
  g.x.assign(nx + 1, 0.0); g.z.assign(nz + 1, 0.0);
  for (int i = 1; i <= nx; ++i) g.x[i] = g.x0 + (i - 1) * g.dx;
  for (int i = 1; i <= nz; ++i) g.z[i] = g.z0 + (i - 1) * g.dz;
  g.vel.assign(vel_pgrid, vel_pgrid + (size_t)nx * nz);
  g.node_region.assign((size_t)nx * nz, 0);
  g.rnode_id.assign((size_t)nx * nz, 0);
  g.cc_assoc.assign((size_t)nx * nz, 0);
  g.cc_idx.assign((size_t)nx * nz * 6, 0);
  m.vwater = vwater;
  // interface nodes sit at the smesh x positions (invert2d_main.f90:155-199)
  std::vector<double> xs(xpos, xpos + nx);
  for (int k = 1; k <= 5; ++k) {
    m.isec[k] = Isec();
    m.isec[k].id = k;
    find_intersection2d(m, m.isec[k], xs.data(), iface_z + (size_t)(k - 1) * nx, nx);
  }
  // invert2d_main.f90:420-452 — regions 1..4 between consecutive interfaces,
  // 5 = seafloor..bottom, 6 = seafloor..Moho.  Later definitions overwrite
  // the intersections' rright/rleft tables exactly as the reference does.
  for (int k = 1; k <= 6; ++k) { m.reg[k] = Region(); m.reg[k].id = k; }
  for (int k = 1; k <= 4; ++k) define_region2d(m, m.reg[k], k, k + 1);
  m.isec[2].has_rright = false; m.isec[2].rright.clear();
  m.isec[5].has_rleft = false; m.isec[5].rleft.clear();
  define_region2d(m, m.reg[5], 2, 5);
  define_region2d(m, m.reg[6], 2, 4);
  tag_regular_nodes2d(m);
  // the velocity grid keeps the smesh x positions (invert2d_main.f90:371-373)
  std::vector<double> vgx(nx + 1, 0.0);
  for (int i = 1; i <= nx; ++i) vgx[i] = xpos[i - 1];
  m.vgx = vgx;
  for (int k = 1; k <= 5; ++k) {
    Isec& is = m.isec[k];
    is.vel_top.assign(is.nnode + 1, 0.0);
    is.vel_bot.assign(is.nnode + 1, 0.0);
    for (int n = 1; n <= is.nnode; ++n) {
      is.vel_top[n] = vel_side(m, vgx, is.x[n], is.z[n] - g.dz);
      is.vel_bot[n] = vel_side(m, vgx, is.x[n], is.z[n] + g.dz);
    }
  }
  for (int k = 1; k <= 6; ++k) velocities_to_region2d(m, m.reg[k]);
  // invert2d_main.f90:487-500 region pointers of the intersections
  m.isec[1].regleft = 0; m.isec[1].regright = 1;
  m.isec[2].regleft = 1; m.isec[2].regright = 5;
  m.isec[3].regleft = 2; m.isec[3].regright = 3;
  m.isec[4].regleft = 3; m.isec[4].regright = 4;
  m.isec[5].regleft = 5; m.isec[5].regright = 0;
  m.nsurf_x = nx;
  // frechet2d.f90:55-63 and invert2d_main.f90:456-477: active velocity nodes
  // are those at or below the seafloor; numbered iz outer, ix inner.
  m.active.assign((size_t)nx * nz, 0);
  m.inv_idx.assign((size_t)nx * nz, 0);
  const double* topo = iface_z + (size_t)1 * nx;
  for (int ix = 1; ix <= nx; ++ix) {
    int iv = ix;
    if (iv >= nx) iv = nx - 1;
    double wx = std::min(1.0, std::max(0.0, double(ix - iv)));
    const double zsf = (1.0 - wx) * topo[iv - 1] + wx * topo[iv];
    for (int iz = 1; iz <= nz; ++iz)
      m.active[g.g(ix, iz)] = (g.z[iz] - zsf >= 0.0) ? 1 : 0;
  }
  int np = 0;
  for (int iz = 1; iz <= nz; ++iz)
    for (int ix = 1; ix <= nx; ++ix)
      if (m.active[g.g(ix, iz)]) m.inv_idx[g.g(ix, iz)] = ++np;
  m.n_vel_parms = np;
  m.iface_inv = iface_inv;
  m.iface_start = np;
  m.n_inv_parms = np + (iface_inv > 0 ? m.isec[iface_inv].nnode : 0);
  // invert2d_main.f90:564-700 — the five phases
  auto setp = [&](int p, std::vector<int> seq, std::vector<int> tfs) {
    Path& P = m.path[p];
    P.n_tf = (int)tfs.size();
    P.sequence.assign(1, 0); P.sequence.insert(P.sequence.end(), seq.begin(), seq.end());
    P.tf_sequence.assign(1, 0); P.tf_sequence.insert(P.tf_sequence.end(), tfs.begin(), tfs.end());
  };
  setp(1, {0, 2}, {1});
  setp(2, {0, 3, 3, 0}, {2, 3});
  setp(3, {0, 4, 4, 0}, {4, 5});
  setp(4, {0, 2, 2, 1, 1, 2, 2, 2}, {1, 6, 7, 8});
  setp(5, {0, 1, 1, 2, 2, 2, 2, 2}, {9, 10, 11, 12});
}

}  // namespace orc
