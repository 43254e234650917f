// Host-side model build for the device solver (see model.h for the layout).
#include "model.h"
#include <algorithm>
#include <cmath>
#include <thread>

namespace fmt2d {

namespace {

// Depth of an interface at horizontal position px: linear between nodes,
// clamped to the end nodes (propagate2d.f90:1623-1645 and rays2d.f90:1222).
double iface_z_at(const Model& m, const std::vector<double>& xs, const std::vector<double>& zs,
                  double px) {
  const int n = (int)zs.size();
  if (n < 2) return zs[0];
  const int k = (int)std::floor((px - xs[0]) / m.dx);  // 0-based left node
  if (k < 0) return zs[0];
  if (k >= n - 1) return zs[n - 1];
  double w = (px - xs[k]) / m.dx;
  w = std::min(1.0, std::max(0.0, w));
  return (1.0 - w) * zs[k] + w * zs[k + 1];
}

double grid_x(const Model& m, int ix) { return m.x0 + ix * m.dx; }
double grid_z(const Model& m, int iz) { return iz * m.dx; }

// Bilinear velocity-grid sample one grid step above/below an interface node
// (propagate2d.f90:1695-1797).  The velocity grid is the resampled grid with
// the smesh x positions.
double vel_side(const Model& m, double px, double pzoff) {
  const int nx = m.nx, nz = m.nz;
  const double dxv = m.xpos[1] - m.xpos[0];
  int ivx = (int)std::floor((px - m.xpos[0]) / dxv);
  ivx = std::max(0, std::min(nx - 2, ivx));
  const double wx = std::min(1.0, std::max(0.0, (px - m.xpos[ivx]) / dxv));
  int ivz;
  double wz;
  if (pzoff < grid_z(m, 0)) { ivz = 0; wz = 0.0; }
  else if (pzoff >= grid_z(m, nz - 1)) { ivz = nz - 2; wz = 1.0; }
  else {
    for (ivz = 0; ivz < nz - 1; ++ivz)
      if (pzoff >= grid_z(m, ivz) && pzoff < grid_z(m, ivz + 1)) break;
    if (ivz >= nz - 1) ivz = nz - 2;
    const double up = grid_z(m, ivz + 1) - grid_z(m, ivz);
    wz = up > 0.0 ? (pzoff - grid_z(m, ivz)) / up : 0.0;
  }
  wz = std::min(1.0, std::max(0.0, wz));
  auto V = [&](int a, int b) { return m.vel[m.g(a, b)]; };
  return (1.0 - wx) * (1.0 - wz) * V(ivx, ivz) + wx * (1.0 - wz) * V(ivx + 1, ivz) +
         (1.0 - wx) * wz * V(ivx, ivz + 1) + wx * wz * V(ivx + 1, ivz + 1);
}

void build_interface(Model& m, int k, const double* zs) {
  Interface& f = m.ifc[k];
  const int n = m.nx;
  f.z.assign(zs, zs + n);
  f.nrm_x.assign(n, 0.0);
  f.nrm_z.assign(n, 0.0);
  const std::vector<double>& X = m.xpos;
  for (int i = 0; i < n; ++i) {
    double dzdx;
    if (i > 0 && i < n - 1) dzdx = (f.z[i + 1] - f.z[i - 1]) / (X[i + 1] - X[i - 1]);
    else if (i == 0 && n >= 2) dzdx = (f.z[1] - f.z[0]) / (X[1] - X[0]);
    else if (i == n - 1 && n >= 2) dzdx = (f.z[i] - f.z[i - 1]) / (X[i] - X[i - 1]);
    else dzdx = 0.0;
    const double len = std::sqrt(1.0 + dzdx * dzdx);
    f.nrm_x[i] = -dzdx / len;
    f.nrm_z[i] = 1.0 / len;
  }
  // cut cell of node i: the grid cell in column i whose rows bracket z
  f.izc.assign(n, -1);
  f.inode_ok.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    const double zv = f.z[i];
    int c = -1;
    for (int iz = 0; iz < m.nz - 1; ++iz)
      if (grid_z(m, iz) <= zv && zv < grid_z(m, iz + 1)) { c = iz; break; }
    if (c < 0) {
      if (zv <= grid_z(m, 0)) c = 0;
      if (zv >= grid_z(m, m.nz - 1)) c = m.nz - 2;
    }
    f.izc[i] = c;
    if (c >= 0) {
      f.inode_ok[i] = (grid_z(m, c) <= zv && zv <= grid_z(m, c + 1)) ? 1 : 0;
      // only cells inside the grid are registered for neighbour lookups
      if (i < m.nx - 1 && c < m.nz - 1) m.cell_cut[(size_t)c * m.nx + i] |= (uint8_t)(1u << k);
    }
  }
}

// A region's own tables (row range per column, node numbering, slots): they
// read only the interfaces, so the six regions are built concurrently.
void define_region(const Model& m, Region& r, int itop, int ibot) {
  r.itop = itop;
  r.ibot = ibot;
  const int nx = m.nx, nz = m.nz;
  r.r0.assign(nx, 0);
  r.r1.assign(nx, -1);
  r.col_base.assign(nx, 0);
  int ng = 0, zlo = nz, zhi = -1;
  for (int ix = 0; ix < nx; ++ix) {
    const double zt = iface_z_at(m, m.xpos, m.ifc[itop].z, grid_x(m, ix));
    const double zb = iface_z_at(m, m.xpos, m.ifc[ibot].z, grid_x(m, ix));
    // the rows with zt <= z <= zb form one range (z = iz*dx grows with iz):
    // start from the estimate and settle it with those same comparisons
    int a = (int)std::ceil(zt / m.dx);
    a = std::max(0, std::min(nz, a));
    while (a > 0 && zt <= grid_z(m, a - 1)) --a;
    while (a < nz && !(zt <= grid_z(m, a))) ++a;
    int b = (int)std::floor(zb / m.dx);
    b = std::max(-1, std::min(nz - 1, b));
    while (b < nz - 1 && grid_z(m, b + 1) <= zb) ++b;
    while (b >= 0 && !(grid_z(m, b) <= zb)) --b;
    r.col_base[ix] = ng;
    if (a <= b) {
      r.r0[ix] = a;
      r.r1[ix] = b;
      ng += b - a + 1;
      zlo = std::min(zlo, a);
      zhi = std::max(zhi, b);
    } else {
      r.r0[ix] = 0;
      r.r1[ix] = -1;
    }
  }
  r.ngnode = ng;
  r.nnode = ng + 2 * nx;
  if (zhi < 0) { zlo = 0; zhi = 0; }
  r.z_lo = zlo;
  r.z_hi = zhi;
  r.H = zhi - zlo + 1;
  r.tiles_x = (nx + kTileW - 1) / kTileW;
  r.tiles_y = (r.H + kTileH - 1) / kTileH;
  r.pitch = r.tiles_x * kTileW;
  r.slot_of_node.assign(r.nnode, 0);
  // node ids run down each column (the reference's order), slots row by row
  for (int iz = zlo; iz <= zhi; ++iz)
    for (int ix = 0; ix < nx; ++ix) {
      if (iz < r.r0[ix] || iz > r.r1[ix]) continue;
      r.slot_of_node[r.col_base[ix] + (iz - r.r0[ix])] = r.slot_grid(ix, iz);
    }
  for (int k = 0; k < nx; ++k) {
    r.slot_of_node[ng + k] = r.slot_top(k);
    r.slot_of_node[ng + nx + k] = r.slot_bot(k);
  }
}

// The model-wide tables a region definition leaves (the last region that
// claims a grid node owns it; the interface node id tables of its top and
// bottom interface), applied in the reference's region order.
void claim_region(Model& m, const Region& r) {
  const int nx = m.nx;
  for (int iz = r.z_lo; iz <= r.z_hi; ++iz)
    for (int ix = 0; ix < nx; ++ix) {
      if (iz < r.r0[ix] || iz > r.r1[ix]) continue;
      const size_t gi = m.g(ix, iz);
      m.node_region[gi] = r.id;
      m.rnode_id[gi] = r.col_base[ix] + (iz - r.r0[ix]) + 1;
    }
  m.rright[r.itop].assign(nx, 0);
  m.rleft[r.ibot].assign(nx, 0);
  for (int k = 0; k < nx; ++k) {
    m.rright[r.itop][k] = r.ngnode + k + 1;
    m.rleft[r.ibot][k] = r.ngnode + nx + k + 1;
  }
}

bool in_region(const Region& r, int ix, int iz) {
  return ix >= 0 && ix < (int)r.r0.size() && iz >= r.r0[ix] && iz <= r.r1[ix];
}

// Region velocity and per-slot codes (velocities_to_region2d semantics for
// the velocity, propagate2d.f90:1800-1938).
void finish_region(Model& m, Region& r) {
  const int nx = m.nx;
  const size_t ns = r.nslots();
  r.code.assign(ns, 0);
  r.vel.assign(ns, 0.0f);
  r.vel64.assign(ns, 0.0);
  r.iface_dz.assign((size_t)2 * r.pitch, 0.0f);
  r.izc_top.assign(r.pitch, -1);
  r.izc_bot.assign(r.pitch, -1);
  const Interface& ft = m.ifc[r.itop];
  const Interface& fb = m.ifc[r.ibot];
  const uint8_t tbit = (uint8_t)(1u << r.itop), bbit = (uint8_t)(1u << r.ibot);
  auto cut = [&](int cx, int cz) { return m.cell_cut[(size_t)cz * nx + cx]; };
  // rows outer, columns inner: every per-node array is row-major, and each
  // slot's code and velocity depend on nothing computed here
  for (int iz = r.z_lo; iz <= r.z_hi; ++iz) {
    for (int ix = 0; ix < nx; ++ix) {
      if (iz < r.r0[ix] || iz > r.r1[ix]) continue;
      const int s = r.slot_grid(ix, iz);
      double v = m.vel[m.g(ix, iz)];
      if (iz < m.nz - 1 && !in_region(r, ix, iz + 1)) {
        int k = (int)std::lround((grid_x(m, ix) - m.xpos[0]) / m.dx);
        k = std::max(0, std::min(nx - 1, k));
        v = fb.vel_top[k];
      }
      if (iz > 0 && !in_region(r, ix, iz - 1)) {
        int k = (int)std::lround((grid_x(m, ix) - m.xpos[0]) / m.dx);
        k = std::max(0, std::min(nx - 1, k));
        v = ft.vel_bot[k];
      }
      r.vel[s] = (float)v;
      r.vel64[s] = v;
      uint32_t code = kInRegion | kUpdatable;
      if (m.fully_regular[m.g(ix, iz)]) code |= kFullyRegular;
      for (int c = 0; c < 4; ++c) {
        const int cx = ix - (c >= 2 ? 1 : 0), cz = iz - ((c & 1) ? 1 : 0);
        if (cx < 0 || cx > nx - 2 || cz < 0 || cz > m.nz - 2) continue;
        code |= cell_exists_bit(c);
        const uint8_t cc = cut(cx, cz);
        if (cc) code |= cell_any_bit(c);
        if (cc & (tbit | bbit)) {
          code |= cell_irr_bit(c);
          if ((cc & tbit) && ft.inode_ok[cx]) code |= cell_top_bit(c);
          if ((cc & bbit) && fb.inode_ok[cx]) code |= cell_bot_bit(c);
        }
      }
      r.code[s] = code;
    }
  }
  for (int side = 0; side < 2; ++side) {
    const Interface& f = side == 0 ? ft : fb;
    const int fbit = side == 0 ? r.itop : r.ibot;
    for (int k = 0; k < nx; ++k) {
      const int s = side == 0 ? r.slot_top(k) : r.slot_bot(k);
      r.vel64[s] = side == 0 ? ft.vel_bot[k] : fb.vel_top[k];
      r.vel[s] = (float)r.vel64[s];
      uint32_t code = kInRegion | kIfaceNode;
      const int c = f.izc[k];
      (side == 0 ? r.izc_top : r.izc_bot)[k] = c;
      if (c >= 0) r.iface_dz[(size_t)side * r.pitch + k] = (float)(f.z[k] - grid_z(m, c));
      if (c >= 0 && k < nx - 1) code |= cell_any_bit(0);
      if (c >= 0 && k < nx - 1 && f.inode_ok[k]) {
        code |= kUpdatable | cell_irr_bit(0);
        const uint8_t cc = cut(k, c);
        if ((cc & tbit) && ft.inode_ok[k]) code |= cell_top_bit(0);
        if ((cc & bbit) && fb.inode_ok[k]) code |= cell_bot_bit(0);
      }
      (void)fbit;
      r.code[s] = code;
    }
  }
}

}  // namespace

std::string build_model(Model& m, int nx, int nzs, const double* xpos, const double* topo,
                        const double* zrel, const double* vel, double vwater,
                        const double* sed_z, const double* moho_z, int iface_inv) {
  if (nx < 3 || nzs < 2) return "model too small";
  const double dx = xpos[1] - xpos[0];
  if (!(dx > 0.0)) return "xpos must increase";
  m.nx = nx;
  m.dx = dx;
  m.x0 = xpos[0];
  m.tolerance = dx * 0.01;
  m.vwater = vwater;
  m.xpos.assign(xpos, xpos + nx);
  // resample the smesh onto dz = dx rows (invert2d_main.f90:279-340)
  const double maxtopo = *std::max_element(topo, topo + nx);
  const double zmax = zrel[nzs - 1] + maxtopo + 5.0;
  m.nz = (int)std::lround(zmax / dx) + 1;
  const int nz = m.nz;
  m.vel.assign((size_t)nx * nz, 0.0);
  // the seafloor depth of every column
  std::vector<double> zsf(nx);
  for (int ix = 0; ix < nx; ++ix) {
    const int iv = std::min(ix, nx - 2);
    const double wx = std::min(1.0, std::max(0.0, double(ix - iv)));
    zsf[ix] = (1.0 - wx) * topo[iv] + wx * topo[iv + 1];
  }
  // With zrel non-decreasing, the smesh row that brackets a node is unique
  // and never moves up a column (pz grows down it): each column's search
  // resumes at the row the node above found, with the same result as a
  // search from the top.  Otherwise every search starts at the top.
  bool monotone = true;
  for (int io = 0; io + 1 < nzs; ++io) monotone = monotone && zrel[io] <= zrel[io + 1];
  std::vector<int> from(nx, 0);
  // rows outer: m.vel is row-major
  for (int iz = 0; iz < nz; ++iz) {
    double* vrow = &m.vel[m.g(0, iz)];
    for (int ix = 0; ix < nx; ++ix) {
      const double pz = grid_z(m, iz) - zsf[ix];
      double v;
      if (pz < 0.0) v = vwater;
      else if (pz >= zrel[nzs - 1]) v = vel[(size_t)(nzs - 1) * nx + ix];
      else {
        int io = monotone ? from[ix] : 0;
        for (; io < nzs - 1; ++io)
          if (pz >= zrel[io] && pz < zrel[io + 1]) break;
        if (io >= nzs - 1) io = nzs - 2;   // no bracketing row
        else if (monotone) from[ix] = io;
        const double wz = (pz - zrel[io]) / (zrel[io + 1] - zrel[io]);
        v = (1.0 - wz) * vel[(size_t)io * nx + ix] + wz * vel[(size_t)(io + 1) * nx + ix];
      }
      vrow[ix] = v;
    }
  }
  m.zbot = zrel[nzs - 1] + maxtopo;
  m.iface_inv = iface_inv;
  build_geometry(m, topo, sed_z, moho_z);
  return std::string();
}

// Interfaces, regions, codes and the inversion numbering from the
// propagation-grid velocity m.vel and the seafloor, sediment-base and Moho
// depths (invert2d_main.f90:342-477; rebuild_geometry2d,
// inversion2d.f90:3661-3816, redoes the same after an interface update).
void build_geometry(Model& m, const double* topo, const double* sed_z, const double* moho_z) {
  const int nx = m.nx, nz = m.nz;
  const double dx = m.dx;
  m.cell_cut.assign((size_t)nx * nz, 0);
  std::vector<double> z1(nx, 0.0), z5(nx, m.zbot);
  build_interface(m, 1, z1.data());
  build_interface(m, 2, topo);
  build_interface(m, 3, sed_z);
  build_interface(m, 4, moho_z);
  build_interface(m, 5, z5.data());
  // regions in the reference's definition order (invert2d_main.f90:420-452)
  m.node_region.assign((size_t)nx * nz, 0);
  m.rnode_id.assign((size_t)nx * nz, 0);
  for (int k = 1; k <= 6; ++k) m.reg[k] = Region(), m.reg[k].id = k;
  {
    // top / bottom interface of regions 1..6
    static const int kBounds[7][2] = {{0, 0}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {2, 5}, {2, 4}};
    std::vector<std::thread> th;
    for (int k = 2; k <= 6; ++k)
      th.emplace_back([&m, k] { define_region(m, m.reg[k], kBounds[k][0], kBounds[k][1]); });
    define_region(m, m.reg[1], kBounds[1][0], kBounds[1][1]);
    for (auto& t : th) t.join();
  }
  for (int k = 1; k <= 4; ++k) claim_region(m, m.reg[k]);
  m.rright[2].clear();
  m.rleft[5].clear();
  claim_region(m, m.reg[5]);
  claim_region(m, m.reg[6]);
  // fully regular: inside some region, no cut cell among the four around it,
  // not on the grid border (propagate2d.f90:1941-1979)
  m.fully_regular.assign((size_t)nx * nz, 0);
  for (int iz = 1; iz < nz - 1; ++iz)
    for (int ix = 1; ix < nx - 1; ++ix) {
      if (m.node_region[m.g(ix, iz)] <= 0) continue;
      bool reg = true;
      for (int i = 0; i <= 1; ++i)
        for (int j = 0; j <= 1; ++j)
          if (m.cell_cut[(size_t)(iz - j) * nx + (ix - i)]) reg = false;
      m.fully_regular[m.g(ix, iz)] = reg ? 1 : 0;
    }
  for (int k = 1; k <= 5; ++k) {
    Interface& f = m.ifc[k];
    f.vel_top.assign(nx, 0.0);
    f.vel_bot.assign(nx, 0.0);
    for (int i = 0; i < nx; ++i) {
      f.vel_top[i] = vel_side(m, m.xpos[i], f.z[i] - dx);
      f.vel_bot[i] = vel_side(m, m.xpos[i], f.z[i] + dx);
    }
  }
  // each region's codes and velocities read the shared model and write only
  // that region: one thread per region
  {
    std::vector<std::thread> th;
    for (int k = 2; k <= 6; ++k) th.emplace_back([&m, k] { finish_region(m, m.reg[k]); });
    finish_region(m, m.reg[1]);
    for (auto& t : th) t.join();
  }
  // inversion numbering: velocity nodes at or below the seafloor, iz outer
  // (frechet2d.f90:55-63, invert2d_main.f90:456-477)
  m.inv_idx.assign((size_t)nx * nz, 0);
  int np = 0;
  for (int iz = 0; iz < nz; ++iz)
    for (int ix = 0; ix < nx; ++ix) {
      const int iv = std::min(ix, nx - 2);
      const double wx = std::min(1.0, std::max(0.0, double(ix - iv)));
      const double zsf = (1.0 - wx) * topo[iv] + wx * topo[iv + 1];
      if (grid_z(m, iz) - zsf >= 0.0) m.inv_idx[m.g(ix, iz)] = ++np;
    }
  m.n_vel_parms = np;
  m.n_inv_parms = np + (m.iface_inv > 0 ? nx : 0);
}

std::string update_model(Model& m, const double* vel, const double* iface_z) {
  if (m.nx == 0) return "no model";
  const size_t n = (size_t)m.nx * m.nz;
  if (vel) {
    for (size_t i = 0; i < n; ++i)
      if (!(vel[i] > 0.0)) return "velocities must be positive";
    m.vel.assign(vel, vel + n);
  }
  std::vector<double> z[6];
  for (int k = 2; k <= 4; ++k) z[k] = m.ifc[k].z;
  if (iface_z) {
    if (m.iface_inv < 2 || m.iface_inv > 4) return "no inverted interface to update";
    z[m.iface_inv].assign(iface_z, iface_z + m.nx);
  }
  const int nvp = m.n_vel_parms, npar = m.n_inv_parms;
  build_geometry(m, z[2].data(), z[3].data(), z[4].data());
  if (m.n_vel_parms != nvp || m.n_inv_parms != npar)
    return "the update changed the inversion parameters";
  return std::string();
}

namespace {

// One Gaussian row: exp(-d^2 / c^2) * mvscale(j) for the listed neighbours j
// of parameter i in the given order, then the diagonal -sum * mvscale(i).
struct GaussRow {
  std::vector<int> col;
  std::vector<double> val;
  double bsum = 0.0;
  void add(int j, double d, double c, const double* mvscale) {
    const double beta = std::exp(-(d * d) / (c * c));
    bsum = bsum + beta;
    col.push_back(j);
    val.push_back(beta * mvscale[j - 1]);
  }
  void close(int i, const double* mvscale) {
    col.push_back(i);
    val.push_back(-bsum * mvscale[i - 1]);
  }
};

}  // namespace

std::string gauss_smooth_csr(const Model& m, int which, double corr_x, double corr_z,
                             double corr_x_iface, const double* mvscale, std::vector<int>& rp,
                             std::vector<int>& col, std::vector<double>& val) {
  const int np = m.n_inv_parms;
  std::vector<GaussRow> rows(np + 1);
  if (which == 0 || which == 1) {
    if (which == 0 && !(corr_x > 0.0)) return "corr_x must be > 0";
    if (which == 1 && !(corr_z > 0.0)) return "corr_z must be > 0";
    // R_h: neighbours along the grid row within int(3 cx / dx) + 1 columns;
    // R_v: along the grid column within 3 cz (build_gauss_smooth_matrix)
    const int reach = (int)(3.0 * corr_x / m.dx) + 1;
    for (int iz = 0; iz < m.nz; ++iz)
      for (int ix = 0; ix < m.nx; ++ix) {
        const int i = m.inv_idx[m.g(ix, iz)];
        if (i <= 0) continue;
        GaussRow& R = rows[i];
        if (which == 0) {
          const int lo = std::max(0, ix - reach), hi = std::min(m.nx - 1, ix + reach);
          for (int jx = lo; jx <= hi; ++jx) {
            const int j = jx == ix ? 0 : m.inv_idx[m.g(jx, iz)];
            if (j > 0) R.add(j, grid_x(m, jx) - grid_x(m, ix), corr_x, mvscale);
          }
        } else {
          for (int jz = 0; jz < m.nz; ++jz) {
            if (jz == iz) continue;
            const double d = grid_z(m, jz) - grid_z(m, iz);
            if (std::fabs(d) > 3.0 * corr_z) continue;
            const int j = m.inv_idx[m.g(ix, jz)];
            if (j > 0) R.add(j, d, corr_z, mvscale);
          }
        }
        R.close(i, mvscale);
      }
  } else if (which == 2) {
    // interface R_h over the inverted interface's nodes (parameters
    // n_vel_parms + 1 ..), build_iface_gauss_smooth_matrix; none when the
    // correlation length is 0 or no interface is inverted
    if (corr_x_iface > 0.0 && m.iface_inv > 0) {
      const double dx_if = m.xpos[1] - m.xpos[0];
      const int reach = (int)(3.0 * corr_x_iface / dx_if) + 1;
      for (int ix = 0; ix < m.nx; ++ix) {
        const int i = m.n_vel_parms + ix + 1;
        if (i < 1 || i > np) continue;
        GaussRow& R = rows[i];
        const int lo = std::max(0, ix - reach), hi = std::min(m.nx - 1, ix + reach);
        for (int jx = lo; jx <= hi; ++jx) {
          const int j = m.n_vel_parms + jx + 1;
          if (jx != ix && j >= 1 && j <= np) R.add(j, m.xpos[jx] - m.xpos[ix], corr_x_iface, mvscale);
        }
        R.close(i, mvscale);
      }
    }
  } else {
    return "which must be 0 (R_h), 1 (R_v) or 2 (interface R_h)";
  }
  rp.assign(np + 1, 1);
  col.clear();
  val.clear();
  for (int i = 1; i <= np; ++i) {
    col.insert(col.end(), rows[i].col.begin(), rows[i].col.end());
    val.insert(val.end(), rows[i].val.begin(), rows[i].val.end());
    rp[i] = (int)col.size() + 1;
  }
  return std::string();
}

std::string projection(const Model& m, int kx, int kz, int ki, std::vector<int>& coarse_idx,
                       int& nxc, int& nzc, int& nvp_c, int& npar_c, std::vector<int>& rp,
                       std::vector<int>& col, std::vector<double>& val) {
  if (kx < 1 || kz < 1 || ki < 1) return "refinement ratios must be >= 1";
  nxc = (m.nx - 1 + kx - 1) / kx + 1;
  nzc = (m.nz - 1 + kz - 1) / kz + 1;
  // corners and weights of each fine velocity parameter: fine node (ix, iz)
  // lies in coarse cell (ix / kx, iz / kz) at fractions (ix % kx) / kx,
  // (iz % kz) / kz, exact for integer ratios (ratio 1 gives weight 1)
  struct W { int c[4]; double w[4]; };
  std::vector<W> fw(m.n_vel_parms + 1);
  std::vector<uint8_t> used((size_t)nxc * nzc, 0);
  for (int iz = 0; iz < m.nz; ++iz)
    for (int ix = 0; ix < m.nx; ++ix) {
      const int f = m.inv_idx[m.g(ix, iz)];
      if (f <= 0) continue;
      const int i = ix / kx, j = iz / kz;
      const double a = (double)(ix % kx) / kx, b = (double)(iz % kz) / kz;
      W& w = fw[f];
      const int ci[4] = {i, i + 1, i, i + 1}, cj[4] = {j, j, j + 1, j + 1};
      const double ww[4] = {(1.0 - a) * (1.0 - b), a * (1.0 - b), (1.0 - a) * b, a * b};
      for (int k = 0; k < 4; ++k) {
        const bool in = ci[k] < nxc && cj[k] < nzc && ww[k] != 0.0;
        w.c[k] = in ? cj[k] * nxc + ci[k] : -1;
        w.w[k] = ww[k];
        if (in) used[(size_t)w.c[k]] = 1;
      }
    }
  // coarse velocity parameters: the touched coarse nodes, iz outer / ix inner
  coarse_idx.assign((size_t)nxc * nzc, 0);
  nvp_c = 0;
  for (size_t c = 0; c < used.size(); ++c)
    if (used[c]) coarse_idx[c] = ++nvp_c;
  // coarse interface nodes every ki fine interface nodes
  const int nic = m.iface_inv > 0 ? (m.nx - 1 + ki - 1) / ki + 1 : 0;
  npar_c = nvp_c + nic;
  rp.assign(m.n_inv_parms + 1, 1);
  col.clear();
  val.clear();
  for (int f = 1; f <= m.n_inv_parms; ++f) {
    if (f <= m.n_vel_parms) {
      const W& w = fw[f];
      for (int k = 0; k < 4; ++k)
        if (w.c[k] >= 0) {
          col.push_back(coarse_idx[(size_t)w.c[k]]);
          val.push_back(w.w[k]);
        }
    } else {
      const int ix = f - m.n_vel_parms - 1, i = ix / ki;
      const double a = (double)(ix % ki) / ki;
      col.push_back(nvp_c + i + 1);
      val.push_back(1.0 - a);
      if (a != 0.0 && i + 1 < nic) {
        col.push_back(nvp_c + i + 2);
        val.push_back(a);
      }
    }
    rp[f] = (int)col.size() + 1;
  }
  return std::string();
}

void project_rows(int ndata, const int* row_ptr, const int* gindx, const double* gval,
                  int nfine, const int* prp, const int* pcol, const double* pval,
                  std::vector<int>& rp, std::vector<int>& col, std::vector<double>& val) {
  rp.assign(ndata + 1, 1);
  col.clear();
  val.clear();
  std::vector<std::pair<int, double>> acc;
  for (int i = 0; i < ndata; ++i) {
    acc.clear();
    for (int k = row_ptr[i] - 1; k < row_ptr[i + 1] - 1; ++k) {
      const int f = gindx[k];
      if (f < 1 || f > nfine) continue;
      for (int q = prp[f - 1] - 1; q < prp[f] - 1; ++q) acc.emplace_back(pcol[q], gval[k] * pval[q]);
    }
    // ascending coarse columns; equal columns summed in the order of the fine entries
    std::stable_sort(acc.begin(), acc.end(),
                     [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                       return a.first < b.first;
                     });
    for (size_t q = 0; q < acc.size();) {
      double s = 0.0;
      const int c = acc[q].first;
      for (; q < acc.size() && acc[q].first == c; ++q) s = s + acc[q].second;
      col.push_back(c);
      val.push_back(s);
    }
    rp[i + 1] = (int)col.size() + 1;
  }
}

int select_data(int npick, const int* phase, const double* obs, const double* t_calc,
                const int* valid, const int* row_ptr, const int* gindx, const double* gval,
                int nparm, const double* mvscale, double crit_chi, const double* phase_wt,
                int* row_ptr_out, int* gindx_out, double* gval_out, double* residual,
                double* data_wt, int* pick_of_row) {
  int nd = 0, kk = 0;
  row_ptr_out[0] = 1;
  for (int p = 0; p < npick; ++p) {
    if (!valid[p] || obs[p] < 0.0) continue;
    const double res = obs[p] - t_calc[p];
    if (std::fabs(res) > crit_chi) continue;
    const int ph = phase[p];
    const double wt = (ph == 2 || ph == 3) ? 1.0 * phase_wt[ph - 2]
                      : (ph == 4 || ph == 5) ? 1.0 * phase_wt[2] : 1.0;
    for (int k = row_ptr[p] - 1; k < row_ptr[p + 1] - 1; ++k) {
      const int j = gindx[k];
      gindx_out[kk] = j;
      gval_out[kk] = (j >= 1 && j <= nparm) ? gval[k] * mvscale[j - 1] * wt : gval[k];
      ++kk;
    }
    residual[nd] = res * wt;
    data_wt[nd] = wt;
    pick_of_row[nd] = p;
    ++nd;
    row_ptr_out[nd] = kk + 1;
  }
  return nd;
}

namespace {

// The four propagation-grid nodes and bilinear weights of vel_side(m, px,
// pzoff): vel_side's value is sum_k w[k] * m.vel[node[k]], summed in k order.
void vel_side_w(const Model& m, double px, double pzoff, int* node, double* w) {
  const int nx = m.nx, nz = m.nz;
  const double dxv = m.xpos[1] - m.xpos[0];
  int ivx = (int)std::floor((px - m.xpos[0]) / dxv);
  ivx = std::max(0, std::min(nx - 2, ivx));
  const double wx = std::min(1.0, std::max(0.0, (px - m.xpos[ivx]) / dxv));
  int ivz;
  double wz;
  if (pzoff < grid_z(m, 0)) { ivz = 0; wz = 0.0; }
  else if (pzoff >= grid_z(m, nz - 1)) { ivz = nz - 2; wz = 1.0; }
  else {
    for (ivz = 0; ivz < nz - 1; ++ivz)
      if (pzoff >= grid_z(m, ivz) && pzoff < grid_z(m, ivz + 1)) break;
    if (ivz >= nz - 1) ivz = nz - 2;
    const double up = grid_z(m, ivz + 1) - grid_z(m, ivz);
    wz = up > 0.0 ? (pzoff - grid_z(m, ivz)) / up : 0.0;
  }
  wz = std::min(1.0, std::max(0.0, wz));
  node[0] = (int)m.g(ivx, ivz);
  node[1] = (int)m.g(ivx + 1, ivz);
  node[2] = (int)m.g(ivx, ivz + 1);
  node[3] = (int)m.g(ivx + 1, ivz + 1);
  w[0] = (1.0 - wx) * (1.0 - wz);
  w[1] = wx * (1.0 - wz);
  w[2] = (1.0 - wx) * wz;
  w[3] = wx * wz;
}

// d vel_side(m, px, pzoff) / d pzoff: the bilinear sample's slope in depth
// inside the bracketing rows (0 where the sample is clamped to the grid).
double vel_side_dz(const Model& m, double px, double pzoff) {
  const int nx = m.nx, nz = m.nz;
  const double dxv = m.xpos[1] - m.xpos[0];
  int ivx = (int)std::floor((px - m.xpos[0]) / dxv);
  ivx = std::max(0, std::min(nx - 2, ivx));
  const double wx = std::min(1.0, std::max(0.0, (px - m.xpos[ivx]) / dxv));
  if (pzoff < grid_z(m, 0) || pzoff >= grid_z(m, nz - 1)) return 0.0;
  int ivz;
  for (ivz = 0; ivz < nz - 1; ++ivz)
    if (pzoff >= grid_z(m, ivz) && pzoff < grid_z(m, ivz + 1)) break;
  if (ivz >= nz - 1) return 0.0;
  const double up = grid_z(m, ivz + 1) - grid_z(m, ivz);
  if (!(up > 0.0)) return 0.0;
  auto V = [&](int a, int b) { return m.vel[m.g(a, b)]; };
  return ((1.0 - wx) * (V(ivx, ivz + 1) - V(ivx, ivz)) +
          wx * (V(ivx + 1, ivz + 1) - V(ivx + 1, ivz))) / up;
}

}  // namespace

std::string slot_velocity_map(const Model& m, int reg, std::vector<int>& rp,
                              std::vector<int>& slot, std::vector<double>& w,
                              std::vector<int>* zrp, std::vector<int>* zslot,
                              std::vector<int>* zside, std::vector<double>* zdv) {
  if (reg < 1 || reg > 6) return "region out of range";
  const Region& r = m.reg[reg];
  const int nx = m.nx;
  const Interface& ft = m.ifc[r.itop];
  const Interface& fb = m.ifc[r.ibot];
  const double dx = m.dx;
  const size_t nn = (size_t)nx * m.nz;
  // per slot: up to four (node, weight) pairs, as finish_region assigns the
  // slot's velocity
  const size_t ns = r.nslots();
  std::vector<int> sn(ns * 4, -1);
  std::vector<double> sw(ns * 4, 0.0);
  auto side_k = [&](int ix) {
    int k = (int)std::lround((grid_x(m, ix) - m.xpos[0]) / m.dx);
    return std::max(0, std::min(nx - 1, k));
  };
  // slots sampled off an interface: (column k, side 0 top / 1 bottom, slot,
  // d velocity / d interface depth)
  struct ZE { int k, side, s; double dv; };
  std::vector<ZE> ze;
  for (int iz = r.z_lo; iz <= r.z_hi; ++iz)
    for (int ix = 0; ix < nx; ++ix) {
      if (iz < r.r0[ix] || iz > r.r1[ix]) continue;
      const size_t s = (size_t)r.slot_grid(ix, iz);
      if (iz > 0 && !in_region(r, ix, iz - 1)) {
        const int k = side_k(ix);
        vel_side_w(m, m.xpos[k], ft.z[k] + dx, &sn[4 * s], &sw[4 * s]);
        ze.push_back({k, 0, (int)s, vel_side_dz(m, m.xpos[k], ft.z[k] + dx)});
      } else if (iz < m.nz - 1 && !in_region(r, ix, iz + 1)) {
        const int k = side_k(ix);
        vel_side_w(m, m.xpos[k], fb.z[k] - dx, &sn[4 * s], &sw[4 * s]);
        ze.push_back({k, 1, (int)s, vel_side_dz(m, m.xpos[k], fb.z[k] - dx)});
      } else {
        sn[4 * s] = (int)m.g(ix, iz);
        sw[4 * s] = 1.0;
      }
    }
  for (int k = 0; k < nx; ++k) {
    const size_t st = (size_t)r.slot_top(k), sb = (size_t)r.slot_bot(k);
    vel_side_w(m, m.xpos[k], ft.z[k] + dx, &sn[4 * st], &sw[4 * st]);
    vel_side_w(m, m.xpos[k], fb.z[k] - dx, &sn[4 * sb], &sw[4 * sb]);
    ze.push_back({k, 0, (int)st, vel_side_dz(m, m.xpos[k], ft.z[k] + dx)});
    ze.push_back({k, 1, (int)sb, vel_side_dz(m, m.xpos[k], fb.z[k] - dx)});
  }
  if (zrp) {
    std::stable_sort(ze.begin(), ze.end(), [](const ZE& a, const ZE& b) {
      return a.k != b.k ? a.k < b.k : a.s < b.s;
    });
    zrp->assign(nx + 1, 0);
    zslot->resize(ze.size());
    zside->resize(ze.size());
    zdv->resize(ze.size());
    for (size_t i = 0; i < ze.size(); ++i) {
      ++(*zrp)[ze[i].k + 1];
      (*zslot)[i] = ze[i].s;
      (*zside)[i] = ze[i].side;
      (*zdv)[i] = ze[i].dv;
    }
    for (int k = 0; k < nx; ++k) (*zrp)[k + 1] += (*zrp)[k];
  }
  // the map must reproduce every slot's velocity bit for bit
  for (size_t s = 0; s < ns; ++s) {
    if (sn[4 * s] < 0) continue;
    double v = sw[4 * s] * m.vel[sn[4 * s]];
    if (sw[4 * s] != 1.0 || sn[4 * s + 1] >= 0)
      for (int k = 1; k < 4; ++k) v = v + sw[4 * s + k] * m.vel[sn[4 * s + k]];
    if (v != r.vel64[s])
      return "slot velocity map does not reproduce region " + std::to_string(reg) +
             " slot " + std::to_string(s);
  }
  // transposed, node-major, slots ascending within a node
  rp.assign(nn + 1, 0);
  for (size_t s = 0; s < ns; ++s)
    for (int k = 0; k < 4; ++k)
      if (sn[4 * s + k] >= 0 && sw[4 * s + k] != 0.0) ++rp[sn[4 * s + k] + 1];
  for (size_t i = 0; i < nn; ++i) rp[i + 1] += rp[i];
  slot.assign(rp[nn], 0);
  w.assign(rp[nn], 0.0);
  std::vector<int> fill(rp.begin(), rp.end() - 1);
  for (size_t s = 0; s < ns; ++s)
    for (int k = 0; k < 4; ++k)
      if (sn[4 * s + k] >= 0 && sw[4 * s + k] != 0.0) {
        const int j = fill[sn[4 * s + k]]++;
        slot[j] = (int)s;
        w[j] = sw[4 * s + k];
      }
  return std::string();
}

}  // namespace fmt2d
