// Ray backtrace, water-leg entry search and Frechet rows on the device, one
// thread per pick, FP64 with the reference's expression order (this file is
// compiled without FMA contraction, like the eikonal stencil).
//
//   trace_ray_from_receiver2d   src/rays2d.f90:7-153
//   trace_ray_section2d         src/rays2d.f90:157-720 (Heun steps along -grad T
//                               with step halving; interface, head-wave and
//                               diffraction handling; source snap)
//   find_interface_crossing2d   src/rays2d.f90:764-821
//   interpolate_*               src/rays2d.f90:825-1131, 1222-1350
//   find_optimal_entry_inv      src/inversion2d.f90:6344-6438
//   compute_frechet_for_ray2d   src/inversion2d.f90:4548-4787
//
// A section's points are not stored: each segment is turned into its four
// slowness-derivative contributions as soon as both ends are final (only the
// last point of a section is ever moved after it is computed), consecutive
// segments that touch the same four parameters are merged, and the
// contributions are written as (pick, parameter) keys.  The caller sorts
// the keys and sums equal ones into CSR rows.
#include "rays.cuh"
#include "model.h"
#include <cmath>

namespace fmt2d {

namespace {

constexpr double kHugeT = 1.0e20;   // mod_fmt2d.f90:616
constexpr int kMaxPoints = 5000;    // rays2d.f90:206
constexpr int kMaxSec = 4;

// Phase tables (invert2d_main.f90:564-700): interface sequence (1-based,
// 2*n_tf entries) and time-field sequence.
__constant__ int c_ntf[6] = {0, 1, 2, 2, 4, 4};
__constant__ int c_seq[6][9] = {{0}, {0, 0, 2}, {0, 0, 3, 3, 0}, {0, 0, 4, 4, 0},
                                {0, 0, 2, 2, 1, 1, 2, 2, 2}, {0, 0, 1, 1, 2, 2, 2, 2, 2}};
__constant__ int c_tfs[6][5] = {{0}, {0, 1}, {0, 2, 3}, {0, 4, 5}, {0, 1, 6, 7, 8},
                                {0, 9, 10, 11, 12}};
__constant__ int c_tfreg[13] = {0, 5, 2, 2, 6, 6, 1, 1, 1, 1, 1, 5, 1};

__device__ __forceinline__ double gxc(const TrModel& M, int ix) { return M.x0 + (ix - 1) * M.dx; }
__device__ __forceinline__ double gzc(const TrModel& M, int iz) { return 0.0 + (iz - 1) * M.dx; }
__device__ __forceinline__ double clamp01(double w) { return fmin(1.0, fmax(0.0, w)); }

// Slot of grid node (ix, iz) (1-based) if it belongs to region r, else -1.
__device__ __forceinline__ int region_node(const TrModel& M, const TrRegion& r, int ix, int iz) {
  if (ix < 1 || ix > M.nx || iz < 1 || iz > M.nz) return -1;
  const int br = iz - 1 - r.z_lo;
  if (br < 0 || br >= r.H) return -1;
  const int s = br * r.pitch + (ix - 1);
  return (r.code[s] & kInRegion) ? s : -1;
}

__device__ void node_pos(const TrModel& M, const TrRegion& r, int s, double& x, double& z) {
  const int row = s / r.pitch, col = s - row * r.pitch;
  if (row < r.H) {
    x = gxc(M, col + 1);
    z = gzc(M, r.z_lo + row + 1);
  } else {
    x = M.xpos[col];
    z = M.ifz[row == r.H ? r.itop : r.ibot][col];
  }
}

// rays2d.f90:996-1020: nearest region node in the same column, up to five
// rows away (below first).
__device__ int nearby_node(const TrModel& M, const TrRegion& r, int ix, int iz) {
  for (int d = 1; d <= 5; ++d) {
    int s = region_node(M, r, ix, iz + d);
    if (s >= 0) return s;
    s = region_node(M, r, ix, iz - d);
    if (s >= 0) return s;
  }
  return -1;
}

// The region node nearest to (px, pz), the first in the reference's node
// order among equals (grid nodes column by column, rows down each column,
// then the top and the bottom interface nodes by column): what a scan of
// every node with a strict "closer" test returns (rays2d.f90:966-972,
// 1118-1127).  The region's grid nodes are one row range per column, so the
// search widens column by column from the query and stops once a column's
// horizontal distance alone exceeds the best distance found; each column
// costs its nearest rows and its two interface nodes.
__device__ int nearest_node(const TrModel& M, const TrRegion& r, double px, double pz) {
  double best = 1.0e300;
  int bcls = 3, bcol = 0, brow = 0, bslot = -1;
  auto offer = [&](double d, int cls, int col, int row, int slot) {
    if (d < best || (d == best && (cls < bcls || (cls == bcls && (col < bcol ||
                                                  (col == bcol && row < brow)))))) {
      best = d; bcls = cls; bcol = col; brow = row; bslot = slot;
    }
  };
  const int nx = M.nx;
  int c0 = (int)floor((px - M.x0) / M.dx);
  c0 = max(0, min(nx - 1, c0));
  const int fr = (int)floor(pz / M.dx);
  // columns c0, c0 - 1, c0 + 1, c0 - 2, ...: the horizontal distance grows on
  // each side, so once neither side's next column can hold a node as close as
  // the best (d >= its horizontal term), no farther column can either
  for (int k = 0;; ++k) {
    bool near = false;
    for (int side = 0; side < (k == 0 ? 1 : 2); ++side) {
      const int c = side == 0 ? c0 - k : c0 + k;
      if (c < 0 || c >= nx) continue;
      const double gx = gxc(M, c + 1), xi = M.xpos[c];
      if ((px - gx) * (px - gx) > best && (px - xi) * (px - xi) > best) continue;
      near = true;
      const int a = r.r0[c], b = r.r1[c];
      if (a <= b) {
#pragma unroll
        for (int q = -1; q <= 2; ++q) {
          const int row = min(b, max(a, fr + q));
          const double z = gzc(M, row + 1);
          offer((px - gx) * (px - gx) + (pz - z) * (pz - z), 0, c, row,
                (row - r.z_lo) * r.pitch + c);
        }
      }
      const double zt = M.ifz[r.itop][c], zb = M.ifz[r.ibot][c];
      offer((px - xi) * (px - xi) + (pz - zt) * (pz - zt), 1, c, 0, r.H * r.pitch + c);
      offer((px - xi) * (px - xi) + (pz - zb) * (pz - zb), 2, c, 0, (r.H + 1) * r.pitch + c);
    }
    if (!near && k > 0) break;
  }
  return bslot;
}

// rays2d.f90:1070-1131: nearest of the cell corners, else of every region
// node (in the reference's node order).
__device__ int position_in_region(const TrModel& M, const TrRegion& r, double px, double pz) {
  int ix = (int)floor((px - M.x0) / M.dx) + 1;
  int iz = (int)floor((pz - 0.0) / M.dx) + 1;
  ix = max(1, min(M.nx - 1, ix));
  iz = max(1, min(M.nz - 1, iz));
  double dmin = 1.0e100;
  int best = -1;
  for (int ii = ix; ii <= ix + 1; ++ii)
    for (int jj = iz; jj <= iz + 1; ++jj) {
      const int s = region_node(M, r, ii, jj);
      if (s >= 0) {
        double x, z;
        node_pos(M, r, s, x, z);
        const double d = (px - x) * (px - x) + (pz - z) * (pz - z);
        if (d < dmin) { best = s; dmin = d; }
      }
    }
  if (best < 0) best = nearest_node(M, r, px, pz);
  return best;
}

// rays2d.f90:825-894
__device__ void grad_at(const TrModel& M, const TrRegion& r, const double2* G, double px,
                        double pz, double& dtdx, double& dtdz) {
  int ix = (int)floor((px - M.x0) / M.dx) + 1;
  int iz = (int)floor((pz - 0.0) / M.dx) + 1;
  ix = max(1, min(M.nx - 1, ix));
  iz = max(1, min(M.nz - 1, iz));
  const double w1 = clamp01((px - gxc(M, ix)) / M.dx);
  const double w2 = clamp01((pz - gzc(M, iz)) / M.dx);
  int n1 = region_node(M, r, ix, iz), n2 = region_node(M, r, ix + 1, iz);
  int n3 = region_node(M, r, ix, iz + 1), n4 = region_node(M, r, ix + 1, iz + 1);
  if (n1 < 0) n1 = nearby_node(M, r, ix, iz);
  if (n2 < 0) n2 = nearby_node(M, r, ix + 1, iz);
  if (n3 < 0) n3 = nearby_node(M, r, ix, iz + 1);
  if (n4 < 0) n4 = nearby_node(M, r, ix + 1, iz + 1);
  double g1x = 0, g2x = 0, g3x = 0, g4x = 0, g1z = 0, g2z = 0, g3z = 0, g4z = 0;
  if (n1 >= 0) { g1x = G[n1].x; g1z = G[n1].y; }
  if (n2 >= 0) { g2x = G[n2].x; g2z = G[n2].y; }
  if (n3 >= 0) { g3x = G[n3].x; g3z = G[n3].y; }
  if (n4 >= 0) { g4x = G[n4].x; g4z = G[n4].y; }
  double gx = (1.0 - w1) * (1.0 - w2) * g1x + w1 * (1.0 - w2) * g2x + (1.0 - w1) * w2 * g3x +
              w1 * w2 * g4x;
  double gz = (1.0 - w1) * (1.0 - w2) * g1z + w1 * (1.0 - w2) * g2z + (1.0 - w1) * w2 * g3z +
              w1 * w2 * g4z;
  if (sqrt(gx * gx + gz * gz) < 0.01) {
    const int nm = position_in_region(M, r, px, pz);
    gx = 0.0;
    gz = 0.0;
    if (nm >= 0) { gx = G[nm].x; gz = G[nm].y; }
  }
  dtdx = gx;
  dtdz = gz;
}

// rays2d.f90:898-975
__device__ double time_at(const TrModel& M, const TrRegion& r, const double* T, double px,
                          double pz) {
  int ix = (int)floor((px - M.x0) / M.dx) + 1;
  int iz = (int)floor((pz - 0.0) / M.dx) + 1;
  ix = max(1, min(M.nx - 1, ix));
  iz = max(1, min(M.nz - 1, iz));
  const double w1 = clamp01((px - gxc(M, ix)) / M.dx);
  const double w2 = clamp01((pz - gzc(M, iz)) / M.dx);
  auto tn = [&](int a, int b) {
    int s = region_node(M, r, a, b);
    if (s < 0) s = nearby_node(M, r, a, b);
    return s >= 0 ? T[s] : kHugeT;
  };
  const double t1 = tn(ix, iz), t2 = tn(ix + 1, iz), t3 = tn(ix, iz + 1), t4 = tn(ix + 1, iz + 1);
  const double hh = kHugeT * 0.5;
  if (t1 < hh && t2 < hh && t3 < hh && t4 < hh)
    return (1.0 - w1) * (1.0 - w2) * t1 + w1 * (1.0 - w2) * t2 + (1.0 - w1) * w2 * t3 +
           w1 * w2 * t4;
  const int s = nearest_node(M, r, px, pz);
  return s >= 0 ? T[s] : kHugeT;
}

// rays2d.f90:1222-1257
__device__ double iface_z(const TrModel& M, double px, int k) {
  const int nn = M.nx;
  const double* z = M.ifz[k];
  if (nn < 2) return z[0];
  const int ix = (int)floor((px - M.xpos[0]) / M.dx) + 1;
  if (ix < 1) return z[0];
  if (ix >= nn) return z[nn - 1];
  const double w = clamp01((px - M.xpos[ix - 1]) / M.dx);
  return (1.0 - w) * z[ix - 1] + w * z[ix];
}

// rays2d.f90:1261-1306
__device__ void iface_normal(const TrModel& M, double px, int k, double& nx, double& nz) {
  const int nn = M.nx;
  const double* z = M.ifz[k];
  const double dx = M.dx;
  if (nn < 2) { nx = 0.0; nz = 1.0; return; }
  int ix = (int)floor((px - M.xpos[0]) / dx) + 1;
  if (ix < 1) ix = 1;
  if (ix >= nn) ix = nn - 1;
  double dzdx;
  if (ix > 1 && ix < nn - 1) dzdx = (z[ix] - z[ix - 2]) / (2.0 * dx);
  else if (ix == 1 && nn >= 3) dzdx = (z[ix] - z[ix - 1]) / dx;
  else if (ix == nn - 1 && nn >= 3) dzdx = (z[ix] - z[ix - 2]) / (2.0 * dx);
  else dzdx = 0.0;
  const double l = sqrt(1.0 + dzdx * dzdx);
  nx = -dzdx / l;
  nz = 1.0 / l;
}

// rays2d.f90:1310-1350: bilinear propagation-grid velocity.
__device__ double vel_at(const TrModel& M, double px, double pz) {
  int ix = (int)floor((px - M.x0) / M.dx) + 1;
  int iz = (int)floor((pz - 0.0) / M.dx) + 1;
  ix = max(1, min(M.nx - 1, ix));
  iz = max(1, min(M.nz - 1, iz));
  const double w1 = clamp01((px - gxc(M, ix)) / M.dx);
  const double w2 = clamp01((pz - gzc(M, iz)) / M.dx);
  auto V = [&](int a, int b) { return M.vel[(size_t)(b - 1) * M.nx + (a - 1)]; };
  return (1.0 - w1) * (1.0 - w2) * V(ix, iz) + w1 * (1.0 - w2) * V(ix + 1, iz) +
         (1.0 - w1) * w2 * V(ix, iz + 1) + w1 * w2 * V(ix + 1, iz + 1);
}

// Frechet contributions of one pick, written or counted.
struct Sink {
  unsigned long long* keys;
  double* vals;
  unsigned long long base;   // first entry of this pick
  unsigned n;                // entries so far
  unsigned long long row;    // pick << 32
  int pend_idx[4];
  double pend_val[4];
  int npend;
};

__device__ __forceinline__ void sink_flush(Sink& k) {
  for (int i = 0; i < k.npend; ++i) {
    if (k.keys) {
      k.keys[k.base + k.n] = k.row | (unsigned)k.pend_idx[i];
      k.vals[k.base + k.n] = k.pend_val[i];
    }
    ++k.n;
  }
  k.npend = 0;
}

// inversion2d.f90:4581-4673: midpoint-rule bilinear splat of one segment's
// length onto the four inversion nodes around its midpoint.
__device__ void segment(const TrModel& M, Sink& k, double x0, double z0, double x1, double z1) {
  const double px = 0.5 * (x0 + x1), pz = 0.5 * (z0 + z1);
  const double ddx = x1 - x0, ddz = z1 - z0;
  const double sl = sqrt(ddx * ddx + ddz * ddz);
  if (sl < 1.0e-10) return;
  const double vdx = M.xpos[1] - M.xpos[0];
  int ivx = (int)floor((px - M.xpos[0]) / vdx) + 1;
  ivx = max(1, min(M.nx - 1, ivx));
  int ivz;
  double wz;
  if (pz < gzc(M, 1)) return;
  if (pz >= gzc(M, M.nz)) {
    ivz = M.nz - 1;
    wz = 1.0;
  } else {
    ivz = (int)floor((pz - gzc(M, 1)) / M.dx) + 1;
    ivz = max(1, min(M.nz - 1, ivz));
    wz = (pz - gzc(M, ivz)) / M.dx;
  }
  const double wx = clamp01((px - M.xpos[ivx - 1]) / vdx);
  wz = clamp01(wz);
  int idx[4];
  double w[4];
  idx[0] = M.inv_idx[(size_t)(ivz - 1) * M.nx + (ivx - 1)];
  idx[1] = M.inv_idx[(size_t)(ivz - 1) * M.nx + ivx];
  idx[2] = M.inv_idx[(size_t)ivz * M.nx + (ivx - 1)];
  idx[3] = M.inv_idx[(size_t)ivz * M.nx + ivx];
  w[0] = (1.0 - wx) * (1.0 - wz) * sl;
  w[1] = wx * (1.0 - wz) * sl;
  w[2] = (1.0 - wx) * wz * sl;
  w[3] = wx * wz * sl;
  // merge with the previous segment when it touched the same parameters
  int m = 0, q[4];
  double v[4];
  for (int i = 0; i < 4; ++i)
    if (idx[i] > 0) { q[m] = idx[i]; v[m] = w[i]; ++m; }
  bool same = m == k.npend;
  for (int i = 0; same && i < m; ++i) same = q[i] == k.pend_idx[i];
  if (same) {
    for (int i = 0; i < m; ++i) k.pend_val[i] += v[i];
    return;
  }
  sink_flush(k);
  for (int i = 0; i < m; ++i) { k.pend_idx[i] = q[i]; k.pend_val[i] = v[i]; }
  k.npend = m;
}

__device__ void add_one(Sink& k, int idx, double v) {
  sink_flush(k);
  k.pend_idx[0] = idx;
  k.pend_val[0] = v;
  k.npend = 1;
  sink_flush(k);
}

struct Section {
  int tf, reg, istart, iend;
  int npts;
  double x1, z1;           // first point
  bool headwave, diffracted;
};

struct RayState {
  const TrModel* M;
  const TrField* F;        // this pick's source fields (indexed by tf)
  double sx, sz;           // source
  int raypath, nsec;
  Section sec[kMaxSec + 1];
  bool valid, headwave, diffracted;
  Sink* sink;
};

// find_interface_crossing2d (rays2d.f90:764-821).  On success X/Z (the
// current point) hold the crossing.
__device__ bool crossing(const TrModel& M, double Xp, double Zp, double& Xc, double& Zc,
                         double ppx, double ppz, int ie, double g0x, double g0z, double dl) {
  const double tol = 0.01 * M.tol;
  const double zi = iface_z(M, ppx, ie);
  const double x1 = 0.0, x2 = dl;
  const double f = Zp - iface_z(M, Xp, ie);
  double fmid = ppz - zi;
  if (f * fmid > tol) return false;
  if (fabs(f * fmid) <= tol) {
    Xc = Xp;
    Zc = iface_z(M, Xc, ie);
    return true;
  }
  if (f * fmid < -tol) {
    double rtbis, dxx;
    if (f < 0.0) { rtbis = x1; dxx = x2 - x1; }
    else { rtbis = x2; dxx = x1 - x2; }
    for (int k = 1; k <= 10; ++k) {
      dxx *= 0.5;
      const double xm = rtbis + dxx;
      Xc = Xp - xm * g0x;
      Zc = Zp - xm * g0z;
      fmid = Zc - iface_z(M, Xc, ie);
      if (fmid <= 0.0) rtbis = xm;
    }
    Xc = Xp - rtbis * g0x;
    Zc = Zp - rtbis * g0z;
    Zc = iface_z(M, Xc, ie);
  }
  return true;
}

// trace_ray_section2d (rays2d.f90:157-720) of section seqnum.
__device__ void trace_section(RayState& R, int seqnum, double x_in, double z_in, double& x_out,
                              double& z_out) {
  const TrModel& M = *R.M;
  Section& rs = R.sec[seqnum];
  const TrRegion& reg = M.reg[rs.reg];
  const TrField& tf = R.F[rs.tf];
  const int iftop = reg.itop, ifbot = reg.ibot;
  const double v_average = 5.0;
  bool refraction = false;
  int start_direction = 0;
  int ifend = 0;               // interface id the section ends on (0 none)
  int tfn = 0;                 // next section's time field
  const int nsec = R.nsec;
  if (seqnum < nsec && seqnum > 1) {
    ifend = rs.iend;
    tfn = R.sec[seqnum - 1].tf;
    start_direction = reg.id - M.reg[c_tfreg[R.sec[seqnum + 1].tf]].id;
    refraction = M.reg[c_tfreg[tfn]].id != reg.id;
  }
  if (seqnum == nsec && seqnum > 1) {
    ifend = rs.iend;
    tfn = R.sec[seqnum - 1].tf;
    start_direction = 0;
    refraction = M.reg[c_tfreg[tfn]].id != reg.id;
  }
  if (seqnum == 1) {
    ifend = 0;
    tfn = 0;
    start_direction =
        (seqnum + 1 <= nsec) ? reg.id - M.reg[c_tfreg[R.sec[seqnum + 1].tf]].id : 0;
  }
  bool same_internal = false, left_start = true;
  if (ifend && rs.istart) {
    same_internal = (ifend == rs.istart && ifend != iftop && ifend != ifbot);
    if (same_internal) left_start = false;
  }
  const double dlmax = 0.1 * M.dx * v_average;
  const double p_tol = 5.0e-4 * M.dx;
  const double s_tol = 2.5 * M.dx;
  const bool emit = rs.reg != 1;   // water sections carry no slowness derivatives
  // points: current (n), previous (n-1), the one before (n-2)
  int n = 1;
  double Xc = x_in, Zc = z_in, Xp = 0, Zp = 0, Xpp = 0, Zpp = 0;
  double dist_hw = 0.0;
  const bool on_bot = fabs(z_in - iface_z(M, x_in, ifbot)) < 0.1 * M.dx;
  const bool on_top = fabs(z_in - iface_z(M, x_in, iftop)) < 0.1 * M.dx;
  const TrRegion* nreg = tfn ? &M.reg[c_tfreg[tfn]] : nullptr;
  const TrField* nfield = tfn ? &R.F[tfn] : nullptr;
  rs.x1 = x_in;
  rs.z1 = z_in;
  rs.headwave = false;
  rs.diffracted = false;
  auto finish = [&](int npts) {
    rs.npts = npts;
    if (emit && npts >= 2) segment(M, *R.sink, Xp, Zp, Xc, Zc);
  };
  auto near_src = [&](double x, double z) {
    const double dx = x - R.sx, dz = z - R.sz;
    return sqrt(dx * dx + dz * dz) < s_tol;
  };
  auto refracts = [&](double px, double zi, double& g0x, double& g0z) {
    double nx, nz;
    iface_normal(M, px, ifend, nx, nz);
    double g1x, g1z;
    grad_at(M, reg, tf.G, px, zi, g0x, g0z);
    grad_at(M, *nreg, nfield->G, px, zi, g1x, g1z);
    const double d = nx * g1x + nz * g1z;
    const double tx = g1x - d * nx, tz = g1z - d * nz;
    return sqrt(tx * tx + tz * tz) <= sqrt(g0x * g0x + g0z * g0z);
  };
  double g0x = 0, g0z = 0, g1x = 0, g1z = 0, ppx = 0, ppz = 0, dl = dlmax;
  for (;;) {  // ploop
    ++n;
    Xpp = Xp; Zpp = Zp;
    Xp = Xc; Zp = Zc;
    if (emit && n >= 3) segment(M, *R.sink, Xpp, Zpp, Xp, Zp);
    if (n > kMaxPoints) { R.valid = false; return; }
    if (seqnum == 1 && n > 2 && near_src(Xp, Zp)) {
      Xc = R.sx; Zc = R.sz;
      finish(n);
      return;
    }
    if (R.headwave || R.diffracted) {
      if (n > 2) {
        const double ddx = Xp - Xpp, ddz = Zp - Zpp;
        dist_hw += sqrt(ddx * ddx + ddz * ddz);
      }
      if (dist_hw > 200.0) { R.valid = false; return; }
    }
    dl = dlmax;
    if (n == 2 && (on_bot || on_top)) dl = 10.0 * dlmax;
    grad_at(M, reg, tf.G, Xp, Zp, g0x, g0z);
    ppx = Xp - dl * g0x;
    ppz = Zp - dl * g0z;
    if (on_bot && ppz > Zp) ppz = 2.0 * Zp - ppz;
    if (on_top && ppz < Zp) ppz = 2.0 * Zp - ppz;
    if (n == 2 && start_direction != 0 && !refraction && seqnum != 1) {
      double nx, nz;
      iface_normal(M, x_in, rs.istart, nx, nz);
      if (g0x * start_direction * nx + g0z * start_direction * nz > 0.0) { R.valid = false; return; }
    }
    if (ifend && ifend != iftop && ifend != ifbot) {
      const double fp = Zp - iface_z(M, Xp, ifend);
      const double fn = ppz - iface_z(M, ppx, ifend);
      if (same_internal && !left_start) {
        if (fabs(fn) > 0.5 * M.dx) left_start = true;
      } else if (fabs(fp) > 1.0e-3) {
        if (fp * fn <= 0.0) {
          double fr = fabs(fp - fn) > 1.0e-12 ? fp / (fp - fn) : 1.0;
          fr = fmin(1.0, fmax(0.0, fr));
          Xc = Xp + fr * (ppx - Xp);
          Zc = iface_z(M, Xc, ifend);
          if (seqnum == 1 && near_src(Xc, Zc)) { Xc = R.sx; Zc = R.sz; }
          finish(n);
          return;   // the reference leaves the exit point unset on this branch
        }
      }
    }
    bool exit_ploop = false, cycle_ploop = false;
    {
      const double zi = iface_z(M, ppx, iftop);
      if (ppz <= zi) {
        if (iftop == ifend) {
          if (refraction) {
            if (refracts(ppx, zi, g0x, g0z)) {
              exit_ploop = true;
            } else {
              Xc = ppx; Zc = zi;
              rs.headwave = true; R.headwave = true;
              if (seqnum == 1 && near_src(Xc, Zc)) { Xc = R.sx; Zc = R.sz; finish(n); return; }
              cycle_ploop = true;
            }
          } else {
            exit_ploop = true;
          }
        } else if (n == 2 && on_top && rs.istart && rs.istart == iftop) {
        } else {
          Xc = ppx; Zc = zi;
          rs.diffracted = true; R.diffracted = true;
          if (seqnum == 1 && near_src(Xc, Zc)) { Xc = R.sx; Zc = R.sz; finish(n); return; }
          cycle_ploop = true;
        }
      }
    }
    if (exit_ploop) break;
    if (cycle_ploop) continue;
    {
      const double zi = iface_z(M, ppx, ifbot);
      if (ppz >= zi) {
        if (ifbot == ifend) {
          if (refraction) {
            if (R.raypath == 4 && seqnum == 2) {
              exit_ploop = true;
            } else if (refracts(ppx, zi, g0x, g0z)) {
              exit_ploop = true;
            } else {
              Xc = ppx; Zc = zi;
              rs.headwave = true; R.headwave = true;
              if (seqnum == 1 && near_src(Xc, Zc)) { Xc = R.sx; Zc = R.sz; finish(n); return; }
              cycle_ploop = true;
            }
          } else {
            exit_ploop = true;
          }
        } else if (n == 2 && on_bot && rs.istart && rs.istart == ifbot) {
        } else {
          Xc = ppx; Zc = zi;
          rs.diffracted = true; R.diffracted = true;
          if (seqnum == 1 && near_src(Xc, Zc)) { Xc = R.sx; Zc = R.sz; finish(n); return; }
          cycle_ploop = true;
        }
      }
    }
    if (exit_ploop) break;
    if (cycle_ploop) continue;
    int iter = 1;
    for (;;) {  // itloop: Heun step with step halving
      ppx = Xp - dl * g0x;
      ppz = Zp - dl * g0z;
      grad_at(M, reg, tf.G, ppx, ppz, g1x, g1z);
      Xc = Xp - dl * (g0x + g1x) * 0.5;
      Zc = Zp - dl * (g0z + g1z) * 0.5;
      {
        const double zi = iface_z(M, Xc, iftop);
        if (Zc <= zi) {
          if (iftop == ifend) {
            if (refraction) {
              if (refracts(Xc, zi, g0x, g0z)) {
                ppx = Xc; ppz = Zc;
                exit_ploop = true;
              } else {
                Zc = zi;
                rs.headwave = true; R.headwave = true;
                cycle_ploop = true;
              }
            } else {
              ppx = Xc; ppz = Zc;
              exit_ploop = true;
            }
          } else if (n == 2 && on_top && rs.istart && rs.istart == iftop) {
          } else {
            Zc = zi;
            rs.diffracted = true; R.diffracted = true;
            cycle_ploop = true;
          }
        }
      }
      if (exit_ploop || cycle_ploop) break;
      {
        const double zi = iface_z(M, Xc, ifbot);
        if (Zc >= zi) {
          if (ifbot == ifend) {
            if (refraction) {
              if (R.raypath == 4 && seqnum == 2) {
                ppx = Xc; ppz = Zc;
                exit_ploop = true;
              } else if (refracts(Xc, zi, g0x, g0z)) {
                ppx = Xc; ppz = Zc;
                exit_ploop = true;
              } else {
                Zc = zi;
                rs.headwave = true; R.headwave = true;
                cycle_ploop = true;
              }
            } else {
              ppx = Xc; ppz = Zc;
              exit_ploop = true;
            }
          } else if (n == 2 && on_bot && rs.istart && rs.istart == ifbot) {
          } else {
            Zc = zi;
            rs.diffracted = true; R.diffracted = true;
            cycle_ploop = true;
          }
        }
      }
      if (exit_ploop || cycle_ploop) break;
      const double ex = Xc - ppx, ez = Zc - ppz;
      if (sqrt(ex * ex + ez * ez) < p_tol) break;
      ++iter;
      if (iter > 10) { R.valid = false; return; }
      dl = 0.5 * dl;
    }
    if (exit_ploop) break;
    if (cycle_ploop) continue;
    if (seqnum == 1 && near_src(Xc, Zc)) { Xc = R.sx; Zc = R.sz; finish(n); return; }
  }
  if (seqnum == 1) { R.valid = false; return; }
  if (ifend) {
    if (!crossing(M, Xp, Zp, Xc, Zc, ppx, ppz, ifend, g0x, g0z, dl)) {
      R.valid = false;
      return;
    }
  }
  x_out = Xc;
  z_out = Zc;
  finish(n);
}

// inversion2d.f90:6344-6438: best seafloor entry point of an in-water pick.
__device__ void optimal_entry(const TrModel& M, const TrRegion& r, const double* T,
                              const double* sft, double rx, double rz, double& ex, double& ez,
                              double& wt) {
  const int nsf = M.nx;
  const double* sz = M.ifz[2];
  const double* sxp = M.xpos;
  const double dxs = sxp[1] - sxp[0];
  auto sf_z = [&](double px) {
    if (nsf < 2) return sz[0];
    const int ixx = (int)floor((px - sxp[0]) / dxs) + 1;
    if (ixx < 1) return sz[0];
    if (ixx >= nsf) return sz[nsf - 1];
    const double w = clamp01((px - sxp[ixx - 1]) / dxs);
    return (1.0 - w) * sz[ixx - 1] + w * sz[ixx];
  };
  double tbest = kHugeT;
  const double z0 = sf_z(rx);
  double xb = rx, zb = z0, wb = (z0 - rz) / M.vwater;
  // the field's time at each seafloor node is the same for every pick of the
  // source: precomputed once per field (sft), else interpolated here
  for (int i = 0; i < nsf; ++i) {
    const double xt = sxp[i], zs = sz[i];
    const double tf = sft ? sft[i] : time_at(M, r, T, xt, zs);
    if (tf > kHugeT * 0.5) continue;
    const double tw = sqrt((xt - rx) * (xt - rx) + (zs - rz) * (zs - rz)) / M.vwater;
    if (tf + tw < tbest) { tbest = tf + tw; xb = xt; zb = zs; wb = tw; }
  }
  if (xb <= sxp[0] || xb >= sxp[nsf - 1]) { ex = xb; ez = zb; wt = wb; return; }
  double xl = 0, xr = 0;
  for (int i = 0; i < nsf - 1; ++i)
    if (xb >= sxp[i] && xb <= sxp[i + 1]) { xl = sxp[i]; xr = sxp[i + 1]; break; }
  const int nref = 10;
  const double dr = (xr - xl) / double(nref);
  for (int k = 1; k <= nref - 1; ++k) {
    const double xt = xl + double(k) * dr;
    const double zs = sf_z(xt);
    const double tf = time_at(M, r, T, xt, zs);
    if (tf > kHugeT * 0.5) continue;
    const double tw = sqrt((xt - rx) * (xt - rx) + (zs - rz) * (zs - rz)) / M.vwater;
    if (tf + tw < tbest) { tbest = tf + tw; xb = xt; zb = zs; wb = tw; }
  }
  ex = xb; ez = zb; wt = wb;
}

// inversion2d.f90:4675-4759: interface-depth entries of a reflection or
// transmission at the inverted interface.
__device__ void iface_entries(RayState& R) {
  const TrModel& M = *R.M;
  if (M.iface_inv <= 0) return;
  const int np = M.n_inv;
  bool done_rec = false, do_if = false;
  int prev = 0;
  for (int k = R.nsec; k >= 1; --k) {
    const Section& rs = R.sec[k];
    if (rs.npts <= 2) continue;
    if (!done_rec) { prev = k; done_rec = true; }
    else do_if = true;
    if (do_if) {
      if (rs.istart == 0) { prev = k; continue; }
      if (rs.istart == M.iface_inv) {
        const double px = rs.x1, pz = rs.z1;
        double gx, gz;
        grad_at(M, M.reg[rs.reg], R.F[rs.tf].G, px, pz, gx, gz);
        const double vin = vel_at(M, px, pz);
        const double nl = sqrt(gx * gx + gz * gz);
        if (nl > 0.0) { gx = gx / (vin * nl); gz = gz / (vin * nl); }
        double nx, nz;
        iface_normal(M, px, rs.istart, nx, nz);
        const double gin = gx * nx + gz * nz;
        double gout;
        if (rs.reg == R.sec[prev].reg) {
          gout = -gin;
        } else {
          const double tx = gx - gin * nx, tz = gz - gin * nz;
          const double par = sqrt(tx * tx + tz * tz);
          const double vout = vel_at(M, px, pz);
          double det = 1.0 / (vout * vout) - par * par;
          if (det < 0.0) det = 0.0;
          gout = copysign(sqrt(det), gin);
        }
        const double geo = (gin - gout) * nz;
        const double dxi = M.xpos[1] - M.xpos[0];
        int ivx = (int)floor((px - M.xpos[0]) / dxi) + 1;
        ivx = max(1, min(M.nx - 1, ivx));
        const double wx = clamp01((px - M.xpos[ivx - 1]) / dxi);
        int idx = M.iface_start + ivx - 1;
        if (idx >= 1 && idx + 1 <= np) add_one(*R.sink, idx + 1, (1.0 - wx) * geo);
        idx = M.iface_start + ivx;
        if (idx >= 1 && idx + 1 <= np) add_one(*R.sink, idx + 1, wx * geo);
      }
    }
    prev = k;
  }
}

__device__ double seafloor_z(const TrModel& M, double px) {
  const int n = M.nx;
  const double* z = M.ifz[2];
  if (n < 2) return z[0];
  const double dx = M.xpos[1] - M.xpos[0];
  const int ixx = (int)floor((px - M.xpos[0]) / dx) + 1;
  if (ixx < 1) return z[0];
  if (ixx >= n) return z[n - 1];
  const double w = clamp01((px - M.xpos[ixx - 1]) / dx);
  return (1.0 - w) * z[ixx - 1] + w * z[ixx];
}

__global__ void __launch_bounds__(128) k_trace(const TrModel* Mp, const TrField* fields,
                                               const double* src_x, const double* src_z,
                                               const TrPick* picks, int npick, double* t_calc,
                                               int* valid, unsigned* cnt,
                                               const unsigned long long* off,
                                               unsigned long long* keys, double* vals,
                                               double* entry) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npick) return;
  const TrModel& M = *Mp;
  const TrPick pk = picks[p];
  if (keys && !valid[p]) return;   // second pass: rows of valid picks only
  RayState R;
  R.M = Mp;
  R.F = fields + (size_t)pk.src * 13;
  R.sx = src_x[pk.src];
  R.sz = src_z[pk.src];
  R.raypath = pk.phase;
  R.valid = true;
  R.headwave = false;
  R.diffracted = false;
  Sink sk;
  sk.keys = keys;
  sk.vals = vals;
  sk.base = keys ? off[p] : 0;
  sk.n = 0;
  sk.row = (unsigned long long)p << 32;
  sk.npend = 0;
  R.sink = &sk;
  const int ns = c_ntf[pk.phase];
  R.nsec = ns;
  bool ok = ns > 0;
  for (int n = ns; n >= 1 && ok; --n) {
    Section& rs = R.sec[n];
    rs.tf = c_tfs[pk.phase][n];
    rs.reg = c_tfreg[rs.tf];
    rs.istart = (n < ns) ? c_seq[pk.phase][2 * n] : 0;
    rs.iend = (n > 1) ? c_seq[pk.phase][2 * n - 1] : 0;
    rs.npts = 0;
    if (!R.F[rs.tf].T) ok = false;   // field not solved
  }
  double tr = kHugeT;
  double ent_x = pk.rx, ent_z = pk.rz, ent_w = 0.0;   // the ray's receiver end, water time
  if (ok) {
    // invert2d_main.f90:517-537: a receiver above the seafloor is in water
    const double zsf = seafloor_z(M, pk.rx);
    const bool in_water = pk.rz < zsf;
    double recx = pk.rx, recz = in_water ? zsf : pk.rz, wt = 0.0;
    const int last_tf = R.sec[ns].tf;
    const TrRegion& lr = M.reg[c_tfreg[last_tf]];
    if (in_water) {
      if (pk.phase == 4 || pk.phase == 5) {
        recx = pk.rx;
        recz = pk.rz;
      } else {
        optimal_entry(M, lr, R.F[last_tf].T, R.F[last_tf].sft, pk.rx, pk.rz, recx, recz, wt);
      }
    }
    ent_x = recx;
    ent_z = recz;
    ent_w = wt;
    // trace_ray_from_receiver2d
    tr = time_at(M, lr, R.F[last_tf].T, recx, recz);
    double rgx, rgz;
    grad_at(M, lr, R.F[last_tf].G, recx, recz, rgx, rgz);
    if (tr > 1.0e10) R.valid = false;
    if (rgx == 0.0 && rgz == 0.0) R.valid = false;
    double x_in = recx, z_in = recz, x_out = 0, z_out = 0;
    for (int n = ns; n >= 1 && R.valid; --n) {
      trace_section(R, n, x_in, z_in, x_out, z_out);
      if (!R.valid) break;
      if (n > 1) { x_in = x_out; z_in = z_out; }
    }
    if (R.valid) tr = tr + wt;
    ok = R.valid;
  }
  if (ok) {
    sink_flush(sk);
    iface_entries(R);
    sink_flush(sk);
  }
  if (!keys) {
    t_calc[p] = tr;
    valid[p] = ok ? 1 : 0;
    cnt[p] = ok ? sk.n : 0u;
    if (entry) {
      entry[3 * (size_t)p] = ent_x;
      entry[3 * (size_t)p + 1] = ent_z;
      entry[3 * (size_t)p + 2] = ent_w;
    }
  }
}

__global__ void k_sf_times(const TrModel* Mp, const SfJob* jobs, int njobs, int nx) {
  const TrModel& M = *Mp;
  const SfJob J = jobs[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x)
    J.out[i] = time_at(M, M.reg[J.reg], J.T, M.xpos[i], M.ifz[2][i]);
}

// The slots and weights through which time_at(px, pz) reads the field:
// time_at = sum_k w[k] * T[s[k]] (k < the returned count), or 0 nodes where
// it returns huge_time.
__device__ int time_weights(const TrModel& M, const TrRegion& r, const double* T, double px,
                            double pz, int* s, double* w) {
  int ix = (int)floor((px - M.x0) / M.dx) + 1;
  int iz = (int)floor((pz - 0.0) / M.dx) + 1;
  ix = max(1, min(M.nx - 1, ix));
  iz = max(1, min(M.nz - 1, iz));
  const double w1 = clamp01((px - gxc(M, ix)) / M.dx);
  const double w2 = clamp01((pz - gzc(M, iz)) / M.dx);
  auto sn = [&](int a, int b) {
    int q = region_node(M, r, a, b);
    if (q < 0) q = nearby_node(M, r, a, b);
    return q;
  };
  s[0] = sn(ix, iz);
  s[1] = sn(ix + 1, iz);
  s[2] = sn(ix, iz + 1);
  s[3] = sn(ix + 1, iz + 1);
  const double hh = kHugeT * 0.5;
  bool all = true;
  for (int k = 0; k < 4; ++k) all = all && s[k] >= 0 && T[s[k]] < hh;
  if (all) {
    w[0] = (1.0 - w1) * (1.0 - w2);
    w[1] = w1 * (1.0 - w2);
    w[2] = (1.0 - w1) * w2;
    w[3] = w1 * w2;
    return 4;
  }
  s[0] = nearest_node(M, r, px, pz);
  if (s[0] < 0 || !(T[s[0]] < hh)) return 0;
  w[0] = 1.0;
  return 1;
}

// One block per target field (src*13 + tf in tgt), whose picks are
// tpk[tp[k] .. tp[k+1]) in pick order: the threads find the weights of a
// chunk of picks at once, then one thread adds coef[p] times them to d in
// pick order, so the sums do not depend on thread timing.
__global__ void __launch_bounds__(128) k_adj_picks(const TrModel* Mp, const TrField* fields,
                                                   const TrPick* picks, const double* entry,
                                                   const double* coef, const int* tgt,
                                                   const int* tp, const int* tpk,
                                                   double* const* d) {
  const int k = blockIdx.x;
  const TrModel& M = *Mp;
  const int src = tgt[k] / 13, tf = tgt[k] % 13;
  const double* T = fields[(size_t)src * 13 + tf].T;
  const TrRegion& r = M.reg[c_tfreg[tf]];
  double* dk = d[k];
  __shared__ int s_n[128], s_sl[128][4];
  __shared__ double s_w[128][4];
  for (int base = tp[k]; base < tp[k + 1]; base += blockDim.x) {
    const int i = base + threadIdx.x;
    s_n[threadIdx.x] = 0;
    if (i < tp[k + 1]) {
      const int p = tpk[i];
      int sl[4];
      double w[4];
      const int n = time_weights(M, r, T, entry[3 * (size_t)p], entry[3 * (size_t)p + 1], sl, w);
      s_n[threadIdx.x] = n;
      for (int j = 0; j < n; ++j) {
        s_sl[threadIdx.x][j] = sl[j];
        s_w[threadIdx.x][j] = coef[p] * w[j];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int m = min((int)blockDim.x, tp[k + 1] - base);
      for (int t = 0; t < m; ++t)
        for (int j = 0; j < s_n[t]; ++j) dk[s_sl[t][j]] += s_w[t][j];
    }
    __syncthreads();
  }
}

}  // namespace

void tr_adj_picks(const TrModel* m, const TrField* fields, const TrPick* picks,
                  const double* entry, const double* coef, const int* tgt, const int* tp,
                  const int* tpk, double* const* d, int ntgt, cudaStream_t st) {
  if (ntgt <= 0) return;
  k_adj_picks<<<ntgt, 128, 0, st>>>(m, fields, picks, entry, coef, tgt, tp, tpk, d);
}

void tr_sf_times(const TrModel* m, const SfJob* jobs, int njobs, int nx, cudaStream_t st) {
  if (njobs <= 0) return;
  k_sf_times<<<dim3((nx + 127) / 128, njobs), 128, 0, st>>>(m, jobs, njobs, nx);
}

void tr_launch(const TrModel* m, const TrField* fields, const double* src_x, const double* src_z,
               const TrPick* picks, int npick, double* t_calc, int* valid, unsigned* cnt,
               const unsigned long long* off, unsigned long long* keys, double* vals,
               double* entry, cudaStream_t st) {
  k_trace<<<(npick + 127) / 128, 128, 0, st>>>(m, fields, src_x, src_z, picks, npick, t_calc,
                                               valid, cnt, off, keys, vals, entry);
}

}  // namespace fmt2d
