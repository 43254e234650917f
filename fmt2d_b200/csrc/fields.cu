// Stage coupling (source and interface seeding) and field post-processing.
// Coupling arithmetic is FP64 (the time and gradient handed from one stage to
// the next), stored back as the solver's (hi, lo) FP32 pair.
#include "fields.cuh"
#include "model.h"

namespace fmt2d {

namespace {

__device__ __forceinline__ void split_d(double t, float& hi, float& lo) {
  hi = (float)t;
  lo = (float)(t - (double)hi);
}

__device__ __forceinline__ double tdbl(float2 t) {
  return t.x >= kReachedF ? 1.0e20 : (double)t.x + (double)t.y;
}

// A seeded node lowers the key of its tile and of the tiles whose halo holds
// it; k_seed_masks then opens every node of the tiles with a key.
__device__ __forceinline__ void mark_grid(const DevField& F, int col, int brow, float t) {
  const DevRegion& R = F.R;
  const unsigned key = key_of(t);
  const int tx0 = max(0, (col - kHalo) / kTW), tx1 = min(R.tiles_x - 1, (col + kHalo) / kTW);
  const int ty0 = max(0, (brow - kHalo) / kTH), ty1 = min(R.tiles_y - 1, (brow + kHalo) / kTH);
  for (int ty = ty0; ty <= ty1; ++ty)
    for (int tx = tx0; tx <= tx1; ++tx) atomicMin(F.tkey + ty * R.tiles_x + tx, key);
}

__device__ __forceinline__ void mark_iface(const DevField& F, int side, int col, float t) {
  const DevRegion& R = F.R;
  int row = R.izc[side * R.pitch + col] - R.z_lo;
  row = row < 0 ? 0 : (row >= R.H ? R.H - 1 : row);
  mark_grid(F, col, row, t);
}

// rays-free fit of the time gradient at one node (propagate2d.f90:949-1196).
__device__ void fit_grad(const DevRegion& R, const DevRegionX& X, const float2* T, int slot,
                         double& dtdx, double& dtdz) {
  const uint32_t code = R.code[slot];
  const bool iface = (code & kIfaceNode) != 0;
  const int side = iface ? (slot / R.pitch - R.H) : 0;
  const int col = slot % R.pitch;
  const int brow = iface ? -1 : slot / R.pitch;
  const double h = R.dx;
  auto in_reg = [&](int c, int absrow) -> int {
    const int br = absrow - R.z_lo;
    if (c < 0 || c >= R.nx || br < 0 || br >= R.H) return -1;
    const int s = br * R.pitch + c;
    return (R.code[s] & kInRegion) ? s : -1;
  };
  auto tt = [&](int s) { return tdbl(T[s]); };
  double xu, zu;
  if (iface) { xu = X.iface_x[col]; zu = X.iface_z[side * R.pitch + col]; }
  else { xu = R.x0 + col * h; zu = (brow + R.z_lo) * h; }
  // cells around the node
  int ncl = 0, clx[4], clz[4];
  bool any[4];
  if (!iface) {
    for (int c = 0; c < 4; ++c) {
      if (!(code & (1u << (4 + c)))) continue;
      clx[ncl] = col - (c >= 2 ? 1 : 0);
      clz[ncl] = brow + R.z_lo - ((c & 1) ? 1 : 0);
      any[ncl] = (code & (1u << (20 + c))) != 0;
      ++ncl;
    }
  } else {
    const int izc = R.izc[side * R.pitch + col];
    if (izc >= 0) { clx[0] = col; clz[0] = izc; any[0] = (code & (1u << 20)) != 0; ncl = 1; }
  }
  int nirr = 0;
  for (int n = 0; n < ncl; ++n) nirr += any[n] ? 1 : 0;
  if (nirr == 0) {
    if (!iface) {
      const int absr = brow + R.z_lo;
      int m = in_reg(max(0, col - 1), absr), n = in_reg(min(R.nx - 1, col + 1), absr);
      const double xm = R.x0 + max(0, col - 1) * h, xn = R.x0 + min(R.nx - 1, col + 1) * h;
      if (m >= 0 && n >= 0) dtdx = (tt(n) - tt(m)) / (xn - xm);
      else if (m >= 0) dtdx = (tt(slot) - tt(m)) / (xu - xm);
      else if (n >= 0) dtdx = (tt(n) - tt(slot)) / (xn - xu);
      else dtdx = 0.0;
      const int zm = max(0, absr - 1), zn = min(X.nz - 1, absr + 1);
      m = in_reg(col, zm);
      n = in_reg(col, zn);
      if (m >= 0 && n >= 0) dtdz = (tt(n) - tt(m)) / ((zn - zm) * h);
      else if (m >= 0) dtdz = (tt(slot) - tt(m)) / (zu - zm * h);
      else if (n >= 0) dtdz = (tt(n) - tt(slot)) / (zn * h - zu);
      else dtdz = 0.0;
      return;
    }
    if (ncl == 0) { dtdx = 0.0; dtdz = 0.0; return; }
  }
  int ns = 0, store[30];
  double rx[30], rz[30], at[30];
  auto take = [&](int s, double x, double z) {
    if (s == slot || s < 0) return;
    for (int k = 0; k < ns; ++k)
      if (store[k] == s) return;
    if (ns < 30) { store[ns] = s; rx[ns] = x; rz[ns] = z; at[ns] = tt(s); ++ns; }
  };
  for (int n = 0; n < ncl; ++n) {
    if (any[n]) {
      // inodes of the cut cell: the interface node of the cell's column
      const int cx = clx[n];
      for (int sd = 0; sd < 2; ++sd) {
        if (R.izc[sd * R.pitch + cx] != clz[n]) continue;
        const int s = (R.H + sd) * R.pitch + cx;
        // present only when the node lies inside the cell (inode_ok)
        const double zi = X.iface_z[sd * R.pitch + cx];
        if (!(zi >= clz[n] * h && zi <= (clz[n] + 1) * h)) continue;
        take(s, X.iface_x[cx], zi);
      }
    }
    for (int i = 0; i <= 1; ++i)
      for (int j = 0; j <= 1; ++j) {
        const int a = clx[n] + i, b = clz[n] + j;
        const int s = in_reg(a, b);
        if (s >= 0) take(s, R.x0 + a * h, b * h);
      }
  }
  double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0;
  const double tu = tt(slot);
  for (int i = 0; i < ns; ++i) {
    const double ddx = rx[i] - xu, ddz = rz[i] - zu;
    const double dw = 1.0 / (sqrt(ddx * ddx + ddz * ddz) + R.tol);
    a11 += ddx * ddx * dw * dw;
    a12 += ddx * ddz * dw * dw;
    a22 += ddz * ddz * dw * dw;
    b1 += (at[i] - tu) * ddx * dw * dw;
    b2 += (at[i] - tu) * ddz * dw * dw;
  }
  const double det = a11 * a22 - a12 * a12;
  if (fabs(det) < 1.0e-30) { dtdx = 0.0; dtdz = 0.0; return; }
  dtdx = (a22 * b1 - a12 * b2) / det;
  dtdz = (a11 * b2 - a12 * b1) / det;
}

}  // namespace

// Reset a field: every slot unreached, no gradient, no active tile.
__global__ void k_fill(DevField* fields, int nf, size_t max_slots) {
  const int fi = blockIdx.y;
  DevField& F = fields[fi];
  const size_t ns = (size_t)(F.R.H + 2) * F.R.pitch;
  const int nt = F.R.tiles_x * F.R.tiles_y;
  const size_t nw = (size_t)kTileWords * nt;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns || i < nw;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i < ns) {
      reinterpret_cast<float2*>(F.Th)[i] = make_float2(kHugeF, 0.0f);
      reinterpret_cast<float2*>(F.gx)[i] = make_float2(0.0f, 0.0f);
      F.seed[i] = make_float4(kHugeF, 0.0f, 0.0f, 0.0f);
      F.sflag[i] = 0;
    }
    if (i < nw) F.act[i] = 0u;
    if (i < (size_t)nt) { F.tkey[i] = kKeyNone; F.tvis[i] = 0u; }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    F.frozen_slot = -1;
    *F.front = kHugeF;
  }
  (void)max_slots;
}

// Point source at (sx, sz): the four corners of its cell get dist/v and the
// straight-ray gradient; a corner within 0.01*tolerance takes t0 and stays
// fixed (propagate2d.f90:2307-2411).
__global__ void k_init_source(DevField* fields, const DevRegionX* xs, const double* sx,
                              const double* sz, int nf, int nz) {
  const int fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi >= nf) return;
  DevField& F = fields[fi];
  const DevRegion& R = F.R;
  const DevRegionX& X = xs[fi];
  const double h = R.dx;
  int ix0 = (int)floor((sx[fi] - R.x0) / h);
  int iz0 = (int)floor((sz[fi] - 0.0) / h);
  ix0 = max(0, min(R.nx - 2, ix0));
  iz0 = max(0, min(nz - 2, iz0));
  for (int ix = ix0; ix <= ix0 + 1; ++ix)
    for (int iz = iz0; iz <= iz0 + 1; ++iz) {
      const int br = iz - R.z_lo;
      if (br < 0 || br >= R.H) continue;
      const int s = br * R.pitch + ix;
      if (!(R.code[s] & kInRegion)) continue;
      const double ddx = (R.x0 + ix * h) - sx[fi], ddz = iz * h - sz[fi];
      const double dist = sqrt(ddx * ddx + ddz * ddz);
      double v = X.vel64[s];
      if (v < 0.01) v = 0.01;
      float2 t, g;
      if (dist < 0.01 * R.tol) {
        t = make_float2(0.0f, 0.0f);
        g = make_float2(0.0f, 0.0f);
        F.frozen_slot = s;
      } else {
        split_d(dist / v, t.x, t.y);
        g = make_float2((float)(ddx / (dist * v)), (float)(ddz / (dist * v)));
      }
      reinterpret_cast<float2*>(F.Th)[s] = t;
      reinterpret_cast<float2*>(F.gx)[s] = g;
      F.seed[s] = make_float4(t.x, t.y, g.x, g.y);
      F.sflag[s] = 1;
      mark_grid(F, ix, br, t.x);
    }
}

// Interface hand-off of a stage: copy time and gradient from the previous
// field's boundary nodes (transfer_times_to_intersection), optionally rebuild
// the normal slowness on the target side (reflect_gradient_at_interface), seed
// the target region's interface nodes and the grid nodes up to three rows into
// the region, first interface node first (sweep_region_from_interface2d).
__global__ void k_seed_iface(const SeedDesc* descs, int nd, int nz) {
  const SeedDesc& D = descs[blockIdx.y];
  const DevRegion& R = D.dst.R;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R.nx) return;
  const double h = R.dx;
  auto iface_val = [&](int k, double& T, double& gx, double& gz) {
    const int ss = D.src_row * D.src_pitch + k;
    const float2 t = reinterpret_cast<const float2*>(D.src_t)[ss];
    const float2 g = reinterpret_cast<const float2*>(D.src_g)[ss];
    T = tdbl(t);
    gx = g.x;
    gz = g.y;
    if (!D.reflect) return;
    if (T >= 1.0e20 * 0.5) { gx = 0.0; gz = 0.0; return; }
    const double nx_ = D.ifc.nrm_x[k], nz_ = D.ifc.nrm_z[k];
    const double gp = gx * nx_ + gz * nz_;
    const double px = gx - gp * nx_, pz = gz - gp * nz_;
    const int side = D.target_side;
    double v = side > 0 ? D.ifc.vel_bot[k] : D.ifc.vel_top[k];
    if (!(v > 0.01)) v = D.dstx.vel64[(R.H + D.dst_side) * R.pitch + k];
    if (v <= 0.01) { T = 1.0e20; gx = 0.0; gz = 0.0; return; }
    const double pn2 = 1.0 / (v * v) - (px * px + pz * pz);
    if (pn2 < -1.0e-10) { T = 1.0e20; gx = 0.0; gz = 0.0; return; }
    const double pn = sqrt(pn2 < 0.0 ? 0.0 : pn2);
    gx = px + side * pn * nx_;
    gz = pz + side * pn * nz_;
  };
  double T, gx, gz;
  iface_val(c, T, gx, gz);
  {
    const int s = (R.H + D.dst_side) * R.pitch + c;
    float2 t;
    if (T >= 1.0e20 * 0.5) t = make_float2(kHugeF, 0.0f);
    else split_d(T, t.x, t.y);
    reinterpret_cast<float2*>(D.dst.Th)[s] = t;
    reinterpret_cast<float2*>(D.dst.gx)[s] = make_float2((float)gx, (float)gz);
    D.dst.seed[s] = make_float4(t.x, t.y, (float)gx, (float)gz);
    D.dst.sflag[s] = 1;
    mark_iface(D.dst, D.dst_side, c, t.x);
  }
  // grid nodes of column c: the first interface node (c-1, c, c+1) whose
  // three-row box holds a node seeds it
  int done[9], ndone = 0;   // rows of column c seeded so far
  for (int n = c - 1; n <= c + 1; ++n) {
    if (n < 0 || n >= R.nx) continue;
    const int izf = D.ifc.izc[n];
    if (izf < 0) continue;
    int r_a, r_b, st;
    if (D.dst_side == 1) { r_a = izf; r_b = max(0, izf - 2); st = -1; }
    else { r_a = izf + 1; r_b = min(nz - 1, izf + 3); st = 1; }
    double Tn, gxn, gzn;
    iface_val(n, Tn, gxn, gzn);
    const double xm = D.dstx.iface_x[n], zm = D.ifc.z[n];
    for (int r = r_a; st > 0 ? r <= r_b : r >= r_b; r += st) {
      if (r < D.dstx.r0[c] || r > D.dstx.r1[c]) continue;
      bool seen = false;
      for (int q = 0; q < ndone; ++q) seen = seen || (done[q] == r);
      if (seen) continue;
      done[ndone++] = r;
      const int br = r - R.z_lo;
      const int s = br * R.pitch + c;
      const double ddx = (R.x0 + c * h) - xm, ddz = r * h - zm;
      const double dist = sqrt(ddx * ddx + ddz * ddz);
      double v = D.dstx.vel64[s];
      if (v < 0.01) v = 0.01;
      const double tn = Tn + dist / v;
      float2 t;
      if (tn >= 1.0e20 * 0.5) t = make_float2(kHugeF, 0.0f);
      else split_d(tn, t.x, t.y);
      const float2 gs = make_float2((float)(ddx / (dist * v)), (float)(ddz / (dist * v)));
      reinterpret_cast<float2*>(D.dst.Th)[s] = t;
      reinterpret_cast<float2*>(D.dst.gx)[s] = gs;
      D.dst.seed[s] = make_float4(t.x, t.y, gs.x, gs.y);
      D.dst.sflag[s] = 1;
      mark_grid(D.dst, c, br, t.x);
    }
  }
}

// Refit the gradient of suspect nodes (propagate2d.f90:119-123).
__global__ void k_fit_suspect(const DevField* fields, const DevRegionX* xs, float* const* gout,
                              uint8_t* const* susp, int nf) {
  const int fi = blockIdx.y;
  const DevField& F = fields[fi];
  const DevRegion& R = F.R;
  const size_t ns = (size_t)(R.H + 2) * R.pitch;
  const float2* T = reinterpret_cast<const float2*>(F.Th);
  float2* G = reinterpret_cast<float2*>(gout[fi]);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns;
       i += (size_t)gridDim.x * blockDim.x) {
    if (!(R.code[i] & kInRegion) || !susp[fi][i]) continue;
    double gx, gz;
    fit_grad(R, xs[fi], T, (int)i, gx, gz);
    G[i] = make_float2((float)gx, (float)gz);
  }
}

// Top-row gradient fix of the water-layer fields (inversion2d.f90:4264-4292):
// upward = 1 requires dT/dz < 0 at the sea surface, upward = 0 requires > 0.
__global__ void k_water_fix(const DevField* fields, float* const* gout, const int* upward,
                            int nf) {
  const int fi = blockIdx.y;
  const DevField& F = fields[fi];
  const DevRegion& R = F.R;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R.nx || upward[fi] < 0) return;
  const int bt = 0 - R.z_lo, bb = 1 - R.z_lo;
  if (bt < 0 || bb >= R.H) return;
  const int st = bt * R.pitch + c, sb = bb * R.pitch + c;
  if (!(R.code[st] & kInRegion) || !(R.code[sb] & kInRegion)) return;
  float2* G = reinterpret_cast<float2*>(gout[fi]);
  const float gz = G[st].y;
  const bool bad = upward[fi] ? (gz > 0.0f || fabsf(gz) < 0.01f) : (gz < 0.0f || fabsf(gz) < 0.01f);
  if (bad) G[st] = G[sb];
}

// PmP head-wave min-plus sweep along the Moho (inversion2d.f90:4294-4409) for
// one field per thread; node table and velocities are precomputed per model.
__global__ void k_headwave(const DevField* fields, const DevRegionX* xs, float* const* gout,
                           const int* hw_slot, const double* hw_v, double dx_if, int nx,
                           double* scratch, const int* which, int nsel) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsel) return;
  const int fi = which[q];
  const DevField& F = fields[fi];
  const DevRegion& R = F.R;
  float2* T = reinterpret_cast<float2*>(F.Th);
  float2* G = reinterpret_cast<float2*>(gout[fi]);
  double* th = scratch + (size_t)q * nx;
  for (int n = 0; n < nx; ++n) th[n] = hw_slot[n] >= 0 ? tdbl(T[hw_slot[n]]) : 1.0e20;
  for (int n = 1; n < nx; ++n)
    if (hw_v[n] > 0.0) th[n] = fmin(th[n], th[n - 1] + dx_if / hw_v[n]);
  for (int n = nx - 2; n >= 0; --n)
    if (hw_v[n] > 0.0) th[n] = fmin(th[n], th[n + 1] + dx_if / hw_v[n]);
  for (int n = 0; n < nx; ++n) {
    const int s = hw_slot[n];
    if (s < 0) continue;
    if (th[n] < tdbl(T[s]) - 1.0e-10) {
      float2 t;
      split_d(th[n], t.x, t.y);
      T[s] = t;
    }
  }
  for (int n = 0; n < nx; ++n) {
    const int s = hw_slot[n];
    if (s < 0 || T[s].x >= kReachedF) continue;
    if (!(R.code[s] & kIfaceNode)) {
      double gx, gz;
      fit_grad(R, xs[fi], T, s, gx, gz);
      G[s] = make_float2((float)gx, (float)gz);
    } else {
      double dtdx;
      if (n > 0 && n < nx - 1) dtdx = (th[n + 1] - th[n - 1]) / (2.0 * dx_if);
      else if (n == 0 && nx > 1) dtdx = (th[1] - th[0]) / dx_if;
      else if (n == nx - 1 && nx > 1) dtdx = (th[nx - 1] - th[nx - 2]) / dx_if;
      else dtdx = 0.0;
      double dtdz = 0.0;
      if (hw_v[n] > 0.0) {
        const double s2 = 1.0 / (hw_v[n] * hw_v[n]) - dtdx * dtdx;
        dtdz = s2 > 0.0 ? sqrt(s2) : 0.0;
      }
      G[s] = make_float2((float)dtdx, (float)dtdz);
    }
  }
}

// Copy a field out in the reference's region node order, FP64.
__global__ void k_export(const float* t2, const float* g2, const int* slot_of_node, int nnode,
                         double* T, double* gx, double* gz) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nnode; n += gridDim.x * blockDim.x) {
    const int s = slot_of_node[n];
    const float2 t = reinterpret_cast<const float2*>(t2)[s];
    const float2 g = reinterpret_cast<const float2*>(g2)[s];
    if (T) T[n] = tdbl(t);
    if (gx) gx[n] = g.x;
    if (gz) gz[n] = g.y;
  }
}

// Every node of a seeded tile (one with a key after seeding) starts active.
__global__ void k_seed_masks(DevField* fields, int nf) {
  const DevField& F = fields[blockIdx.y];
  const int nt = F.R.tiles_x * F.R.tiles_y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt * kTileWords;
       i += gridDim.x * blockDim.x)
    if (F.tkey[i / kTileWords] != kKeyNone) F.act[i] = 0xffffffffu;
}

}  // namespace fmt2d
