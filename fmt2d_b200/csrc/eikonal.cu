// Tiled fixed-point eikonal solver for one batch of time fields.
//
// The stencil is the reference FMM's (propagate2d.f90:482-946).  Fast marching
// gives every node the minimum of its seed value and of the candidates its
// update events produce, each event using the final (accepted) values of the
// nodes involved:
//   * per regular quadrant the one-sided update from the earlier neighbour and
//     the two-sided update (mixed 1st/2nd order, face-averaged velocity, det
//     clamp, t >= tmax) -- regular_update2d;
//   * per cut cell of the region's own interfaces the point-source update from
//     every accepted member and the planar-front update of every member pair
//     -- time_from_1_node2d / time_from_2_nodes2d.  A member closer than
//     0.01*tolerance hands its time over unchanged ("copy").
// This solver computes the same fixed point T(u) = min(seed(u), best
// candidate of the current neighbour state) without a heap.  Tiles of 32x32
// nodes are staged in shared memory with a 2-node halo.  Inside a tile every
// row keeps a bit mask of nodes whose inputs moved; directional Gauss-Seidel
// sweeps (+z, -z, +x, -x) visit only rows/columns with active nodes and a
// changed node re-activates its stencil neighbours, so a visit ends when no
// node is active.  A tile whose edge values moved re-activates the neighbour
// tile on that side for the next round.
// Values are replaced, not min-ed with their history, because the 2nd-order
// switch depends on neighbour gradients that are only final at the fixed
// point; a copy is only taken from a node whose own value is not a copy,
// which is what the heap's acceptance order guarantees for coincident nodes.
#include "eikonal.cuh"
#include "model.h"

namespace fmt2d {

namespace {

struct TileSmem {
  float Th[kSR * kSP], Tl[kSR * kSP], gx[kSR * kSP], gz[kSR * kSP], vel[kSR * kSP];
  uint8_t fl[kSR * kSP];    // kFlagSeed / kFlagCopy of grid nodes (halo included)
  float iTh[2][kSI], iTl[2][kSI], igx[2][kSI], igz[2][kSI], ivel[2][kSI], idz[2][kSI];
  int izc[2][kSI];
  uint32_t icode[2][kSI];
  uint8_t ifl[2][kSI];
};

// Per-direction neighbour data of a grid node (one of L, R, U, D).
struct Nb {
  bool ok, single_ok, second, t2zero;
  float tau, tau2, hv, inv_d;   // time offsets, h/vbar, 1/(x_u - x_n) along the axis
};

struct Cand {
  float t, gx, gz;
  bool suspect;
};

__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

__device__ __forceinline__ void nb_eval(const TileSmem& S, int sn, int s2, float vu, float tref,
                                        float two_h, float inv_d, int frozen_local, Nb& n) {
  const float vn = S.vel[sn];
  const float thn = S.Th[sn];
  n.ok = vn > 0.0f && thn < kReachedF;
  n.second = false;
  n.t2zero = false;
  n.single_ok = n.ok && sn != frozen_local;
  n.inv_d = inv_d;
  n.tau = 0.0f;
  n.tau2 = 0.0f;
  n.hv = 0.0f;
  if (!n.ok) return;
  n.tau = (thn - tref) + S.Tl[sn];
  n.hv = two_h * rcp(vu + vn);
  const float v2 = S.vel[s2];
  const float th2 = S.Th[s2];
  if (v2 > 0.0f && th2 < kReachedF) {
    const float tau2 = (th2 - tref) + S.Tl[s2];
    if (n.tau >= tau2 && vn * v2 > 0.0f) {
      const float dot = S.gx[sn] * S.gx[s2] + S.gz[sn] * S.gz[s2];
      if (dot * (vn * v2) >= 0.71f) {
        n.second = true;
        n.tau2 = tau2;
        n.t2zero = (th2 == 0.0f && S.Tl[s2] == 0.0f);
      }
    }
  }
}

// One-sided update: closed form of regular_update2d with one accepted neighbour.
__device__ __forceinline__ float single_t(const Nb& n) {
  const float t = n.second ? (2.0f * n.tau - 0.5f * n.tau2 + n.hv) * (1.0f / 1.5f) : n.tau + n.hv;
  return fmaxf(t, n.tau);
}

__device__ __forceinline__ float axis_grad(const Nb& n, float t) {
  if (n.second && !n.t2zero) return 0.5f * (3.0f * t - 4.0f * n.tau + n.tau2) * n.inv_d;
  return (t - n.tau) * n.inv_d;
}

__device__ __forceinline__ void coef(const Nb& n, float& a, float& b, float& c) {
  const float r = rcp(n.hv);
  const float d2 = r * r;
  if (n.second) {
    a += 2.25f * d2;
    b += (-6.0f * n.tau + 1.5f * n.tau2) * d2;
    c += (4.0f * n.tau * n.tau - 2.0f * n.tau * n.tau2 + 0.25f * n.tau2 * n.tau2) * d2;
  } else {
    a += d2;
    b += -2.0f * n.tau * d2;
    c += n.tau * n.tau * d2;
  }
}

__device__ __forceinline__ float pair_t(const Nb& X, const Nb& Z) {
  float a = 0.0f, b = 0.0f, c = 0.0f;
  coef(X, a, b, c);
  coef(Z, a, b, c);
  c -= 1.0f;
  float det = b * b - 4.0f * a * c;
  if (det < 0.0f) det = 0.0f;
  const float t = 0.5f * (-b + sqrtf(det)) * rcp(a);
  return fmaxf(t, fmaxf(X.tau, Z.tau));
}

__device__ __forceinline__ void take(Cand& best, float t, float gx, float gz, bool sus) {
  if (t < best.t) { best.t = t; best.gx = gx; best.gz = gz; best.suspect = sus; }
}

// Candidates of one regular quadrant (update_time2d's four-quadrant loop).
__device__ __forceinline__ void quadrant(const Nb& X, const Nb& Z, Cand& best) {
  if (X.ok && Z.ok) {
    const bool xlow = X.tau <= Z.tau;
    const Nb& lo = xlow ? X : Z;
    if (lo.single_ok) {
      const float t = single_t(lo);
      if (xlow) take(best, t, axis_grad(X, t), 0.0f, true);
      else take(best, t, 0.0f, axis_grad(Z, t), true);
    }
    const float t = pair_t(X, Z);
    take(best, t, axis_grad(X, t), axis_grad(Z, t), false);
  } else if (X.ok) {
    if (X.single_ok) { const float t = single_t(X); take(best, t, axis_grad(X, t), 0.0f, true); }
  } else if (Z.ok) {
    if (Z.single_ok) { const float t = single_t(Z); take(best, t, 0.0f, axis_grad(Z, t), true); }
  }
}

// ---------------------------------------------------------------------------
// Cut-cell updates in FP64 (time_from_1_node2d / time_from_2_nodes2d).
struct Member {
  double x, z, t;   // position relative to the updated node, time
  float gx, gz, v;
  bool single_ok, copied;
};

struct CandD {
  double t;
  float gx, gz;
  bool suspect, copy;
};

__device__ __forceinline__ void takeD(CandD& best, double t, float gx, float gz, bool sus,
                                      bool copy) {
  if (t < best.t) { best.t = t; best.gx = gx; best.gz = gz; best.suspect = sus; best.copy = copy; }
}

__device__ void from_1(const Member& a, float vu, double tol, CandD& best) {
  const double dist = sqrt(a.x * a.x + a.z * a.z);
  if (dist < 0.01 * tol) {
    if (!a.copied) takeD(best, a.t, a.gx, a.gz, false, true);
    return;
  }
  const double t = a.t + dist / (0.5 * ((double)vu + (double)a.v));
  takeD(best, t, (float)(-a.x / (dist * vu)), (float)(-a.z / (dist * vu)), false, false);
}

__device__ void from_2(const Member& A, const Member& B, float vu, double tol, CandD& best) {
  const Member& n1 = (A.t < B.t) ? B : A;   // later (larger time) node first
  const Member& n2 = (A.t < B.t) ? A : B;
  const double r1x = n1.x, r1z = n1.z, r2x = n2.x, r2z = n2.z;
  if (sqrt(r1x * r1x + r1z * r1z) < 0.01 * tol) {
    if (!n1.copied) takeD(best, n1.t, n1.gx, n1.gz, false, true);
    return;
  }
  if (sqrt(r2x * r2x + r2z * r2z) < 0.01 * tol) {
    if (!n2.copied) takeD(best, n2.t, n2.gx, n2.gz, false, true);
    return;
  }
  const double ex = n2.x - n1.x, ez = n2.z - n1.z;
  if (sqrt(ex * ex + ez * ez) < 0.01 * tol) { from_1(n1, vu, tol, best); return; }
  const double v12 = 0.5 * ((double)n1.v + (double)n2.v);
  const double dx = (n1.x - n2.x) / v12, dz = (n1.z - n2.z) / v12;
  const double dd = dx * dx + dz * dz;
  const double px = (n1.t - n2.t) / dd * dx, pz = (n1.t - n2.t) / dd * dz;
  const double qx = -dz, qz = dx;
  const double ae = qx * qx + qz * qz, be = 2.0 * (px * qx + pz * qz);
  const double ce = px * px + pz * pz - 1.0;
  const double det = be * be - 4.0 * ae * ce;
  if (det < 0.0) return;
  const double sq = sqrt(det);
  double n1x = -r1z, n1z = r1x, l = sqrt(n1x * n1x + n1z * n1z);
  n1x /= l; n1z /= l;
  if (n1x * r2x + n1z * r2z < 0.0) { n1x = -n1x; n1z = -n1z; }
  double n2x = -r2z, n2z = r2x;
  l = sqrt(n2x * n2x + n2z * n2z);
  n2x /= l; n2z /= l;
  if (n2x * r1x + n2z * r1z < 0.0) { n2x = -n2x; n2z = -n2z; }
  const double vb = 0.5 * ((double)vu + (double)n1.v);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double uu = 0.5 * (-be + (k == 0 ? sq : -sq)) / ae;
    const double wx = px + uu * qx, wz = pz + uu * qz;
    if (wx * n1x + wz * n1z <= 0.0 && wx * n2x + wz * n2z <= 0.0) {
      const double t = n1.t - (wx * r1x + wz * r1z) / vb;
      if (t >= n1.t) {
        const double wl = sqrt(wx * wx + wz * wz);
        takeD(best, t, (float)(wx / (wl * n1.v)), (float)(wz / (wl * n1.v)), false, false);
      }
    }
  }
}

__device__ void cell_generic(const Member* mem, int nm, float vu, double tol, CandD& best) {
  for (int a = 0; a < nm; ++a)
    if (mem[a].single_ok) from_1(mem[a], vu, tol, best);
  for (int a = 0; a < nm; ++a)
    for (int b = a + 1; b < nm; ++b) from_2(mem[a], mem[b], vu, tol, best);
}

struct TileCtx {
  const DevField* F;
  int c0, r0;          // tile origin (column, bbox row)
  int frozen_local;    // smem index of the frozen node, -1 if none here
  double h;
};

__device__ __forceinline__ double tval(const TileSmem& S, int s) {
  return (double)S.Th[s] + (double)S.Tl[s];
}

__device__ __forceinline__ void split(double t, float& hi, float& lo) {
  hi = (float)t;
  lo = (float)(t - (double)hi);
}

// Members of an irregular cell as seen from a grid node at smem (i,j).
__device__ int gather_cell_grid(const TileSmem& S, const TileCtx& C, uint32_t code, int c,
                                int i, int j, Member* mem) {
  const int ci = i - ((c & 1) ? 1 : 0), cj = j - (c >= 2 ? 1 : 0);
  const double h = C.h;
  int nm = 0;
  const int kk = cj;  // interface entry of the cell's column
  const int zrow_u = C.r0 - kHalo + i + C.F->R.z_lo;   // absolute row of the node
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const bool has = side == 0 ? (code & (1u << (12 + c))) : (code & (1u << (16 + c)));
    if (!has) continue;
    if (S.iTh[side][kk] >= kReachedF) continue;
    Member& m = mem[nm++];
    m.x = (double)(kk - j) * h;
    m.z = (double)(S.izc[side][kk] - zrow_u) * h + (double)S.idz[side][kk];
    m.t = (double)S.iTh[side][kk] + (double)S.iTl[side][kk];
    m.gx = S.igx[side][kk];
    m.gz = S.igz[side][kk];
    m.v = S.ivel[side][kk];
    m.single_ok = true;
    m.copied = (S.ifl[side][kk] & kFlagCopy) != 0;
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int ii = ci + b, jj = cj + a;
      if (ii == i && jj == j) continue;
      const int s = ii * kSP + jj;
      if (!(S.vel[s] > 0.0f) || S.Th[s] >= kReachedF) continue;
      Member& m = mem[nm++];
      m.x = (double)(jj - j) * h;
      m.z = (double)(ii - i) * h;
      m.t = tval(S, s);
      m.gx = S.gx[s];
      m.gz = S.gz[s];
      m.v = S.vel[s];
      m.single_ok = (s != C.frozen_local);
      m.copied = (S.fl[s] & kFlagCopy) != 0;
    }
  return nm;
}

// New value of one node.  sig: 0 no significant change, 1 change above
// kLocalDT (re-activates in-tile neighbours), 2 change above kSigDT (also
// propagates to neighbour tiles).  write: the stored value must be replaced.
struct NewV {
  int sig;
  bool write;
  float th, tl, gx, gz;
  bool suspect, copy;
};

// Seed of a node: (time, gradient) it was initialised with, huge if none.
__device__ __forceinline__ void seed_of(const DevField& F, bool flagged, int slot, double& t,
                                        float& gx, float& gz) {
  if (!flagged) { t = 1.0e30; gx = 0.0f; gz = 0.0f; return; }
  const float4 s = F.seed[slot];
  t = s.x >= kReachedF ? 1.0e30 : (double)s.x + (double)s.y;
  gx = s.z;
  gz = s.w;
}

// New value = min(seed, best candidate), classified against the current one.
__device__ __forceinline__ NewV finish(double cand, float cgx, float cgz, bool sus, bool copy,
                                       double seed, float sgx, float sgz, double cur,
                                       bool cur_copy) {
  NewV out{0, false, kHugeF, 0.0f, 0.0f, 0.0f, false, false};
  double t = cand;
  float gx = cgx, gz = cgz;
  bool su = sus, cp = copy;
  if (seed <= cand) { t = seed; gx = sgx; gz = sgz; su = false; cp = false; }
  if (!(t < 1.0e29)) {
    // nothing reaches the node (any more)
    if (cur < 1.0e19) { out.write = true; out.sig = 2; }
    return out;
  }
  split(t, out.th, out.tl);
  out.gx = gx;
  out.gz = gz;
  out.suspect = su;
  out.copy = cp;
  const double ad = fabs(t - cur);
  out.write = ad > 1.0e-13 * (1.0 + fabs(cur)) || cp != cur_copy || cur >= 1.0e19;
  out.sig = (ad > (double)kSigDT || cur >= 1.0e19) ? 2 : (ad > kLocalDT ? 1 : 0);
  return out;
}

// Update of a grid node at smem (i,j); reads shared memory only (plus the
// seed of a seeded node).
__device__ NewV update_grid(const TileSmem& S, const TileCtx& C, int i, int j, uint32_t code,
                            int slot) {
  const NewV none{0, false, kHugeF, 0.0f, 0.0f, 0.0f, false, false};
  const int s = i * kSP + j;
  if (!(code & kUpdatable) || s == C.frozen_local) return none;
  const float vu = S.vel[s];
  const float h = (float)C.h;
  float tref = kHugeF;
  tref = fminf(tref, S.vel[s - 1] > 0.0f ? S.Th[s - 1] : kHugeF);
  tref = fminf(tref, S.vel[s + 1] > 0.0f ? S.Th[s + 1] : kHugeF);
  tref = fminf(tref, S.vel[s - kSP] > 0.0f ? S.Th[s - kSP] : kHugeF);
  tref = fminf(tref, S.vel[s + kSP] > 0.0f ? S.Th[s + kSP] : kHugeF);
  const bool any_irr = (code & 0xF00u) != 0;
  double seed;
  float sgx, sgz;
  seed_of(*C.F, (S.fl[s] & kFlagSeed) != 0, slot, seed, sgx, sgz);
  const double cur = tval(S, s);
  const bool cur_copy = (S.fl[s] & kFlagCopy) != 0;
  if (tref >= kReachedF && !any_irr)
    return finish(1.0e30, 0.0f, 0.0f, false, false, seed, sgx, sgz, cur, cur_copy);
  if (tref >= kReachedF) tref = 0.0f;
  const float two_h = 2.0f * h, ih = 1.0f / h;
  Nb L, R, U, D;
  nb_eval(S, s - 1, s - 2, vu, tref, two_h, +ih, C.frozen_local, L);
  nb_eval(S, s + 1, s + 2, vu, tref, two_h, -ih, C.frozen_local, R);
  nb_eval(S, s - kSP, s - 2 * kSP, vu, tref, two_h, +ih, C.frozen_local, U);
  nb_eval(S, s + kSP, s + 2 * kSP, vu, tref, two_h, -ih, C.frozen_local, D);
  // quadrants in update_time2d order (i,j) = (-1,-1),(+1,-1),(-1,+1),(+1,+1):
  // cells 3 (L,U), 1 (R,U), 2 (L,D), 0 (R,D)
  if (!any_irr) {
    Cand best{kHugeF, 0.0f, 0.0f, false};
    if (code & (1u << 7)) quadrant(L, U, best);
    if (code & (1u << 5)) quadrant(R, U, best);
    if (code & (1u << 6)) quadrant(L, D, best);
    if (code & (1u << 4)) quadrant(R, D, best);
    const double cand = best.t < kHugeF ? (double)tref + (double)best.t : 1.0e30;
    return finish(cand, best.gx, best.gz, best.suspect, false, seed, sgx, sgz, cur, cur_copy);
  }
  // next to a cut cell of the region's own interfaces: FP64 for those cells
  CandD bd{1.0e30, 0.0f, 0.0f, false, false};
  const int order[4] = {3, 1, 2, 0};
  for (int q = 0; q < 4; ++q) {
    const int c = order[q];
    if (!(code & (1u << (4 + c)))) continue;
    if (code & (1u << (8 + c))) {
      Member mem[6];
      const int nm = gather_cell_grid(S, C, code, c, i, j, mem);
      cell_generic(mem, nm, vu, C.F->R.tol, bd);
    } else {
      Cand b1{kHugeF, 0.0f, 0.0f, false};
      quadrant((c >= 2) ? L : R, (c & 1) ? U : D, b1);
      if (b1.t < kHugeF) takeD(bd, (double)tref + (double)b1.t, b1.gx, b1.gz, b1.suspect, false);
    }
  }
  return finish(bd.t, bd.gx, bd.gz, bd.suspect, bd.copy, seed, sgx, sgz, cur, cur_copy);
}

// Update of an interface node (side, smem interface entry k) owned by the tile.
__device__ NewV update_iface(const TileSmem& S, const TileCtx& C, int side, int k, int slot) {
  const NewV none{0, false, kHugeF, 0.0f, 0.0f, 0.0f, false, false};
  const uint32_t code = S.icode[side][k];
  if (!(code & kUpdatable)) return none;
  const int izc = S.izc[side][k];
  const double h = C.h;
  const int ci = izc - C.F->R.z_lo - C.r0 + kHalo;   // smem row of the cell's top
  const int cj = k;                                   // smem column of the cell's left
  Member mem[6];
  int nm = 0;
  const double zu = (double)S.idz[side][k];           // node depth relative to z(izc)
#pragma unroll
  for (int o = 0; o < 2; ++o) {
    if (o == side) continue;   // the node itself is the cell's inode on its side
    const bool has = o == 0 ? (code & (1u << 12)) : (code & (1u << 16));
    if (!has || S.iTh[o][k] >= kReachedF) continue;
    Member& m = mem[nm++];
    m.x = 0.0;
    m.z = (double)(S.izc[o][k] - izc) * h + (double)S.idz[o][k] - zu;
    m.t = (double)S.iTh[o][k] + (double)S.iTl[o][k];
    m.gx = S.igx[o][k];
    m.gz = S.igz[o][k];
    m.v = S.ivel[o][k];
    m.single_ok = true;
    m.copied = (S.ifl[o][k] & kFlagCopy) != 0;
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int ii = ci + b, jj = cj + a;
      if (ii < 0 || ii >= kSR || jj < 0 || jj >= kSP - 1) continue;
      const int s = ii * kSP + jj;
      if (!(S.vel[s] > 0.0f) || S.Th[s] >= kReachedF) continue;
      Member& m = mem[nm++];
      m.x = (double)a * h;
      m.z = (double)b * h - zu;
      m.t = tval(S, s);
      m.gx = S.gx[s];
      m.gz = S.gz[s];
      m.v = S.vel[s];
      m.single_ok = (s != C.frozen_local);
      m.copied = (S.fl[s] & kFlagCopy) != 0;
    }
  CandD bd{1.0e30, 0.0f, 0.0f, false, false};
  if (nm > 0) cell_generic(mem, nm, S.ivel[side][k], C.F->R.tol, bd);
  double seed;
  float sgx, sgz;
  seed_of(*C.F, (S.ifl[side][k] & kFlagSeed) != 0, slot, seed, sgx, sgz);
  const double cur = (double)S.iTh[side][k] + (double)S.iTl[side][k];
  return finish(bd.t, bd.gx, bd.gz, false, bd.copy, seed, sgx, sgz, cur,
                (S.ifl[side][k] & kFlagCopy) != 0);
}

__device__ __forceinline__ void write_node(TileSmem& S, int s, const NewV& nv) {
  S.Th[s] = nv.th; S.Tl[s] = nv.tl; S.gx[s] = nv.gx; S.gz[s] = nv.gz;
  S.fl[s] = (uint8_t)((S.fl[s] & kFlagSeed) | (nv.copy ? kFlagCopy : 0));
}

__device__ __forceinline__ int find_field(const DevField* fields, int nf, int b) {
  int lo = 0, hi = nf - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (fields[mid].tile_base <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void activate(const DevField& F, int parity_next, int tx, int ty,
                                         unsigned why, unsigned* n_next) {
  const DevRegion& R = F.R;
  if (tx < 0 || ty < 0 || tx >= R.tiles_x || ty >= R.tiles_y) return;
  const int nt = R.tiles_x * R.tiles_y;
  unsigned* a = F.act + (size_t)parity_next * nt + (size_t)ty * R.tiles_x + tx;
  if (atomicOr(a, why) == 0u) atomicAdd(n_next, 1u);
}

// Stage a tile plus its 2-node halo and the interface rows of its columns
// (plus halo) into shared memory.
__device__ void load_tile(TileSmem& S, TileCtx& C, const DevField& F, int lane) {
  const DevRegion& R = F.R;
  for (int e = lane; e < kSR * (kSP - 1); e += 32) {
    const int i = e / (kSP - 1), j = e % (kSP - 1);
    const int row = C.r0 - kHalo + i, col = C.c0 - kHalo + j;
    const int s = i * kSP + j;
    if (row >= 0 && row < R.H && col >= 0 && col < R.nx) {
      const int slot = row * R.pitch + col;
      const float2 tt = reinterpret_cast<const float2*>(F.Th)[slot];
      const float2 gg = reinterpret_cast<const float2*>(F.gx)[slot];
      S.Th[s] = tt.x; S.Tl[s] = tt.y; S.gx[s] = gg.x; S.gz[s] = gg.y;
      S.vel[s] = R.vel[slot];
      S.fl[s] = F.sflag[slot];
      if (slot == F.frozen_slot) C.frozen_local = s;
    } else {
      S.Th[s] = kHugeF; S.Tl[s] = 0.0f; S.gx[s] = 0.0f; S.gz[s] = 0.0f; S.vel[s] = 0.0f;
      S.fl[s] = 0;
    }
  }
  for (int e = lane; e < 2 * kSI; e += 32) {
    const int side = e / kSI, k = e % kSI;
    const int col = C.c0 - kHalo + k;
    if (col >= 0 && col < R.nx) {
      const int slot = (R.H + side) * R.pitch + col;
      const float2 tt = reinterpret_cast<const float2*>(F.Th)[slot];
      const float2 gg = reinterpret_cast<const float2*>(F.gx)[slot];
      S.iTh[side][k] = tt.x; S.iTl[side][k] = tt.y; S.igx[side][k] = gg.x; S.igz[side][k] = gg.y;
      S.ivel[side][k] = R.vel[slot];
      S.idz[side][k] = R.iface_dz[side * R.pitch + col];
      S.izc[side][k] = R.izc[side * R.pitch + col];
      S.icode[side][k] = R.code[slot];
      S.ifl[side][k] = F.sflag[slot];
    } else {
      S.iTh[side][k] = kHugeF; S.iTl[side][k] = 0.0f; S.igx[side][k] = 0.0f;
      S.igz[side][k] = 0.0f; S.ivel[side][k] = 0.0f; S.idz[side][k] = 0.0f;
      S.izc[side][k] = -1; S.icode[side][k] = 0u; S.ifl[side][k] = 0;
    }
  }
  int fl = C.frozen_local;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) fl = max(fl, __shfl_xor_sync(0xffffffffu, fl, o));
  C.frozen_local = fl;
  __syncwarp();
}

// Interface nodes owned by the tile: column in the tile and cut-cell row
// (clamped into the band) in the tile's rows.
__device__ void owned_ifaces(const TileSmem& S, const TileCtx& C, const DevField& F, int lane,
                             unsigned* own) {
  const DevRegion& R = F.R;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int k = lane + kHalo;
    const int col = C.c0 + lane;
    int row = S.izc[side][k] - R.z_lo;
    row = row < 0 ? 0 : (row >= R.H ? R.H - 1 : row);
    const bool o = col < R.nx && (S.icode[side][k] & kUpdatable) && row >= C.r0 &&
                   row < C.r0 + kTH;
    own[side] = __ballot_sync(0xffffffffu, o);
  }
}

// Row neighbours (distance 1 and 2) of the columns in m, m itself excluded.
__device__ __forceinline__ unsigned nb_x(unsigned m) {
  return (m << 1) | (m >> 1) | (m << 2) | (m >> 2);
}

}  // namespace

// One round over the active tiles of every field in the batch.
__global__ void __launch_bounds__(32, 4) eik_round(const DevField* __restrict__ fields, int nf,
                                                int parity, unsigned* n_next, int max_passes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem& S = *reinterpret_cast<TileSmem*>(smem_raw);
  const int b = blockIdx.x;
  const int fi = find_field(fields, nf, b);
  const DevField& F = fields[fi];
  const DevRegion& R = F.R;
  const int t = b - F.tile_base;
  const int nt = R.tiles_x * R.tiles_y;
  if (t >= nt) return;
  unsigned* my = F.act + (size_t)parity * nt + t;
  const unsigned why = *my;
  if (why == 0u) return;
  const int lane = threadIdx.x;
  const int tx = t % R.tiles_x, ty = t / R.tiles_x;
  TileCtx C;
  C.F = &F;
  C.c0 = tx * kTW;
  C.r0 = ty * kTH;
  C.h = R.dx;
  C.frozen_local = -1;
  __syncwarp();
  if (lane == 0) *my = 0u;
  load_tile(S, C, F, lane);
  unsigned own[2];
  owned_ifaces(S, C, F, lane, own);
  const int nrows = min(kTH, R.H - C.r0);     // rows of the tile inside the band
  const unsigned cols = (C.c0 + kTW <= R.nx) ? 0xffffffffu : ((1u << (R.nx - C.c0)) - 1u);
  // initial active set: everything, or the band next to the edges that moved
  unsigned act = 0u;   // lane r: active columns of row r
  if (lane < nrows) {
    if (why & kActAll) act = cols;
    if ((why & kActTop) && lane < 2) act = cols;
    if ((why & kActBot) && lane >= kTH - 2) act = cols;
    if (why & kActLeft) act |= 0x3u;
    if (why & kActRight) act |= 0xC0000000u;
    if ((why & kActTL) && lane < 2) act |= 0x3u;
    if ((why & kActTR) && lane < 2) act |= 0xC0000000u;
    if ((why & kActBL) && lane >= kTH - 2) act |= 0x3u;
    if ((why & kActBR) && lane >= kTH - 2) act |= 0xC0000000u;
    act &= cols;
  }
  unsigned iact[2] = {own[0], own[1]};
  unsigned rowsig = 0u;       // lane r: columns of row r that changed significantly
  unsigned isig[2] = {0u, 0u};
  bool converged = false;
  for (int pass = 0; pass < max_passes; ++pass) {
    const unsigned rows_act = __ballot_sync(0xffffffffu, act != 0u);
    if (rows_act == 0u && iact[0] == 0u && iact[1] == 0u) { converged = true; break; }
    const int dir = pass & 3;
    if (dir < 2) {
      // z sweep: lane = column, rows in sweep order
      unsigned todo = rows_act;
      while (todo) {
        const int r = dir == 0 ? __ffs(todo) - 1 : 31 - __clz(todo);
        const int row = C.r0 + r;
        const int slot = row * R.pitch + C.c0 + lane;
        for (int rep = 0; rep < 3; ++rep) {
          const unsigned m = __shfl_sync(0xffffffffu, act, r);
          if (!m) break;
          NewV nv{0, false, 0.0f, 0.0f, 0.0f, 0.0f, false, false};
          if ((m >> lane) & 1u) {
            const uint32_t code = R.code[slot];
            if (code & kInRegion) nv = update_grid(S, C, r + kHalo, lane + kHalo, code, slot);
          }
          __syncwarp();
          if (nv.write) write_node(S, (r + kHalo) * kSP + lane + kHalo, nv);
          __syncwarp();
          const unsigned chg = __ballot_sync(0xffffffffu, nv.sig >= 1);
          const unsigned sig = __ballot_sync(0xffffffffu, nv.sig == 2);
          const int d = lane - r;
          if (d == 0) { act = (act & ~m) | (nb_x(chg) & cols); rowsig |= sig; }
          else if (d == 1 || d == -1) act |= (chg | (chg << 1) | (chg >> 1)) & cols;
          else if (d == 2 || d == -2) act |= chg & cols;
          if (lane >= nrows) act = 0u;
          if (chg) { iact[0] |= (chg | (chg >> 1)) & own[0]; iact[1] |= (chg | (chg >> 1)) & own[1]; }
        }
        const unsigned nxt = __ballot_sync(0xffffffffu, act != 0u);
        // continue the sweep past r only (rows behind it wait for the next pass)
        if (dir == 0) todo = r >= 31 ? 0u : (nxt & ~((2u << r) - 1u));
        else todo = r == 0 ? 0u : (nxt & ((1u << r) - 1u));
      }
    } else {
      // x sweep: lane = row, columns in sweep order
      unsigned todo = __reduce_or_sync(0xffffffffu, act);
      while (todo) {
        const int c = dir == 2 ? __ffs(todo) - 1 : 31 - __clz(todo);
        const int row = C.r0 + lane;
        const int slot = row * R.pitch + C.c0 + c;
        for (int rep = 0; rep < 3; ++rep) {
          const bool mine = (act >> c) & 1u;
          if (!__any_sync(0xffffffffu, mine)) break;
          NewV nv{0, false, 0.0f, 0.0f, 0.0f, 0.0f, false, false};
          if (mine) {
            const uint32_t code = R.code[slot];
            if (code & kInRegion) nv = update_grid(S, C, lane + kHalo, c + kHalo, code, slot);
          }
          __syncwarp();
          if (nv.write) write_node(S, (lane + kHalo) * kSP + c + kHalo, nv);
          __syncwarp();
          const bool ch = nv.sig >= 1;
          if (mine) act &= ~(1u << c);
          const unsigned bit = 1u << c;
          if (ch) act |= nb_x(bit) & cols;
          if (nv.sig == 2) rowsig |= bit;
          const bool u1 = __shfl_up_sync(0xffffffffu, ch, 1) && lane >= 1;
          const bool u2 = __shfl_up_sync(0xffffffffu, ch, 2) && lane >= 2;
          const bool d1 = __shfl_down_sync(0xffffffffu, ch, 1) && lane <= 30;
          const bool d2 = __shfl_down_sync(0xffffffffu, ch, 2) && lane <= 29;
          if (u1 || d1) act |= (bit | (bit << 1) | (bit >> 1)) & cols;
          if (u2 || d2) act |= bit & cols;
          if (lane >= nrows) act = 0u;
          const unsigned anych = __ballot_sync(0xffffffffu, ch);
          if (anych) {
            const unsigned cb = bit | (bit >> 1);
            iact[0] |= cb & own[0];
            iact[1] |= cb & own[1];
          }
        }
        const unsigned nxt = __reduce_or_sync(0xffffffffu, act);
        if (dir == 2) todo = c >= 31 ? 0u : (nxt & ~((2u << c) - 1u));
        else todo = c == 0 ? 0u : (nxt & ((1u << c) - 1u));
      }
    }
    // interface nodes of the tile (lane = column)
    for (int rep = 0; rep < 2; ++rep) {
      if (!iact[0] && !iact[1]) break;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        NewV nv{0, false, 0.0f, 0.0f, 0.0f, 0.0f, false, false};
        const int slot = (R.H + side) * R.pitch + C.c0 + lane;
        const bool mine = (iact[side] >> lane) & 1u;
        if (mine) nv = update_iface(S, C, side, lane + kHalo, slot);
        __syncwarp();
        const int k = lane + kHalo;
        if (nv.write) {
          S.iTh[side][k] = nv.th; S.iTl[side][k] = nv.tl;
          S.igx[side][k] = nv.gx; S.igz[side][k] = nv.gz;
          S.ifl[side][k] = (uint8_t)((S.ifl[side][k] & kFlagSeed) | (nv.copy ? kFlagCopy : 0));
        }
        __syncwarp();
        iact[side] &= ~__ballot_sync(0xffffffffu, mine);
        const unsigned chg = __ballot_sync(0xffffffffu, nv.sig >= 1);
        isig[side] |= __ballot_sync(0xffffffffu, nv.sig == 2);
        // a moved interface node re-activates the grid nodes around its cut cell
        unsigned todo = chg;
        while (todo) {
          const int q = __ffs(todo) - 1;
          todo &= todo - 1u;
          const int rr = __shfl_sync(0xffffffffu, S.izc[side][k] - R.z_lo - C.r0, q);
          const int d = lane - rr;
          if (d >= -1 && d <= 2 && lane < nrows) {
            const unsigned cb = (1u << q) | ((1u << q) >> 1) | ((1u << q) << 1) | ((1u << q) << 2);
            act |= cb & cols;
          }
        }
        // the other interface's node of the same cut cell depends on it too
        iact[side ^ 1] |= chg & own[side ^ 1];
      }
    }
  }
  __syncwarp();
  // ---- write back every tile node whose value moved
  for (int e = lane; e < kTH * kTW; e += 32) {
    const int r = e / kTW, c = e % kTW;
    const int row = C.r0 + r, col = C.c0 + c;
    if (row >= R.H || col >= R.nx) continue;
    const int s = (r + kHalo) * kSP + c + kHalo;
    const int slot = row * R.pitch + col;
    const float2 g0 = reinterpret_cast<const float2*>(F.Th)[slot];
    if (g0.x != S.Th[s] || g0.y != S.Tl[s] || F.sflag[slot] != S.fl[s]) {
      reinterpret_cast<float2*>(F.Th)[slot] = make_float2(S.Th[s], S.Tl[s]);
      reinterpret_cast<float2*>(F.gx)[slot] = make_float2(S.gx[s], S.gz[s]);
      F.sflag[slot] = S.fl[s];
    }
  }
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    if (own[side] & (1u << lane)) {
      const int k = lane + kHalo;
      const int slot = (R.H + side) * R.pitch + C.c0 + lane;
      reinterpret_cast<float2*>(F.Th)[slot] = make_float2(S.iTh[side][k], S.iTl[side][k]);
      reinterpret_cast<float2*>(F.gx)[slot] = make_float2(S.igx[side][k], S.igz[side][k]);
      F.sflag[slot] = S.ifl[side][k];
    }
  }
  // ---- activation of neighbours whose halo moved
  const unsigned colmask = __reduce_or_sync(0xffffffffu, rowsig);
  const unsigned rowsch = __ballot_sync(0xffffffffu, rowsig != 0u);
  bool top = (rowsch & 0x3u) != 0u, bot = (rowsch & 0xC0000000u) != 0u;
  bool left = (colmask & 0x3u) != 0u, right = (colmask & 0xC0000000u) != 0u;
  bool tl = __ballot_sync(0xffffffffu, lane < 2 && (rowsig & 0x3u)) != 0u;
  bool tr = __ballot_sync(0xffffffffu, lane < 2 && (rowsig & 0xC0000000u)) != 0u;
  bool bl = __ballot_sync(0xffffffffu, lane >= kTH - 2 && (rowsig & 0x3u)) != 0u;
  bool br = __ballot_sync(0xffffffffu, lane >= kTH - 2 && (rowsig & 0xC0000000u)) != 0u;
  // interface nodes count as changes at their cut cell's corners
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const unsigned m = isig[side];
    if (!m) continue;
    right = right || (m & 0xC0000000u);
    left = left || (m & 0x3u);
    const bool mine = (m >> lane) & 1u;
    const int row = S.izc[side][lane + kHalo] - R.z_lo - C.r0;
    const bool nt_ = mine && row <= 1;
    const bool nb_ = mine && row >= kTH - 3;
    top = top || __any_sync(0xffffffffu, nt_);
    bot = bot || __any_sync(0xffffffffu, nb_);
    br = br || __any_sync(0xffffffffu, nb_ && lane >= 30);
    bl = bl || __any_sync(0xffffffffu, nb_ && lane < 2);
    tr = tr || __any_sync(0xffffffffu, nt_ && lane >= 30);
    tl = tl || __any_sync(0xffffffffu, nt_ && lane < 2);
  }
  if (lane == 0) {
    const int pn = parity ^ 1;
    if (!converged) activate(F, pn, tx, ty, kActAll, n_next);
    if (top) activate(F, pn, tx, ty - 1, kActBot, n_next);
    if (bot) activate(F, pn, tx, ty + 1, kActTop, n_next);
    if (left) activate(F, pn, tx - 1, ty, kActRight, n_next);
    if (right) activate(F, pn, tx + 1, ty, kActLeft, n_next);
    if (tl) activate(F, pn, tx - 1, ty - 1, kActBR, n_next);
    if (tr) activate(F, pn, tx + 1, ty - 1, kActBL, n_next);
    if (bl) activate(F, pn, tx - 1, ty + 1, kActTR, n_next);
    if (br) activate(F, pn, tx + 1, ty + 1, kActTL, n_next);
  }
}

// Final gradient pass over every tile of every field: re-evaluates each node
// on the converged field, writes the selected value's gradient and suspect
// flag (single-axis winner, refitted afterwards as the reference does when
// its heap is empty), and re-activates tiles where a node would still move by
// more than kSigDT (n_bad counts them; the caller then runs more rounds).
__global__ void __launch_bounds__(32, 4) eik_final(const DevField* __restrict__ fields, int nf,
                                                float* const* gout, uint8_t* const* susp,
                                                int parity, unsigned* n_bad) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem& S = *reinterpret_cast<TileSmem*>(smem_raw);
  const int b = blockIdx.x;
  const int fi = find_field(fields, nf, b);
  const DevField& F = fields[fi];
  const DevRegion& R = F.R;
  const int t = b - F.tile_base;
  const int nt = R.tiles_x * R.tiles_y;
  if (t >= nt) return;
  const int lane = threadIdx.x;
  const int tx = t % R.tiles_x, ty = t / R.tiles_x;
  TileCtx C;
  C.F = &F;
  C.c0 = tx * kTW;
  C.r0 = ty * kTH;
  C.h = R.dx;
  C.frozen_local = -1;
  load_tile(S, C, F, lane);
  unsigned own[2];
  owned_ifaces(S, C, F, lane, own);
  float2* G = reinterpret_cast<float2*>(gout[fi]);
  uint8_t* SU = susp[fi];
  bool bad = false;
  const int col = C.c0 + lane;
  for (int r = 0; r < kTH; ++r) {
    const int row = C.r0 + r;
    if (row >= R.H || col >= R.nx) continue;
    const int slot = row * R.pitch + col;
    const uint32_t code = R.code[slot];
    const int s = (r + kHalo) * kSP + lane + kHalo;
    float2 g = make_float2(S.gx[s], S.gz[s]);
    uint8_t su = 0;
    if ((code & kInRegion) && S.Th[s] < kReachedF) {
      const NewV nv = update_grid(S, C, r + kHalo, lane + kHalo, code, slot);
      if (nv.th < kReachedF) {
        g = make_float2(nv.gx, nv.gz);
        su = nv.suspect ? 1 : 0;
      }
      if (nv.sig == 2) bad = true;
    }
    G[slot] = g;
    SU[slot] = su;
  }
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    if (col >= R.nx) continue;
    const int k = lane + kHalo;
    const int slot = (R.H + side) * R.pitch + col;
    const bool mine = (own[side] >> lane) & 1u;
    // interface nodes that are never updated are written by the top tile row
    const bool writer = mine || (!(S.icode[side][k] & kUpdatable) && ty == 0);
    if (!writer) continue;
    float2 g = make_float2(S.igx[side][k], S.igz[side][k]);
    if (mine && S.iTh[side][k] < kReachedF) {
      const NewV nv = update_iface(S, C, side, k, slot);
      if (nv.th < kReachedF) g = make_float2(nv.gx, nv.gz);
      if (nv.sig == 2) bad = true;
    }
    G[slot] = g;
    SU[slot] = 0;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) {
    unsigned* a = F.act + (size_t)parity * nt + t;
    if (atomicOr(a, kActAll) == 0u) atomicAdd(n_bad, 1u);
  }
}

size_t eik_round_smem() { return sizeof(TileSmem); }

}  // namespace fmt2d
