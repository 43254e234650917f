// Candidate arithmetic of the eikonal stencil, shared by the device solver
// and host code (the same functions compile for both, so a host run of the
// solver's schedule reproduces the device's doubles bit for bit).
//
// Fast marching (src/propagate2d.f90:33-127) gives every node the smallest of
// its seed and of the candidate times its update events produce, each event
// using the accepted (final) values of the nodes involved:
//   * per regular quadrant, the one-sided update triggered by the earlier
//     neighbour and the two-sided update triggered by the later one, with the
//     second-order switch, face-averaged velocity, det clamp and t >= tmax of
//     regular_update2d (:605-790);
//   * per cut cell of the region's own interfaces, time_from_1_node2d for the
//     trigger and time_from_2_nodes2d for the trigger paired with every member
//     accepted before it (:793-946), in update_time2d's order (:482-602).
// Of equal candidates the one produced first wins (updates replace a time
// only when strictly smaller), so candidates carry their event (trigger time,
// position within the trigger's update) and ties go to the earlier event.
//
// Arithmetic is FP64 in the reference's expression order; files including
// this header are compiled without FMA contraction.
//
// Memory: the static region arrays (code, velocity, interface tables) are
// read through the read-only path; times, gradients and flags with plain
// loads.  The solver reads and writes a field from one thread block only, with
// a block barrier between the phases that write and the phases that read, so
// plain (L1-cached) loads see every committed value.
#pragma once
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cuda_runtime.h>
#include "eik64.cuh"
#include "model.h"

// A second translation unit that includes this header defines FMT_HD_LINK as
// `static` so the two copies of these functions do not collide at link time.
#ifndef FMT_HD_LINK
#define FMT_HD_LINK
#endif
#if defined(__CUDACC__)
#define FMT_HD FMT_HD_LINK __host__ __device__
#else
#define FMT_HD FMT_HD_LINK
#endif

#ifdef __CUDA_ARCH__
#define FMT_RO(p) __ldg(p)
#else
#define FMT_RO(p) (*(p))
#endif

namespace fmt2d {
namespace ev {

#ifndef __CUDA_ARCH__
using std::fmax;
using std::fmin;
using std::fabs;
using std::sqrt;
#endif

constexpr double kTinyD = 2.2250738585072014e-308;   // Fortran tiny(1.0_dp)

FMT_HD inline long long bits_of(double d) {
#ifdef __CUDA_ARCH__
  return __double_as_longlong(d);
#else
  long long b;
  std::memcpy(&b, &d, sizeof b);
  return b;
#endif
}

FMT_HD inline double ldT(const Fld64& F, int s) { return F.T[s]; }
FMT_HD inline double2 ldG(const Fld64& F, int s) { return F.G[s]; }
FMT_HD inline uint8_t ldF(const Fld64& F, int s) { return F.fl[s]; }
FMT_HD inline double xg(const Fld64& F, int col) { return F.x0 + (double)col * F.dx; }
FMT_HD inline double zg(const Fld64& F, int brow) { return (double)(F.z_lo + brow) * F.dx; }

// ---------------------------------------------------------------- candidates
// A candidate carries its event and the operands of its gradient; the
// gradient itself (divisions and a square root) is formed for the winner
// only, by the same expressions the reference evaluates when a candidate
// lowers the node.
enum : uint8_t { kGradNone = 0, kGradReg, kGradRay, kGradPlane, kGradGiven };

struct Cand {
  double t, trig;
  double g0, g1, g2, g3, g4, g5;   // gradient operands, by kind (grad_of)
  int ord;
  uint8_t kind;
  bool gxi, gzi;                   // regular: the x / z neighbour took part
  bool sus, copy;
};

FMT_HD inline Cand no_cand() {
  Cand c;
  c.t = kHugeD; c.trig = kHugeD; c.ord = 0x7fffffff;
  c.g0 = c.g1 = c.g2 = c.g3 = c.g4 = c.g5 = 0.0;
  c.kind = kGradNone; c.gxi = c.gzi = false;
  c.sus = false; c.copy = false;
  return c;
}

FMT_HD inline bool earlier(double trig, int ord, const Cand& b) {
  return trig < b.trig || (trig == b.trig && ord < b.ord);
}

// Keep c (its t, trig and ord set) if it beats best.
FMT_HD inline void take(Cand& best, const Cand& c) {
  if (c.t < best.t || (c.t == best.t && earlier(c.trig, c.ord, best))) best = c;
}

// The gradient a winning candidate writes: regular_update2d's one-sided first
// or second-order differences (:766-782), time_from_1_node2d's straight ray
// (:823-826), time_from_2_nodes2d's plane-wave normal (:921-940) or a member's
// gradient handed over.
FMT_HD inline void grad_of(const Cand& w, double& gx, double& gz) {
  gx = 0.0;
  gz = 0.0;
  switch (w.kind) {
    case kGradReg:
      if (w.gxi)
        gx = (w.g1 == 0.0) ? (w.t - w.g0) / w.g2 : 0.5 * (3.0 * w.t - 4.0 * w.g0 + w.g1) / w.g2;
      if (w.gzi)
        gz = (w.g4 == 0.0) ? (w.t - w.g3) / w.g5 : 0.5 * (3.0 * w.t - 4.0 * w.g3 + w.g4) / w.g5;
      break;
    case kGradRay:
      gx = w.g0 / (w.g2 * w.g3);
      gz = w.g1 / (w.g2 * w.g3);
      break;
    case kGradPlane: {
      const double wl = sqrt(w.g0 * w.g0 + w.g1 * w.g1);
      gx = w.g0 / (wl * w.g2);
      gz = w.g1 / (wl * w.g2);
      break;
    }
    case kGradGiven:
      gx = w.g0;
      gz = w.g1;
      break;
    default:
      break;
  }
}

// A direct neighbour of a grid node, as regular_update2d sees it.
struct RNb {
  bool ok, single_ok, second, dirx;
  double T, T2, d2, dpos;
};

// The four direct neighbours (L, R, U, D) of grid node (r, c): reached, the
// face velocity term and the second-order switch (:642-673, :688-719), with
// the loads of all four directions issued together (codes, then times and
// velocities, then the gradients the switch needs), so a node pays a few
// memory round trips instead of a chain per direction.
FMT_HD void rnb4(const Fld64& F, int r, int c, double vu, RNb* n) {
  const int dr[4] = {0, 0, -1, 1}, dc[4] = {-1, 1, 0, 0};
  int s1[4], s2[4];
  bool b1[4], b2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rn = r + dr[k], cn = c + dc[k], r2 = r + 2 * dr[k], c2 = c + 2 * dc[k];
    b1[k] = rn >= 0 && rn < F.H && cn >= 0 && cn < F.nx;
    b2[k] = b1[k] && r2 >= 0 && r2 < F.H && c2 >= 0 && c2 < F.nx;
    s1[k] = b1[k] ? rn * F.pitch + cn : 0;
    s2[k] = b2[k] ? r2 * F.pitch + c2 : 0;
  }
  // codes, times, velocities and gradients are loaded in one round: a slot
  // inside the band but outside the region holds huge_time (never written),
  // so its time is read safely and discarded below
  uint32_t k1[4], k2[4];
  double t1[4], t2[4], v1[4], v2[4];
  double2 g1[4], g2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    k1[k] = b1[k] ? FMT_RO(F.code + s1[k]) : 0u;
    k2[k] = b2[k] ? FMT_RO(F.code + s2[k]) : 0u;
    t1[k] = b1[k] ? ldT(F, s1[k]) : kHugeD;
    v1[k] = b1[k] ? FMT_RO(F.vel + s1[k]) : 0.0;
    t2[k] = b2[k] ? ldT(F, s2[k]) : kHugeD;
    v2[k] = b2[k] ? FMT_RO(F.vel + s2[k]) : 0.0;
    g1[k] = b2[k] ? ldG(F, s1[k]) : make_double2(0.0, 0.0);
    g2[k] = b2[k] ? ldG(F, s2[k]) : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    b1[k] = b1[k] && (k1[k] & kInRegion);
    b2[k] = b2[k] && (k2[k] & kInRegion);
    if (!b1[k]) t1[k] = kHugeD;
    if (!b2[k]) t2[k] = kHugeD;
  }
  bool need[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    RNb& m = n[k];
    m.ok = false;
    m.second = false;
    m.dirx = dc[k] != 0;
    need[k] = false;
    if (!b1[k] || !(t1[k] < kReachD)) continue;
    m.ok = true;
    m.single_ok = s1[k] != F.frozen_slot;
    m.T = t1[k];
    const double velx = 0.5 * (vu + v1[k]);
    const double dd = velx / F.dx;
    m.d2 = dd * dd;
    m.dpos = m.dirx ? xg(F, c) - xg(F, c + dc[k]) : zg(F, r) - zg(F, r + dr[k]);
    if (!b2[k]) continue;
    if (!(t2[k] < kReachD) || !(t1[k] >= t2[k])) continue;
    if (!(v1[k] * v2[k] > kTinyD)) continue;
    need[k] = true;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (need[k] && g1[k].x * g2[k].x + g1[k].y * g2[k].y >= 0.71 / (v1[k] * v2[k])) {
      n[k].second = true;
      n[k].T2 = t2[k];
    }
  }
}

// regular_update2d (:605-790) for one or two accepted neighbours: the
// candidate time, its suspect flag and its gradient operands.
FMT_HD bool reg_cand(const RNb* p, const RNb* q, Cand& o) {
  double a = 0.0, b = 0.0, c = 0.0, t2x = 0.0, t2z = 0.0, tx = 0.0, tz = 0.0, tmax = 0.0;
  double dpx = 1.0, dpz = 1.0;
  bool xi = false, zi = false;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const RNb* n = k == 0 ? p : q;
    if (!n) continue;
    tmax = fmax(tmax, n->T);
    if (n->dirx) {
      xi = true;
      dpx = n->dpos;
      if (n->second) {
        tx = n->T;
        t2x = n->T2;
        a += 2.25 * n->d2;
        b += (-6.0 * tx + 1.5 * t2x) * n->d2;
        c += (4.0 * tx * tx - 2.0 * tx * t2x + 0.25 * t2x * t2x) * n->d2;
      } else {
        tx = n->T;
        a += n->d2;
        b += (-2.0 * tx) * n->d2;
        c += (tx * tx) * n->d2;
      }
    } else {
      zi = true;
      dpz = n->dpos;
      if (n->second) {
        tz = n->T;
        t2z = n->T2;
        a += 2.25 * n->d2;
        b += (-6.0 * tz + 1.5 * t2z) * n->d2;
        c += (4.0 * tz * tz - 2.0 * tz * t2z + 0.25 * t2z * t2z) * n->d2;
      } else {
        tz = n->T;
        a += n->d2;
        b += (-2.0 * tz) * n->d2;
        c += (tz * tz) * n->d2;
      }
    }
  }
  c = c - 1.0;
  if (fabs(a) < kTinyD) return false;
  double det = b * b - 4.0 * a * c;
  if (det < 0.0) {
    if (0.5 * sqrt(fabs(det)) / fabs(a) < 1.0e20) det = 0.0;
    else return false;
  }
  const double t1 = 0.5 * (-b + sqrt(det)) / a;
  o.t = fmax(t1, tmax);
  o.kind = kGradReg;
  o.gxi = xi;
  o.gzi = zi;
  o.g0 = tx; o.g1 = t2x; o.g2 = dpx;
  o.g3 = tz; o.g4 = t2z; o.g5 = dpz;
  o.sus = !(xi && zi);
  o.copy = false;
  return true;
}

// Candidates of one regular quadrant (X along x, Z along z): the one-sided
// update of the earlier neighbour (triggered while the other was not yet
// accepted) and the two-sided update (triggered by the later one).
FMT_HD void quadrant(const RNb& X, const RNb& Z, int ord, Cand& best) {
  Cand c;
  c.ord = ord;
  if (X.ok && Z.ok) {
    const bool xlow = X.T <= Z.T;
    const RNb& lo = xlow ? X : Z;
    if (lo.single_ok && reg_cand(&lo, nullptr, c)) {
      c.trig = lo.T;
      take(best, c);
    }
    if (reg_cand(&X, &Z, c)) {
      c.trig = fmax(X.T, Z.T);
      take(best, c);
    }
  } else if (X.ok) {
    if (X.single_ok && reg_cand(&X, nullptr, c)) {
      c.trig = X.T;
      take(best, c);
    }
  } else if (Z.ok) {
    if (Z.single_ok && reg_cand(&Z, nullptr, c)) {
      c.trig = Z.T;
      take(best, c);
    }
  }
}

// A member of a cut cell (absolute position, accepted values).
struct Mem {
  double x, z, T, gx, gz, v;
  bool single_ok, copied;
};

// Cut-cell candidates.  pre_min tracks the smallest cut-cell candidate that
// comes before the best regular candidate (rtrig, rord) in event order: the
// reference writes the suspect flag only in regular updates, so a node keeps
// that candidate's flag only if it actually lowered the node.
struct CutAcc {
  Cand best;
  double pre_min, rtrig;
  int rord;
};

FMT_HD inline void offer(CutAcc& A, Cand& c, double t, double trig, int ord, bool copy) {
  c.t = t;
  c.trig = trig;
  c.ord = ord;
  c.sus = false;
  c.copy = copy;
  take(A.best, c);
  if (trig < A.rtrig || (trig == A.rtrig && ord < A.rord)) A.pre_min = fmin(A.pre_min, t);
}

// Gradient operands of a member's gradient handed over, of a straight ray
// from a member, of a plane front.
FMT_HD inline void given(Cand& c, double gx, double gz) {
  c.kind = kGradGiven;
  c.g0 = gx;
  c.g1 = gz;
}

// time_from_1_node2d (:793-829).  A member closer than 0.01*tolerance hands
// its values over ("copy"); a copy is only taken from a member whose own value
// is not a copy, which is what the heap's acceptance order guarantees for
// coincident nodes.
FMT_HD void from_1(const Mem& a, double xu, double zu, double vu, double tol, double trig,
                       int ord, CutAcc& A) {
  const double dxu = xu - a.x, dzu = zu - a.z;
  const double dist = sqrt(dxu * dxu + dzu * dzu);
  Cand c;
  if (dist < 0.01 * tol) {
    if (!a.copied) {
      given(c, a.gx, a.gz);
      offer(A, c, a.T, trig, ord, true);
    }
    return;
  }
  const double tt = dist / (0.5 * (vu + a.v));
  const double at = a.T + tt;
  c.kind = kGradRay;
  c.g0 = dxu;
  c.g1 = dzu;
  c.g2 = dist;
  c.g3 = vu;
  offer(A, c, at, trig, ord, false);
}

// time_from_2_nodes2d (:832-946): planar front through the trigger n1 and an
// earlier member n2.
FMT_HD void from_2(const Mem& n1, const Mem& n2, double xu, double zu, double vu, double tol,
                       int ord, CutAcc& A) {
  const double trig = n1.T;
  const double r1x = n1.x - xu, r1z = n1.z - zu;
  const double r2x = n2.x - xu, r2z = n2.z - zu;
  Cand c;
  if (sqrt(r1x * r1x + r1z * r1z) < 0.01 * tol) {
    if (!n1.copied) {
      given(c, n1.gx, n1.gz);
      offer(A, c, n1.T, trig, ord, true);
    }
    return;
  }
  if (sqrt(r2x * r2x + r2z * r2z) < 0.01 * tol) {
    if (!n2.copied) {
      given(c, n2.gx, n2.gz);
      offer(A, c, n2.T, trig, ord, true);
    }
    return;
  }
  const double ex = n2.x - n1.x, ez = n2.z - n1.z;
  if (sqrt(ex * ex + ez * ez) < 0.01 * tol) {
    from_1(n1, xu, zu, vu, tol, trig, ord, A);
    return;
  }
  const double v12 = 0.5 * (n1.v + n2.v);
  const double dx_ = (n1.x - n2.x) / v12, dz_ = (n1.z - n2.z) / v12;
  const double dd = dx_ * dx_ + dz_ * dz_;
  const double px = (n1.T - n2.T) / dd * dx_;
  const double pz = (n1.T - n2.T) / dd * dz_;
  const double qx = -dz_, qz = dx_;
  const double ae = qx * qx + qz * qz;
  const double be = 2.0 * (px * qx + pz * qz);
  const double ce = px * px + pz * pz - 1.0;
  const double det = be * be - 4.0 * ae * ce;
  if (det < 0.0) return;
  const double u1 = 0.5 * (-be + sqrt(det)) / ae;
  const double u2 = 0.5 * (-be - sqrt(det)) / ae;
  double m1x = -r1z, m1z = r1x;
  double l = sqrt(m1x * m1x + m1z * m1z);
  m1x /= l;
  m1z /= l;
  if (m1x * r2x + m1z * r2z < 0.0) { m1x = -m1x; m1z = -m1z; }
  double m2x = -r2z, m2z = r2x;
  l = sqrt(m2x * m2x + m2z * m2z);
  m2x /= l;
  m2z /= l;
  if (m2x * r1x + m2z * r1z < 0.0) { m2x = -m2x; m2z = -m2z; }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double u = k == 0 ? u1 : u2;
    const double wx = px + u * qx, wz = pz + u * qz;
    if (wx * m1x + wz * m1z <= 0.0 && wx * m2x + wz * m2z <= 0.0) {
      const double at = n1.T - (wx * r1x + wz * r1z) / (0.5 * (vu + n1.v));
      if (at >= n1.T) {
        c.kind = kGradPlane;
        c.g0 = wx;
        c.g1 = wz;
        c.g2 = n1.v;
        offer(A, c, at, trig, ord, false);
      }
    }
  }
}

// Every event of one cut cell.  Members are listed in the reference's
// connected-node order.  When member p is accepted the cell's list holds the
// members accepted by then (p included) in that order; update_time2d swaps p
// to the front and calls time_from_1 (p), then time_from_2 (p, list[k]) for
// k = 1.. of the swapped list.
// The events triggered by member p of a cut cell (its acceptance).
FMT_HD void cut_member(const Mem* m, int nm, int p, double xu, double zu, double vu, double tol,
                       int cbase, CutAcc& A) {
  if (!m[p].single_ok) return;
  int lst[6], n = 0, pp = 0;
  for (int q = 0; q < nm; ++q) {
    const bool before = q == p || m[q].T < m[p].T || (m[q].T == m[p].T && q < p);
    if (!before) continue;
    if (q == p) pp = n;
    lst[n++] = q;
  }
  from_1(m[p], xu, zu, vu, tol, m[p].T, cbase, A);
  for (int k = 1; k < n; ++k) {
    const int q = (k == pp) ? lst[0] : lst[k];
    from_2(m[p], m[q], xu, zu, vu, tol, cbase + k, A);
  }
}

FMT_HD void cut_cell(const Mem* m, int nm, double xu, double zu, double vu, double tol,
                         int cbase, CutAcc& A) {
  for (int p = 0; p < nm; ++p) cut_member(m, nm, p, xu, zu, vu, tol, cbase, A);
}

FMT_HD inline bool member_at(const Fld64& F, int brow, int col, Mem& m) {
  if (brow < 0 || brow >= F.H || col < 0 || col >= F.nx) return false;
  const int s = brow * F.pitch + col;
  if (!(FMT_RO(F.code + s) & kInRegion)) return false;
  const double T = ldT(F, s);
  if (!(T < kReachD)) return false;
  const double2 g = ldG(F, s);
  m.x = xg(F, col);
  m.z = zg(F, brow);
  m.T = T;
  m.gx = g.x;
  m.gz = g.y;
  m.v = FMT_RO(F.vel + s);
  m.single_ok = s != F.frozen_slot;
  m.copied = (ldF(F, s) & kFlCopy) != 0;
  return true;
}

FMT_HD inline bool member_iface(const Fld64& F, int side, int col, Mem& m) {
  if (col < 0 || col >= F.nx) return false;
  const int s = (F.H + side) * F.pitch + col;
  const double T = ldT(F, s);
  if (!(T < kReachD)) return false;
  const double2 g = ldG(F, s);
  m.x = FMT_RO(F.ifx + col);
  m.z = FMT_RO(F.ifz + side * F.pitch + col);
  m.T = T;
  m.gx = g.x;
  m.gz = g.y;
  m.v = FMT_RO(F.vel + s);
  m.single_ok = true;
  m.copied = (ldF(F, s) & kFlCopy) != 0;
  return true;
}

// New value of a node and whether it must be written.
struct NewV {
  bool write, spread;   // store it; re-activate the stencil neighbours
  double T, gx, gz;
  bool sus, copy;
};

// Seeds precede every candidate in the reference's order; a seed at or below
// the regular candidate that would set the suspect flag means that update
// never lowered the node.
//
// A seed tied with a copy from a coincident node (an interface node lying on
// a grid node) is the one case the fixed point does not decide: the heap
// accepts either node first, and both end with that node's values.  A grid
// node seeded at zero distance from its interface node carries a NaN gradient
// (sweep_region_from_interface2d divides by the distance), so which of the two
// the heap pops first decides whether rays through that cell can be traced.
// Keeping the seed leaves NaN on the grid node; over PmP picks of twelve test
// models this agreed with the reference's valid flags on 96.6% of picks,
// against 95.2% for letting a finite copy win.
FMT_HD NewV finish(const Fld64& F, int s, const Cand& w, bool sus, double sus_t) {
  NewV o;
  o.write = false;
  o.spread = false;
  double gx, gz;
  grad_of(w, gx, gz);
  double T = w.t < kReachD ? w.t : kHugeD;
  bool su = sus, cp = w.copy;
  const uint8_t fl = ldF(F, s);
  if (fl & kFlSeed) {
    const double4 sd = F.seed[s];
    if (sd.x < kReachD) {
      if (T >= kReachD || sd.x <= T) {
        T = sd.x; gx = sd.y; gz = sd.z; su = false; cp = false;
      } else if (su && sd.x <= sus_t) {
        su = false;
      }
    }
  }
  const double curT = ldT(F, s);
  if (T >= kReachD) {
    T = kHugeD; gx = 0.0; gz = 0.0; su = false; cp = false;
    if (curT >= kReachD) return o;
  }
  // compared bit for bit: a NaN gradient (a seed at zero distance) must not
  // count as a change on every evaluation
  const double2 cg = ldG(F, s);
  auto same = [](double a, double b) { return bits_of(a) == bits_of(b); };
  const bool gchg = !same(T, curT) || !same(gx, cg.x) || !same(gz, cg.y) ||
                    cp != ((fl & kFlCopy) != 0);
  o.T = T; o.gx = gx; o.gz = gz; o.sus = su; o.copy = cp;
  o.spread = gchg;
  o.write = gchg || su != ((fl & kFlSusp) != 0);
  // with a change threshold, a move smaller than it (time in s, gradient in
  // s/km) is stored but re-lists nobody: the fixed point is then solved to
  // within the threshold instead of to the last bit
  if (gchg && F.eps > 0.0 && cp == ((fl & kFlCopy) != 0) && curT < kReachD && T < kReachD &&
      fabs(T - curT) <= F.eps && fabs(gx - cg.x) <= F.eps && fabs(gz - cg.y) <= F.eps)
    o.spread = false;
  return o;
}

// Members of connected cut cell q of grid node (r, c), in the reference's
// connected-node order: the top and bottom interface nodes the cell carries,
// then its corners other than the node itself.
FMT_HD inline int cell_members(const Fld64& F, int r, int c, uint32_t code, int q, Mem* m) {
  const int ci = r - ((q & 1) ? 1 : 0), cj = c - (q >= 2 ? 1 : 0);
  int nm = 0;
  if ((code & (1u << (12 + q))) && member_iface(F, 0, cj, m[nm])) ++nm;
  if ((code & (1u << (16 + q))) && member_iface(F, 1, cj, m[nm])) ++nm;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      const int rr = ci + b, cc = cj + a;
      if (rr == r && cc == c) continue;
      if (member_at(F, rr, cc, m[nm])) ++nm;
    }
  return nm;
}

// Update of the grid node at bbox row r, column c.
FMT_HD NewV update_grid(const Fld64& F, int r, int c) {
  NewV none;
  none.write = false;
  none.spread = false;
  const int s = r * F.pitch + c;
  const uint32_t code = FMT_RO(F.code + s);
  if (!(code & kInRegion) || !(code & kUpdatable) || s == F.frozen_slot) return none;
  const double vu = FMT_RO(F.vel + s);
  RNb nb[4];
  rnb4(F, r, c, vu, nb);
  const RNb &L = nb[0], &R = nb[1], &U = nb[2], &D = nb[3];
  if (code & kFullyRegular) {
    // update_time2d's quadrant loop: (L,U), (R,U), (L,D), (R,D)
    Cand best = no_cand();
    quadrant(L, U, 0, best);
    quadrant(R, U, 1, best);
    quadrant(L, D, 2, best);
    quadrant(R, D, 3, best);
    return finish(F, s, best, best.sus, best.t);
  }
  // connected cells c0..c3 = (R,D), (R,U), (L,D), (L,U)
  Cand rb = no_cand();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (!(code & (1u << (4 + q))) || (code & (1u << (8 + q)))) continue;
    quadrant((q >= 2) ? L : R, (q & 1) ? U : D, q * 32, rb);
  }
  CutAcc A;
  A.best = no_cand();
  A.pre_min = kHugeD;
  A.rtrig = rb.trig;
  A.rord = rb.ord;
  const double xu = xg(F, c), zu = zg(F, r);
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    if (!(code & (1u << (4 + q))) || !(code & (1u << (8 + q)))) continue;
    Mem m[6];
    const int nm = cell_members(F, r, c, code, q, m);
    cut_cell(m, nm, xu, zu, vu, F.tol, q * 32, A);
  }
  const bool reg_wins = rb.t < A.best.t || (rb.t == A.best.t && earlier(rb.trig, rb.ord, A.best));
  const Cand& w = reg_wins ? rb : A.best;
  const bool sus = rb.sus && (reg_wins || rb.t < A.pre_min);
  return finish(F, s, w, sus, rb.t);
}

// Update of interface node `col` on side 0 (top) or 1 (bottom).
FMT_HD NewV update_iface(const Fld64& F, int side, int col) {
  NewV none;
  none.write = false;
  none.spread = false;
  const int s = (F.H + side) * F.pitch + col;
  const uint32_t code = FMT_RO(F.code + s);
  if (!(code & kInRegion) || !(code & kUpdatable)) return none;
  const int izc = FMT_RO(F.izc + side * F.pitch + col);
  if (izc < 0) return none;
  const double vu = FMT_RO(F.vel + s);
  const double xu = FMT_RO(F.ifx + col), zu = FMT_RO(F.ifz + side * F.pitch + col);
  Mem m[6];
  int nm = 0;
  const int o = side ^ 1;
  const bool has_o = o == 0 ? (code & (1u << 12)) : (code & (1u << 16));
  if (has_o && member_iface(F, o, col, m[nm])) ++nm;
  const int br = izc - F.z_lo;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      if (member_at(F, br + b, col + a, m[nm])) ++nm;
  CutAcc A;
  A.best = no_cand();
  A.pre_min = kHugeD;
  A.rtrig = -kHugeD;
  A.rord = -1;
  cut_cell(m, nm, xu, zu, vu, F.tol, 0, A);
  return finish(F, s, A.best, false, kHugeD);
}

// Evaluate node `slot` of field F (grid row or interface row).
FMT_HD inline NewV evaluate(const Fld64& F, int slot) {
  const int row = slot / F.pitch, col = slot - (slot / F.pitch) * F.pitch;
  if (row < F.H) return update_grid(F, row, col);
  return update_iface(F, row - F.H, col);
}

// fit_gradient_at_node2d (:949-1196): central differences in a regular
// neighbourhood, else a distance-weighted 2x2 least-squares fit over the
// nodes of the connected cells.
FMT_HD void fit_grad(const Fld64& F, int slot, double& dtdx, double& dtdz) {
  const uint32_t code = F.code[slot];
  const bool iface = (code & kIfaceNode) != 0;
  const int side = iface ? (slot / F.pitch - F.H) : 0;
  const int col = slot % F.pitch;
  const int brow = iface ? -1 : slot / F.pitch;
  const double h = F.dx;
  auto in_reg = [&](int c, int absrow) -> int {
    const int br = absrow - F.z_lo;
    if (c < 0 || c >= F.nx || br < 0 || br >= F.H) return -1;
    const int s = br * F.pitch + c;
    return (F.code[s] & kInRegion) ? s : -1;
  };
  auto tt = [&](int s) { return F.T[s]; };
  double xu, zu;
  if (iface) { xu = F.ifx[col]; zu = F.ifz[side * F.pitch + col]; }
  else { xu = F.x0 + col * h; zu = (brow + F.z_lo) * h; }
  int ncl = 0, clx[4], clz[4];
  bool any[4];
  if (!iface) {
    for (int c = 0; c < 4; ++c) {
      if (!(code & (1u << (4 + c)))) continue;
      if ((c >= 2 && col == 0) || ((c & 1) && brow + F.z_lo == 0)) continue;
      clx[ncl] = col - (c >= 2 ? 1 : 0);
      clz[ncl] = brow + F.z_lo - ((c & 1) ? 1 : 0);
      any[ncl] = (code & (1u << (20 + c))) != 0;
      ++ncl;
    }
  } else {
    const int izc = F.izc[side * F.pitch + col];
    if (izc >= 0) { clx[0] = col; clz[0] = izc; any[0] = (code & (1u << 20)) != 0; ncl = 1; }
  }
  int nirr = 0;
  for (int n = 0; n < ncl; ++n) nirr += any[n] ? 1 : 0;
  if (nirr == 0) {
    if (!iface) {
      const int absr = brow + F.z_lo;
      int m = in_reg(max(0, col - 1), absr), n = in_reg(min(F.nx - 1, col + 1), absr);
      const double xm = F.x0 + max(0, col - 1) * h, xn = F.x0 + min(F.nx - 1, col + 1) * h;
      if (m >= 0 && n >= 0) dtdx = (tt(n) - tt(m)) / (xn - xm);
      else if (m >= 0) dtdx = (tt(slot) - tt(m)) / (xu - xm);
      else if (n >= 0) dtdx = (tt(n) - tt(slot)) / (xn - xu);
      else dtdx = 0.0;
      const int zm = max(0, absr - 1), zn = min(F.nz - 1, absr + 1);
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
  auto takep = [&](int s, double x, double z) {
    if (s == slot || s < 0) return;
    for (int k = 0; k < ns; ++k)
      if (store[k] == s) return;
    if (ns < 30) { store[ns] = s; rx[ns] = x; rz[ns] = z; at[ns] = tt(s); ++ns; }
  };
  for (int n = 0; n < ncl; ++n) {
    if (any[n] && clx[n] >= 0 && clx[n] < F.nx) {
      const int cx = clx[n];
      for (int sd = 0; sd < 2; ++sd) {
        if (F.izc[sd * F.pitch + cx] != clz[n]) continue;
        const int s = (F.H + sd) * F.pitch + cx;
        const double zi = F.ifz[sd * F.pitch + cx];
        if (!(zi >= clz[n] * h && zi <= (clz[n] + 1) * h)) continue;
        takep(s, F.ifx[cx], zi);
      }
    }
    for (int i = 0; i <= 1; ++i)
      for (int j = 0; j <= 1; ++j) {
        const int a = clx[n] + i, b = clz[n] + j;
        const int s = in_reg(a, b);
        if (s >= 0) takep(s, F.x0 + a * h, b * h);
      }
  }
  double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0;
  const double tu = tt(slot);
  for (int i = 0; i < ns; ++i) {
    const double ddx = rx[i] - xu, ddz = rz[i] - zu;
    const double dw = 1.0 / (sqrt(ddx * ddx + ddz * ddz) + F.tol);
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

// Final gradients: the winning candidate's, suspect nodes refitted

// Nodes whose candidates read node `slot` (the nodes a change of it can
// move), by fixed position q = 0..15: for a grid node its second neighbours
// along the axes and its 3x3 block (q < 12) and the interface nodes of the
// cut cells it is a corner of (q = 12..15); for an interface node the corners
// of its cut cell (q < 4) and the node of the other interface row in the
// same column (q = 4).  Returns the target's slot, or -1 where position q
// holds no node.
FMT_HD inline int spread_target_at(const Fld64& F, int slot, int q) {
  const int row = slot / F.pitch, c = slot - row * F.pitch;
  if (row < F.H) {
    if (q < 12) {
      const int dr = q < 2 ? (q == 0 ? -2 : 2) : (q < 4 ? 0 : (q < 7 ? -1 : (q < 9 ? 0 : 1)));
      const int dc = q < 2 ? 0 : (q < 4 ? (q == 2 ? -2 : 2)
                                        : (q < 7 ? q - 5 : (q < 9 ? (q == 7 ? -1 : 1) : q - 10)));
      const int rr = row + dr, cc = c + dc;
      if (rr < 0 || rr >= F.H || cc < 0 || cc >= F.nx) return -1;
      const int s = rr * F.pitch + cc;
      return (FMT_RO(F.code + s) & kInRegion) ? s : -1;
    }
    const int k = q - 12, side = k >> 1, kc = c - 1 + (k & 1);
    if (kc < 0 || kc >= F.nx) return -1;
    const int izc = FMT_RO(F.izc + side * F.pitch + kc), ar = F.z_lo + row;
    return (izc >= 0 && (izc == ar || izc + 1 == ar)) ? (F.H + side) * F.pitch + kc : -1;
  }
  const int side = row - F.H;
  if (q == 4) return (F.H + (side ^ 1)) * F.pitch + c;
  if (q > 4) return -1;
  const int izc = FMT_RO(F.izc + side * F.pitch + c);
  if (izc < 0) return -1;
  const int rr = izc - F.z_lo + (q & 1), cc = c + (q >> 1);
  if (rr < 0 || rr >= F.H || cc < 0 || cc >= F.nx) return -1;
  const int s = rr * F.pitch + cc;
  return (FMT_RO(F.code + s) & kInRegion) ? s : -1;
}

// Position q of the same neighbourhood without looking at the region: the
// slot, or -1 outside the band (a superset of spread_target_at's nodes).
FMT_HD inline int neighbour_slot(const Fld64& F, int slot, int q) {
  const int row = slot / F.pitch, c = slot - row * F.pitch;
  if (row < F.H) {
    if (q < 12) {
      const int dr = q < 2 ? (q == 0 ? -2 : 2) : (q < 4 ? 0 : (q < 7 ? -1 : (q < 9 ? 0 : 1)));
      const int dc = q < 2 ? 0 : (q < 4 ? (q == 2 ? -2 : 2)
                                        : (q < 7 ? q - 5 : (q < 9 ? (q == 7 ? -1 : 1) : q - 10)));
      const int rr = row + dr, cc = c + dc;
      if (rr < 0 || rr >= F.H || cc < 0 || cc >= F.nx) return -1;
      return rr * F.pitch + cc;
    }
    const int k = q - 12, kc = c - 1 + (k & 1);
    if (kc < 0 || kc >= F.nx) return -1;
    return (F.H + (k >> 1)) * F.pitch + kc;
  }
  const int side = row - F.H;
  if (q == 4) return (F.H + (side ^ 1)) * F.pitch + c;
  if (q > 4) return -1;
  const int izc = FMT_RO(F.izc + side * F.pitch + c);
  if (izc < 0) return -1;
  const int rr = izc - F.z_lo + (q & 1), cc = c + (q >> 1);
  if (rr < 0 || rr >= F.H || cc < 0 || cc >= F.nx) return -1;
  return rr * F.pitch + cc;
}

// The same targets as a list: writes at most 16 slots to t, returns their
// number.
FMT_HD inline int spread_targets(const Fld64& F, int slot, int* t) {
  int n = 0;
  for (int q = 0; q < 16; ++q) {
    const int s = spread_target_at(F, slot, q);
    if (s >= 0) t[n++] = s;
  }
  return n;
}

}  // namespace ev
}  // namespace fmt2d
