// FP64 tiled eikonal solver: the reference's fast-marching stencil solved to
// its fixed point by data-parallel relaxation.
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
// The solve is a fast iterative method over every field of a batch at once:
// nodes whose inputs changed are listed, and each step evaluates every listed
// node once (a thread per node) and lists the nodes a changed node can move.
// A per-field time window bounds what may be written: a node whose new time
// lies beyond it waits, and the window moves on only after a step in which
// nothing inside it changed, so nodes settle in time slices as the heap
// accepts them.  When the list is empty every node is at the fixed point (a
// final check re-lists any that is not).  Reads of other nodes go through L2
// (.cg), since other threads write them during the kernel.
//
// Arithmetic is FP64 with the reference's expression order; this file is
// compiled with --fmad=false so candidate times are bit-identical to the
// FP64 restatement's.
#include "eik64.cuh"
#include "model.h"

namespace fmt2d {

namespace {

constexpr double kTinyD = 2.2250738585072014e-308;   // Fortran tiny(1.0_dp)

__device__ __forceinline__ double ldT(const Fld64& F, int s) { return __ldcg(F.T + s); }
__device__ __forceinline__ double2 ldG(const Fld64& F, int s) { return __ldcg(F.G + s); }
__device__ __forceinline__ uint8_t ldF(const Fld64& F, int s) {
  return (uint8_t)__ldcg(reinterpret_cast<const unsigned char*>(F.fl) + s);
}
__device__ __forceinline__ double xg(const Fld64& F, int col) { return F.x0 + (double)col * F.dx; }
__device__ __forceinline__ double zg(const Fld64& F, int brow) {
  return (double)(F.z_lo + brow) * F.dx;
}
// ---------------------------------------------------------------- candidates
struct Cand {
  double t, trig, gx, gz;
  int ord;
  bool sus, copy;
};

__device__ __forceinline__ Cand no_cand() {
  Cand c;
  c.t = kHugeD; c.trig = kHugeD; c.gx = 0.0; c.gz = 0.0; c.ord = 0x7fffffff;
  c.sus = false; c.copy = false;
  return c;
}

__device__ __forceinline__ bool earlier(double trig, int ord, const Cand& b) {
  return trig < b.trig || (trig == b.trig && ord < b.ord);
}

__device__ __forceinline__ void take(Cand& best, double t, double trig, int ord, double gx,
                                     double gz, bool sus, bool copy) {
  if (t < best.t || (t == best.t && earlier(trig, ord, best))) {
    best.t = t; best.trig = trig; best.ord = ord; best.gx = gx; best.gz = gz;
    best.sus = sus; best.copy = copy;
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
__device__ void rnb4(const Fld64& F, int r, int c, double vu, RNb* n) {
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
  uint32_t k1[4], k2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    k1[k] = b1[k] ? __ldg(F.code + s1[k]) : 0u;
    k2[k] = b2[k] ? __ldg(F.code + s2[k]) : 0u;
  }
  double t1[4], t2[4], v1[4], v2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    b1[k] = b1[k] && (k1[k] & kInRegion);
    b2[k] = b2[k] && (k2[k] & kInRegion);
    t1[k] = b1[k] ? ldT(F, s1[k]) : kHugeD;
    v1[k] = b1[k] ? __ldg(F.vel + s1[k]) : 0.0;
    t2[k] = b2[k] ? ldT(F, s2[k]) : kHugeD;
    v2[k] = b2[k] ? __ldg(F.vel + s2[k]) : 0.0;
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
  double2 g1[4], g2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    g1[k] = need[k] ? ldG(F, s1[k]) : make_double2(0.0, 0.0);
    g2[k] = need[k] ? ldG(F, s2[k]) : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (need[k] && g1[k].x * g2[k].x + g1[k].y * g2[k].y >= 0.71 / (v1[k] * v2[k])) {
      n[k].second = true;
      n[k].T2 = t2[k];
    }
  }
}

// regular_update2d (:605-790) for one or two accepted neighbours.
__device__ bool reg_cand(const RNb* p, const RNb* q, double& t1, double& gx, double& gz,
                         bool& sus) {
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
  t1 = 0.5 * (-b + sqrt(det)) / a;
  t1 = fmax(t1, tmax);
  gx = 0.0;
  gz = 0.0;
  if (xi) gx = (t2x == 0.0) ? (t1 - tx) / dpx : 0.5 * (3.0 * t1 - 4.0 * tx + t2x) / dpx;
  if (zi) gz = (t2z == 0.0) ? (t1 - tz) / dpz : 0.5 * (3.0 * t1 - 4.0 * tz + t2z) / dpz;
  sus = !(xi && zi);
  return true;
}

// Candidates of one regular quadrant (X along x, Z along z): the one-sided
// update of the earlier neighbour (triggered while the other was not yet
// accepted) and the two-sided update (triggered by the later one).
__device__ void quadrant(const RNb& X, const RNb& Z, int ord, Cand& best) {
  double t, gx, gz;
  bool sus;
  if (X.ok && Z.ok) {
    const bool xlow = X.T <= Z.T;
    const RNb& lo = xlow ? X : Z;
    if (lo.single_ok && reg_cand(&lo, nullptr, t, gx, gz, sus))
      take(best, t, lo.T, ord, gx, gz, sus, false);
    if (reg_cand(&X, &Z, t, gx, gz, sus)) take(best, t, fmax(X.T, Z.T), ord, gx, gz, sus, false);
  } else if (X.ok) {
    if (X.single_ok && reg_cand(&X, nullptr, t, gx, gz, sus)) take(best, t, X.T, ord, gx, gz, sus, false);
  } else if (Z.ok) {
    if (Z.single_ok && reg_cand(&Z, nullptr, t, gx, gz, sus)) take(best, t, Z.T, ord, gx, gz, sus, false);
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

__device__ __forceinline__ void offer(CutAcc& A, double t, double trig, int ord, double gx,
                                      double gz, bool copy) {
  take(A.best, t, trig, ord, gx, gz, false, copy);
  if (trig < A.rtrig || (trig == A.rtrig && ord < A.rord)) A.pre_min = fmin(A.pre_min, t);
}

// time_from_1_node2d (:793-829).  A member closer than 0.01*tolerance hands
// its values over ("copy"); a copy is only taken from a member whose own value
// is not a copy, which is what the heap's acceptance order guarantees for
// coincident nodes.
__device__ void from_1(const Mem& a, double xu, double zu, double vu, double tol, double trig,
                       int ord, CutAcc& A) {
  const double dxu = xu - a.x, dzu = zu - a.z;
  const double dist = sqrt(dxu * dxu + dzu * dzu);
  if (dist < 0.01 * tol) {
    if (!a.copied) offer(A, a.T, trig, ord, a.gx, a.gz, true);
    return;
  }
  const double tt = dist / (0.5 * (vu + a.v));
  const double at = a.T + tt;
  offer(A, at, trig, ord, dxu / (dist * vu), dzu / (dist * vu), false);
}

// time_from_2_nodes2d (:832-946): planar front through the trigger n1 and an
// earlier member n2.
__device__ void from_2(const Mem& n1, const Mem& n2, double xu, double zu, double vu, double tol,
                       int ord, CutAcc& A) {
  const double trig = n1.T;
  const double r1x = n1.x - xu, r1z = n1.z - zu;
  const double r2x = n2.x - xu, r2z = n2.z - zu;
  if (sqrt(r1x * r1x + r1z * r1z) < 0.01 * tol) {
    if (!n1.copied) offer(A, n1.T, trig, ord, n1.gx, n1.gz, true);
    return;
  }
  if (sqrt(r2x * r2x + r2z * r2z) < 0.01 * tol) {
    if (!n2.copied) offer(A, n2.T, trig, ord, n2.gx, n2.gz, true);
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
        const double wl = sqrt(wx * wx + wz * wz);
        offer(A, at, trig, ord, wx / (wl * n1.v), wz / (wl * n1.v), false);
      }
    }
  }
}

// Every event of one cut cell.  Members are listed in the reference's
// connected-node order.  When member p is accepted the cell's list holds the
// members accepted by then (p included) in that order; update_time2d swaps p
// to the front and calls time_from_1 (p), then time_from_2 (p, list[k]) for
// k = 1.. of the swapped list.
__device__ void cut_cell(const Mem* m, int nm, double xu, double zu, double vu, double tol,
                         int cbase, CutAcc& A) {
  for (int p = 0; p < nm; ++p) {
    if (!m[p].single_ok) continue;
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
}

__device__ __forceinline__ bool member_at(const Fld64& F, int brow, int col, Mem& m) {
  if (brow < 0 || brow >= F.H || col < 0 || col >= F.nx) return false;
  const int s = brow * F.pitch + col;
  if (!(__ldg(F.code + s) & kInRegion)) return false;
  const double T = ldT(F, s);
  if (!(T < kReachD)) return false;
  const double2 g = ldG(F, s);
  m.x = xg(F, col);
  m.z = zg(F, brow);
  m.T = T;
  m.gx = g.x;
  m.gz = g.y;
  m.v = __ldg(F.vel + s);
  m.single_ok = s != F.frozen_slot;
  m.copied = (ldF(F, s) & kFlCopy) != 0;
  return true;
}

__device__ __forceinline__ bool member_iface(const Fld64& F, int side, int col, Mem& m) {
  if (col < 0 || col >= F.nx) return false;
  const int s = (F.H + side) * F.pitch + col;
  const double T = ldT(F, s);
  if (!(T < kReachD)) return false;
  const double2 g = ldG(F, s);
  m.x = __ldg(F.ifx + col);
  m.z = __ldg(F.ifz + side * F.pitch + col);
  m.T = T;
  m.gx = g.x;
  m.gz = g.y;
  m.v = __ldg(F.vel + s);
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
__device__ NewV finish(const Fld64& F, int s, const Cand& w, bool sus, double sus_t) {
  NewV o;
  o.write = false;
  o.spread = false;
  double T = w.t < kReachD ? w.t : kHugeD, gx = w.gx, gz = w.gz;
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
  auto same = [](double a, double b) { return __double_as_longlong(a) == __double_as_longlong(b); };
  const bool gchg = !same(T, curT) || !same(gx, cg.x) || !same(gz, cg.y) ||
                    cp != ((fl & kFlCopy) != 0);
  o.T = T; o.gx = gx; o.gz = gz; o.sus = su; o.copy = cp;
  o.spread = gchg;
  o.write = gchg || su != ((fl & kFlSusp) != 0);
  return o;
}

// Update of the grid node at bbox row r, column c.
__device__ NewV update_grid(const Fld64& F, int r, int c) {
  NewV none;
  none.write = false;
  none.spread = false;
  const int s = r * F.pitch + c;
  const uint32_t code = __ldg(F.code + s);
  if (!(code & kInRegion) || !(code & kUpdatable) || s == F.frozen_slot) return none;
  const double vu = __ldg(F.vel + s);
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
    const int ci = r - ((q & 1) ? 1 : 0), cj = c - (q >= 2 ? 1 : 0);
    Mem m[6];
    int nm = 0;
    if ((code & (1u << (12 + q))) && member_iface(F, 0, cj, m[nm])) ++nm;
    if ((code & (1u << (16 + q))) && member_iface(F, 1, cj, m[nm])) ++nm;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b) {
        const int rr = ci + b, cc = cj + a;
        if (rr == r && cc == c) continue;
        if (member_at(F, rr, cc, m[nm])) ++nm;
      }
    cut_cell(m, nm, xu, zu, vu, F.tol, q * 32, A);
  }
  const bool reg_wins = rb.t < A.best.t || (rb.t == A.best.t && earlier(rb.trig, rb.ord, A.best));
  const Cand& w = reg_wins ? rb : A.best;
  const bool sus = rb.sus && (reg_wins || rb.t < A.pre_min);
  return finish(F, s, w, sus, rb.t);
}

// Update of interface node `col` on side 0 (top) or 1 (bottom).
__device__ NewV update_iface(const Fld64& F, int side, int col) {
  NewV none;
  none.write = false;
  none.spread = false;
  const int s = (F.H + side) * F.pitch + col;
  const uint32_t code = __ldg(F.code + s);
  if (!(code & kInRegion) || !(code & kUpdatable)) return none;
  const int izc = __ldg(F.izc + side * F.pitch + col);
  if (izc < 0) return none;
  const double vu = __ldg(F.vel + s);
  const double xu = __ldg(F.ifx + col), zu = __ldg(F.ifz + side * F.pitch + col);
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

// ---------------------------------------------------------------- active list
// Nodes whose inputs changed sit in a list of global node ids (a field's
// first id plus its slot); one bit per node says "queued" so a node is listed
// at most once.  Appends are staged per warp in shared memory and flushed
// with one atomic per warp.
constexpr int kQWarps = 8;       // warps per block of the step kernel
constexpr int kQBuf = 256;       // staged appends per warp

struct Queue {
  unsigned* inq;                 // bitset over global node ids
  unsigned* out;                 // list being built
  unsigned* out_cnt;
  unsigned* sbuf;                // shared: this warp's staged appends
  unsigned* scnt;                // shared: their count
  unsigned* ver = nullptr;       // input version per node (bumped when a node it reads changes)
};

// Input version of a node, read before its inputs (acquire: a writer bumps it
// after a fence that follows its write).
__device__ __forceinline__ unsigned ld_ver(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Append a node that this thread has just marked queued.
__device__ __forceinline__ void stage_id(const Queue& q, unsigned gid) {
  const unsigned p = atomicAdd(q.scnt, 1u);
  if (p < (unsigned)kQBuf) {
    q.sbuf[p] = gid;
  } else {
    q.out[atomicAdd(q.out_cnt, 1u)] = gid;
  }
}

__device__ __forceinline__ void push_id(const Queue& q, unsigned gid) {
  const unsigned bit = 1u << (gid & 31);
  if (atomicOr(q.inq + (gid >> 5), bit) & bit) return;   // already queued
  const unsigned p = atomicAdd(q.scnt, 1u);
  if (p < (unsigned)kQBuf) {
    q.sbuf[p] = gid;
  } else {
    q.out[atomicAdd(q.out_cnt, 1u)] = gid;
  }
}

// Flush a warp's staged appends (all lanes).
__device__ __forceinline__ void flush(const Queue& q) {
  __syncwarp();
  const unsigned n = min(*q.scnt, (unsigned)kQBuf);
  unsigned base = 0;
  if ((threadIdx.x & 31) == 0 && n) base = atomicAdd(q.out_cnt, n);
  base = __shfl_sync(0xffffffffu, base, 0);
  for (unsigned k = threadIdx.x & 31; k < n; k += 32) q.out[base + k] = q.sbuf[k];
  __syncwarp();
  if ((threadIdx.x & 31) == 0) *q.scnt = 0u;
  __syncwarp();
}

// Every candidate of a node u that involves node n (as a member, a neighbour
// or a second-order neighbour) is at or above n's time, so a change of n
// from time a to b can only move nodes whose time is at or above min(a, b).
// thr is that bound; nodes stored below it are not re-queued.  Their input
// version moves all the same: a deferred node's stored time is not the one
// it waits with, so its record must not outlive the change.
__device__ __forceinline__ void queue_grid(const Fld64& F, const Queue& q, int r, int c,
                                           double thr) {
  if (r < 0 || r >= F.H || c < 0 || c >= F.nx) return;
  const int s = r * F.pitch + c;
  if (!(__ldg(F.code + s) & kInRegion)) return;
  if (q.ver) atomicAdd(q.ver + F.gbase + s, 1u);
  if (ldT(F, s) < thr) return;
  push_id(q, F.gbase + (unsigned)s);
}

__device__ __forceinline__ void queue_iface(const Fld64& F, const Queue& q, int side, int c,
                                            double thr) {
  if (c < 0 || c >= F.nx) return;
  const int s = (F.H + side) * F.pitch + c;
  if (q.ver) atomicAdd(q.ver + F.gbase + s, 1u);
  if (ldT(F, s) < thr) return;
  push_id(q, F.gbase + (unsigned)s);
}

// Nodes whose candidates read grid node (r, c): its direct, second and
// diagonal neighbours, and the interface nodes of the cut cells it is a
// corner of.
__device__ void spread_grid(const Fld64& F, const Queue& q, int r, int c, double thr) {
  // The targets' loads and atomics are issued in batches (independent of one
  // another), so the latency is paid a few times instead of once per target.
  // Grid targets: the second neighbours along the axes and the 3x3 block.
  constexpr int kN = 12;
  const int dr[kN] = {-2, 2, 0, 0, -1, -1, -1, 0, 0, 1, 1, 1};
  const int dc[kN] = {0, 0, -2, 2, -1, 0, 1, -1, 1, -1, 0, 1};
  int sl[kN];
  bool ok[kN];
#pragma unroll
  for (int k = 0; k < kN; ++k) {
    const int rr = r + dr[k], cc = c + dc[k];
    ok[k] = rr >= 0 && rr < F.H && cc >= 0 && cc < F.nx;
    sl[k] = ok[k] ? rr * F.pitch + cc : 0;
  }
  uint32_t code[kN];
#pragma unroll
  for (int k = 0; k < kN; ++k) code[k] = ok[k] ? __ldg(F.code + sl[k]) : 0u;
#pragma unroll
  for (int k = 0; k < kN; ++k) ok[k] = ok[k] && (code[k] & kInRegion);
  double tv[kN];
#pragma unroll
  for (int k = 0; k < kN; ++k) tv[k] = ok[k] ? ldT(F, sl[k]) : 0.0;
  if (q.ver) {
#pragma unroll
    for (int k = 0; k < kN; ++k)
      if (ok[k]) atomicAdd(q.ver + F.gbase + sl[k], 1u);
  }
  unsigned was[kN];
#pragma unroll
  for (int k = 0; k < kN; ++k) {
    ok[k] = ok[k] && !(tv[k] < thr);
    const unsigned gid = F.gbase + (unsigned)sl[k];
    was[k] = ok[k] ? atomicOr(q.inq + (gid >> 5), 1u << (gid & 31)) : 0u;
  }
#pragma unroll
  for (int k = 0; k < kN; ++k) {
    const unsigned gid = F.gbase + (unsigned)sl[k];
    if (ok[k] && !(was[k] & (1u << (gid & 31)))) stage_id(q, gid);
  }
  // interface nodes of the cut cells (r, c) is a corner of
  const int ar = F.z_lo + r;
  int isl[4];
  bool iok[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int side = k >> 1, kc = c - 1 + (k & 1);
    iok[k] = kc >= 0 && kc < F.nx;
    const int izc = iok[k] ? __ldg(F.izc + side * F.pitch + kc) : -1;
    iok[k] = iok[k] && izc >= 0 && (izc == ar || izc + 1 == ar);
    isl[k] = iok[k] ? (F.H + side) * F.pitch + kc : 0;
  }
  double itv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) itv[k] = iok[k] ? ldT(F, isl[k]) : 0.0;
  if (q.ver) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (iok[k]) atomicAdd(q.ver + F.gbase + isl[k], 1u);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (iok[k] && !(itv[k] < thr)) push_id(q, F.gbase + (unsigned)isl[k]);
}

__device__ void spread_iface(const Fld64& F, const Queue& q, int side, int c, double thr) {
  const int izc = __ldg(F.izc + side * F.pitch + c);
  if (izc >= 0) {
    const int br = izc - F.z_lo;
    queue_grid(F, q, br, c, thr);
    queue_grid(F, q, br + 1, c, thr);
    queue_grid(F, q, br, c + 1, thr);
    queue_grid(F, q, br + 1, c + 1, thr);
  }
  queue_iface(F, q, side ^ 1, c, thr);
}

__device__ __forceinline__ int find_field(const Fld64* f, int nf, unsigned gid) {
  int lo = 0, hi = nf - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (f[mid].gbase <= gid) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Evaluate node `slot` of field F (grid row or interface row).
__device__ __forceinline__ NewV evaluate(const Fld64& F, int slot) {
  const int row = slot / F.pitch, col = slot - (slot / F.pitch) * F.pitch;
  if (row < F.H) return update_grid(F, row, col);
  return update_iface(F, row - F.H, col);
}

__device__ __forceinline__ void spread(const Fld64& F, const Queue& q, int slot, double thr) {
  const int row = slot / F.pitch, col = slot - (slot / F.pitch) * F.pitch;
  if (row < F.H) spread_grid(F, q, row, col, thr);
  else spread_iface(F, q, row - F.H, col, thr);
}

// One step: every listed node is evaluated once (a thread per node).  A new
// time inside the field's window is written and the nodes it can move are
// queued; one beyond the window is deferred (the node re-queues itself and
// records the time with the input version it was computed from, so that
// until the window reaches that time or an input changes, listing it costs
// a compare instead of an evaluation).  The last block to finish moves on
// the window of every field in which nothing changed during the step.  A
// window may take many steps to settle (a front nearly parallel to a grid
// line puts a whole line of nodes, each waiting for the next, into one
// window); moving it earlier would accept times that are not final.
// ctr: [0] evaluations, [1] writes, [2] deferred nodes passed over.

__global__ void __launch_bounds__(32 * kQWarps) k_step(Fld64* fields, int nf, const unsigned* in,
                                                       const unsigned* in_cnt, unsigned* out,
                                                       unsigned* out_cnt, unsigned* zero_cnt,
                                                       unsigned* inq, unsigned* done,
                                                       unsigned* ver, unsigned long long* pend,
                                                       unsigned long long* ctr) {
  __shared__ unsigned s_buf[kQWarps][kQBuf];
  __shared__ unsigned s_cnt[kQWarps];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (lane == 0) s_cnt[wib] = 0u;
  __syncwarp();
  Queue q;
  q.inq = inq;
  q.out = out;
  q.out_cnt = out_cnt;
  q.sbuf = s_buf[wib];
  q.scnt = s_cnt + wib;
  q.ver = ver;
  const unsigned n = __ldcg(in_cnt);
  const unsigned warp = blockIdx.x * kQWarps + wib, nwarp = gridDim.x * kQWarps;
  unsigned long long n_eval = 0, n_write = 0, n_pass = 0;
  for (unsigned base = warp * 32; base < n; base += nwarp * 32) {
    const unsigned i = base + lane;
    if (i < n) {
      const unsigned gid = in[i];
      const int fi = find_field(fields, nf, gid);
      const Fld64& F = fields[fi];
      const int slot = (int)(gid - F.gbase);
      atomicAnd(inq + (gid >> 5), ~(1u << (gid & 31)));   // listed again if moved meanwhile
      const unsigned v0 = ld_ver(ver + gid);
      const unsigned long long rec = __ldcg(pend + gid);
      const double wend = __ldcg(F.clock);
      if ((unsigned)(rec >> 32) == v0 && (double)__uint_as_float((unsigned)rec) > wend) {
        push_id(q, gid);   // still beyond the window, inputs unchanged
        ++n_pass;
      } else {
        const NewV nv = evaluate(F, slot);
        ++n_eval;
        if (nv.write) {
          const double oldT = F.T[slot];
          if (nv.T < kReachD && nv.T > wend) {
            // beyond the window: wait for it (the time rounded down, so the
            // compare above never passes over a node the window has reached)
            pend[gid] = ((unsigned long long)v0 << 32) |
                        (unsigned long long)__float_as_uint(__double2float_rd(nv.T));
            push_id(q, gid);
          } else {
            F.T[slot] = nv.T;
            F.G[slot] = make_double2(nv.gx, nv.gz);
            F.fl[slot] = (uint8_t)((F.fl[slot] & kFlSeed) | (nv.copy ? kFlCopy : 0) |
                                   (nv.sus ? kFlSusp : 0));
            if (nv.spread) {
              ++n_write;
              F.clock[2] = 1.0;   // the window is not settled
              __threadfence();
              spread(F, q, slot, fmin(oldT, nv.T));
            }
          }
        }
      }
    }
    flush(q);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    n_eval += __shfl_xor_sync(0xffffffffu, n_eval, o);
    n_write += __shfl_xor_sync(0xffffffffu, n_write, o);
    n_pass += __shfl_xor_sync(0xffffffffu, n_pass, o);
  }
  if (lane == 0 && ctr && (n_eval || n_pass)) {
    atomicAdd(ctr + 0, n_eval);
    atomicAdd(ctr + 1, n_write);
    atomicAdd(ctr + 2, n_pass);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
      double* c = fields[f].clock;
      if (__ldcg(c + 2) == 0.0) c[0] = __ldcg(c) + __ldcg(c + 1);
      c[2] = 0.0;
    }
    if (threadIdx.x == 0) {
      *zero_cnt = 0u;   // the list after next starts empty
      *done = 0u;
    }
  }
}

// Fixed-point check of every node (window ignored): a node whose update
// would change it is queued and counted.
__global__ void __launch_bounds__(32 * kQWarps) k_verify(Fld64* fields, int nf, unsigned* out,
                                                         unsigned* out_cnt, unsigned* inq,
                                                         unsigned* bad) {
  __shared__ unsigned s_buf[kQWarps][kQBuf];
  __shared__ unsigned s_cnt[kQWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (lane == 0) s_cnt[wib] = 0u;
  __syncwarp();
  Queue q;
  q.inq = inq;
  q.out = out;
  q.out_cnt = out_cnt;
  q.sbuf = s_buf[wib];
  q.scnt = s_cnt + wib;
  Fld64& F = fields[blockIdx.y];
  const int ns = (F.H + 2) * F.pitch;
  unsigned nbad = 0;
  for (int base = (blockIdx.x * kQWarps + wib) * 32; base < ns; base += gridDim.x * kQWarps * 32) {
    const int s = base + lane;
    if (s < ns && (s % F.pitch) < F.nx) {
      const NewV nv = evaluate(F, s);
      if (nv.write) {
        ++nbad;
        push_id(q, F.gbase + (unsigned)s);
      }
    }
    flush(q);
  }
  if (nbad) atomicAdd(bad, nbad);
}

// Queue every seeded node and the nodes around it.
__global__ void __launch_bounds__(32 * kQWarps) k_queue_seeds(Fld64* fields, int nf, unsigned* out,
                                                              unsigned* out_cnt, unsigned* inq) {
  __shared__ unsigned s_buf[kQWarps][kQBuf];
  __shared__ unsigned s_cnt[kQWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (lane == 0) s_cnt[wib] = 0u;
  __syncwarp();
  Queue q;
  q.inq = inq;
  q.out = out;
  q.out_cnt = out_cnt;
  q.sbuf = s_buf[wib];
  q.scnt = s_cnt + wib;
  Fld64& F = fields[blockIdx.y];
  const int ns = (F.H + 2) * F.pitch;
  for (int base = (blockIdx.x * kQWarps + wib) * 32; base < ns; base += gridDim.x * kQWarps * 32) {
    const int s = base + lane;
    if (s < ns && (s % F.pitch) < F.nx && (F.fl[s] & kFlSeed)) {
      push_id(q, F.gbase + (unsigned)s);
      spread(F, q, s, -kHugeD);
    }
    flush(q);
  }
}

// ---------------------------------------------------------------- seeding
__global__ void k_fill(Fld64* fields, int nf) {
  Fld64& F = fields[blockIdx.y];
  const size_t ns = (size_t)(F.H + 2) * F.pitch;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns;
       i += (size_t)gridDim.x * blockDim.x) {
    F.T[i] = kHugeD;
    F.G[i] = make_double2(0.0, 0.0);
    F.Gout[i] = make_double2(0.0, 0.0);
    F.seed[i] = make_double4(kHugeD, 0.0, 0.0, 0.0);
    F.fl[i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) F.frozen_slot = -1;
}

__device__ void put_seed(Fld64& F, int s, double t, double gx, double gz) {
  F.T[s] = t;
  F.G[s] = make_double2(gx, gz);
  F.seed[s] = make_double4(t, gx, gz, 0.0);
  F.fl[s] = kFlSeed;
}

// initialize_region_from_source2d (:2307-2411): the corners of the source
// cell get dist/v and the straight-ray gradient; a corner within
// 0.01*tolerance takes t0 = 0 and stays fixed.
__global__ void k_init_source(Fld64* fields, const double* sx, const double* sz, int nf) {
  const int fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi >= nf) return;
  Fld64& F = fields[fi];
  const double h = F.dx;
  int ix0 = (int)floor((sx[fi] - F.x0) / h);
  int iz0 = (int)floor((sz[fi] - 0.0) / h);
  ix0 = max(0, min(F.nx - 2, ix0));
  iz0 = max(0, min(F.nz - 2, iz0));
  for (int ix = ix0; ix <= ix0 + 1; ++ix)
    for (int iz = iz0; iz <= iz0 + 1; ++iz) {
      const int br = iz - F.z_lo;
      if (br < 0 || br >= F.H) continue;
      const int s = br * F.pitch + ix;
      if (!(F.code[s] & kInRegion)) continue;
      const double ddx = (F.x0 + ix * h) - sx[fi], ddz = iz * h - sz[fi];
      const double dist = sqrt(ddx * ddx + ddz * ddz);
      double v = F.vel[s];
      if (v < 0.01) v = 0.01;
      if (dist < 0.01 * F.tol) {
        put_seed(F, s, 0.0, 0.0, 0.0);
        F.frozen_slot = s;
      } else {
        const double t = dist / v;
        put_seed(F, s, t, ddx / (dist * v), ddz / (dist * v));
      }
    }
}

// Interface hand-off of a stage (transfer_times_to_intersection :2414-2554,
// reflect_gradient_at_interface :2632-2741, sweep_region_from_interface2d
// :1982-2304): the target region's interface nodes take the parent's
// boundary time and gradient (normal slowness rebuilt on the target side when
// reflecting), grid nodes up to three rows into the region take
// T_if + dist/v from the first interface node whose box holds them.
__global__ void k_seed_iface(Fld64* fields, const Seed64* descs, int nd, int nx) {
  const Seed64& D = descs[blockIdx.y];
  Fld64& F = fields[D.dst];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= F.nx) return;
  const double h = F.dx;
  auto iface_val = [&](int k, double& T, double& gx, double& gz) {
    const int ss = D.src_row * D.src_pitch + k;
    T = D.src_T[ss];
    const double2 g = D.src_G[ss];
    gx = g.x;
    gz = g.y;
    if (T >= kReachD) { T = kHugeD; }
    if (!D.reflect) return;
    if (T >= kReachD) { gx = 0.0; gz = 0.0; return; }
    const double nx_ = D.ifc.nrm_x[k], nz_ = D.ifc.nrm_z[k];
    const double gp = gx * nx_ + gz * nz_;
    const double px = gx - gp * nx_, pz = gz - gp * nz_;
    const int side = D.target_side;
    double v = side > 0 ? D.ifc.vel_bot[k] : D.ifc.vel_top[k];
    if (!(v > 0.01)) v = F.vel[(F.H + D.dst_side) * F.pitch + k];
    if (v <= 0.01) { T = kHugeD; gx = 0.0; gz = 0.0; return; }
    const double pn2 = 1.0 / (v * v) - (px * px + pz * pz);
    if (pn2 < -1.0e-10) { T = kHugeD; gx = 0.0; gz = 0.0; return; }
    const double pn = sqrt(pn2 < 0.0 ? 0.0 : pn2);
    gx = px + side * pn * nx_;
    gz = pz + side * pn * nz_;
  };
  double T, gx, gz;
  iface_val(c, T, gx, gz);
  {
    const int s = (F.H + D.dst_side) * F.pitch + c;
    put_seed(F, s, T, gx, gz);
  }
  int done[9], ndone = 0;
  for (int n = c - 1; n <= c + 1; ++n) {
    if (n < 0 || n >= nx) continue;
    const int izf = D.ifc.izc[n];
    if (izf < 0) continue;
    int r_a, r_b, st;
    if (D.dst_side == 1) { r_a = izf; r_b = max(0, izf - 2); st = -1; }
    else { r_a = izf + 1; r_b = min(F.nz - 1, izf + 3); st = 1; }
    double Tn, gxn, gzn;
    iface_val(n, Tn, gxn, gzn);
    const double xm = F.ifx[n], zm = D.ifc.z[n];
    for (int r = r_a; st > 0 ? r <= r_b : r >= r_b; r += st) {
      if (r < D.r0[c] || r > D.r1[c]) continue;
      bool seen = false;
      for (int q = 0; q < ndone; ++q) seen = seen || (done[q] == r);
      if (seen) continue;
      done[ndone++] = r;
      const int br = r - F.z_lo;
      const int s = br * F.pitch + c;
      const double ddx = (F.x0 + c * h) - xm, ddz = r * h - zm;
      const double dist = sqrt(ddx * ddx + ddz * ddz);
      double v = F.vel[s];
      if (v < 0.01) v = 0.01;
      const double tn = Tn >= kReachD ? kHugeD : Tn + dist / v;
      put_seed(F, s, tn, ddx / (dist * v), ddz / (dist * v));
    }
  }
}

// Window of each field: from its earliest seed, advancing by step[f].
__global__ void k_clock(Fld64* fields, int nf, const double* step) {
  Fld64& F = fields[blockIdx.x];
  const int ns = (F.H + 2) * F.pitch;
  double mn = kHugeD;
  for (int s = threadIdx.x; s < ns; s += blockDim.x)
    if (F.fl[s] & kFlSeed) mn = fmin(mn, F.T[s]);
  __shared__ double sm[32];
#pragma unroll
  for (int o = 16; o; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mn;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mn = fmin(mn, sm[w]);
    const double t0 = mn < kReachD ? mn : 0.0;
    F.clock[1] = step[blockIdx.x];
    F.clock[0] = t0 + step[blockIdx.x];
    F.clock[2] = 1.0;
  }
}

// ---------------------------------------------------------------- post-processing
// fit_gradient_at_node2d (:949-1196): central differences in a regular
// neighbourhood, else a distance-weighted 2x2 least-squares fit over the
// nodes of the connected cells.
__device__ void fit_grad(const Fld64& F, int slot, double& dtdx, double& dtdz) {
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
// (propagate2d.f90:119-123).
__global__ void k_final_grad(Fld64* fields, int nf) {
  Fld64& F = fields[blockIdx.y];
  const size_t ns = (size_t)(F.H + 2) * F.pitch;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns;
       i += (size_t)gridDim.x * blockDim.x) {
    if (!(F.code[i] & kInRegion)) continue;
    if ((F.fl[i] & kFlSusp) && F.T[i] < kReachD) {
      double gx, gz;
      fit_grad(F, (int)i, gx, gz);
      F.Gout[i] = make_double2(gx, gz);
    } else {
      F.Gout[i] = F.G[i];
    }
  }
}

// Top-row gradient fix of the water-layer fields (inversion2d.f90:4264-4292):
// upward = 1 requires dT/dz < 0 at the sea surface, upward = 0 requires > 0.
__global__ void k_water_fix(Fld64* fields, const int* upward, int nf) {
  const int fi = blockIdx.y;
  Fld64& F = fields[fi];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= F.nx || upward[fi] < 0) return;
  const int bt = 0 - F.z_lo, bb = 1 - F.z_lo;
  if (bt < 0 || bb >= F.H) return;
  const int st = bt * F.pitch + c, sb = bb * F.pitch + c;
  if (!(F.code[st] & kInRegion) || !(F.code[sb] & kInRegion)) return;
  const double gz = F.Gout[st].y;
  const bool bad = upward[fi] ? (gz > 0.0 || fabs(gz) < 0.01) : (gz < 0.0 || fabs(gz) < 0.01);
  if (bad) F.Gout[st] = F.Gout[sb];
}

// PmP head-wave min-plus sweep along the Moho (inversion2d.f90:4294-4409), one
// field per thread; node table and velocities are precomputed per model.
__global__ void k_headwave(Fld64* fields, const int* hw_slot, const double* hw_v, double dx_if,
                           int nx, double* scratch, const int* which, int nsel) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsel) return;
  Fld64& F = fields[which[q]];
  double* th = scratch + (size_t)q * nx;
  for (int n = 0; n < nx; ++n) th[n] = hw_slot[n] >= 0 ? F.T[hw_slot[n]] : kHugeD;
  for (int n = 1; n < nx; ++n)
    if (hw_v[n] > 0.0) th[n] = fmin(th[n], th[n - 1] + dx_if / hw_v[n]);
  for (int n = nx - 2; n >= 0; --n)
    if (hw_v[n] > 0.0) th[n] = fmin(th[n], th[n + 1] + dx_if / hw_v[n]);
  for (int n = 0; n < nx; ++n) {
    const int s = hw_slot[n];
    if (s < 0) continue;
    if (th[n] < F.T[s] - 1.0e-10) F.T[s] = th[n];
  }
  for (int n = 0; n < nx; ++n) {
    const int s = hw_slot[n];
    if (s < 0 || F.T[s] >= kReachD) continue;
    if (!(F.code[s] & kIfaceNode)) {
      double gx, gz;
      fit_grad(F, s, gx, gz);
      F.Gout[s] = make_double2(gx, gz);
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
      F.Gout[s] = make_double2(dtdx, dtdz);
    }
  }
}

__global__ void k_export(const double* T, const double2* G, const int* slot_of_node, int nnode,
                         double* oT, double* ogx, double* ogz) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nnode; n += gridDim.x * blockDim.x) {
    const int s = slot_of_node[n];
    if (oT) oT[n] = T[s];
    const double2 g = G[s];
    if (ogx) ogx[n] = g.x;
    if (ogz) ogz[n] = g.y;
  }
}

}  // namespace

// ---------------------------------------------------------------- launchers
void e64_fill(Fld64* f, int nf, size_t max_slots, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 1024);
  k_fill<<<dim3(bx, nf), 256, 0, st>>>(f, nf);
}
void e64_init_source(Fld64* f, const double* sx, const double* sz, int nf, cudaStream_t st) {
  k_init_source<<<(nf + 63) / 64, 64, 0, st>>>(f, sx, sz, nf);
}
void e64_seed_iface(Fld64* f, const Seed64* d, int nd, int nx, cudaStream_t st) {
  k_seed_iface<<<dim3((nx + 127) / 128, nd), 128, 0, st>>>(f, d, nd, nx);
}
void e64_start(Fld64* f, int nf, size_t max_slots, const double* step, unsigned* list,
               unsigned* cnt, unsigned* inq, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 32 * kQWarps - 1) / (32 * kQWarps), 256);
  k_queue_seeds<<<dim3(bx, nf), 32 * kQWarps, 0, st>>>(f, nf, list, cnt, inq);
  k_clock<<<nf, 256, 0, st>>>(f, nf, step);
}
void e64_step(Fld64* f, int nf, const unsigned* in, const unsigned* in_cnt, unsigned* out,
              unsigned* out_cnt, unsigned* zero_cnt, unsigned* inq, unsigned* done, unsigned* ver,
              unsigned long long* pend, int grid, unsigned long long* ctr, cudaStream_t st) {
  k_step<<<grid, 32 * kQWarps, 0, st>>>(f, nf, in, in_cnt, out, out_cnt, zero_cnt, inq, done, ver,
                                        pend, ctr);
}
void e64_verify(Fld64* f, int nf, size_t max_slots, unsigned* list, unsigned* cnt, unsigned* inq,
                unsigned* bad, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 32 * kQWarps - 1) / (32 * kQWarps), 512);
  k_verify<<<dim3(bx, nf), 32 * kQWarps, 0, st>>>(f, nf, list, cnt, inq, bad);
}
void e64_finish(Fld64* f, int nf, size_t max_slots, const int* water_up, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 512);
  k_final_grad<<<dim3(bx, nf), 256, 0, st>>>(f, nf);
  k_water_fix<<<dim3(64, nf), 128, 0, st>>>(f, water_up, nf);
}
void e64_headwave(Fld64* f, const int* hw_slot, const double* hw_v, double dx_if, int nx,
                  double* scratch, const int* which, int nsel, cudaStream_t st) {
  k_headwave<<<(nsel + 31) / 32, 32, 0, st>>>(f, hw_slot, hw_v, dx_if, nx, scratch, which, nsel);
}
void e64_export(const double* T, const double2* G, const int* slot_of_node, int nnode, double* oT,
                double* ogx, double* ogz, cudaStream_t st) {
  k_export<<<(nnode + 255) / 256, 256, 0, st>>>(T, G, slot_of_node, nnode, oT, ogx, ogz);
}
int e64_step_grid(int device) {
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step, 32 * kQWarps, 0);
  return std::max(1, nsm) * std::max(1, per_sm);
}

}  // namespace fmt2d
