// Discrete adjoint of the eikonal fields: links, reverse sweep, stage
// hand-off, head-wave sweep and the map onto the propagation grid.
//
// A node's link is found by evaluating the node again at the fixed point with
// the solver's own candidate functions (eik_eval.cuh), noting which candidate
// becomes the best, then evaluating that one candidate again in dual numbers
// (value and partial derivatives).  The dual evaluation repeats the
// candidate's expressions in the same order, so its value is the stored time
// bit for bit; a node where it is not is counted (kAdjCtrMismatch) and gets
// no link.  This file is compiled without FMA contraction, like the solver.
//
// Derivatives follow regular_update2d (src/propagate2d.f90:605-790),
// time_from_1_node2d / time_from_2_nodes2d (:793-946), the source corners of
// initialize_region_from_source2d (:2307-2411), the hand-off seeds of
// sweep_region_from_interface2d (:1982-2304) and the PmP head-wave sweep
// (src/inversion2d.f90:4294-4409).
#include "adjoint.cuh"
#define FMT_HD_LINK static
#include "eik_eval.cuh"

namespace fmt2d {

namespace {

using ev::Cand;
using ev::CutAcc;
using ev::Mem;
using ev::RNb;

// ---------------------------------------------------------------- duals
constexpr int kND = 8;   // independent inputs of one candidate

struct Dn {
  double v;
  double d[kND];
};

__device__ inline Dn dconst(double v) {
  Dn r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = 0.0;
  return r;
}
__device__ inline Dn dvar(double v, int k) {
  Dn r = dconst(v);
  if (k >= 0) r.d[k] = 1.0;
  return r;
}
__device__ inline Dn operator+(const Dn& a, const Dn& b) {
  Dn r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
__device__ inline Dn operator-(const Dn& a, const Dn& b) {
  Dn r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
__device__ inline Dn operator-(const Dn& a) {
  Dn r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = -a.d[k];
  return r;
}
__device__ inline Dn operator*(const Dn& a, const Dn& b) {
  Dn r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
__device__ inline Dn operator/(const Dn& a, const Dn& b) {
  Dn r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
__device__ inline Dn operator*(double a, const Dn& b) {
  Dn r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = a * b.d[k];
  return r;
}
__device__ inline Dn operator*(const Dn& a, double b) {
  Dn r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = a.d[k] * b;
  return r;
}
__device__ inline Dn operator/(const Dn& a, double b) {
  Dn r;
  r.v = a.v / b;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = a.d[k] / b;
  return r;
}
__device__ inline Dn operator/(double a, const Dn& b) {
  Dn r;
  r.v = a / b.v;
  const double f = -r.v / b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = f * b.d[k];
  return r;
}
__device__ inline Dn operator+(double a, const Dn& b) {
  Dn r = b;
  r.v = a + b.v;
  return r;
}
__device__ inline Dn operator-(double a, const Dn& b) {
  Dn r;
  r.v = a - b.v;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = -b.d[k];
  return r;
}
__device__ inline Dn operator-(const Dn& a, double b) {
  Dn r = a;
  r.v = a.v - b;
  return r;
}
__device__ inline Dn dsqrt(const Dn& a) {
  Dn r;
  r.v = sqrt(a.v);
  const double f = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
  for (int k = 0; k < kND; ++k) r.d[k] = f * a.d[k];
  return r;
}
// fmax(a, b) for the non-NaN operands the stencil has: the larger; a on ties
__device__ inline Dn dmax(const Dn& a, const Dn& b) { return b.v > a.v ? b : a; }

// Where each dual input comes from: a same-field time (tslot), a slot
// velocity (vslot) or the parent field's time (xslot).
struct Inputs {
  int tslot[kND], vslot[kND], xslot[kND], zkey[kND];
  __device__ void clear() {
#pragma unroll
    for (int k = 0; k < kND; ++k) tslot[k] = vslot[k] = xslot[k] = zkey[k] = -1;
  }
};

// ------------------------------------------------- candidate re-derivation
// A direct neighbour in dual form (rnb4's values for one direction).
struct DNb {
  bool dirx, second;
  Dn T, T2, d2;
};

// regular_update2d for one or two neighbours (ev::reg_cand's expressions).
__device__ bool reg_dual(const DNb* p, const DNb* q, Dn& out) {
  Dn a = dconst(0.0), b = dconst(0.0), c = dconst(0.0), tmax = dconst(0.0);
  for (int k = 0; k < 2; ++k) {
    const DNb* n = k == 0 ? p : q;
    if (!n) continue;
    tmax = dmax(tmax, n->T);
    if (n->second) {
      const Dn tx = n->T, t2x = n->T2;
      a = a + 2.25 * n->d2;
      b = b + (-6.0 * tx + 1.5 * t2x) * n->d2;
      c = c + (4.0 * tx * tx - 2.0 * tx * t2x + 0.25 * t2x * t2x) * n->d2;
    } else {
      const Dn tx = n->T;
      a = a + n->d2;
      b = b + (-2.0 * tx) * n->d2;
      c = c + (tx * tx) * n->d2;
    }
  }
  c = c - 1.0;
  if (fabs(a.v) < ev::kTinyD) return false;
  Dn det = b * b - 4.0 * a * c;
  if (det.v < 0.0) {
    if (0.5 * sqrt(fabs(det.v)) / fabs(a.v) < 1.0e20) det = dconst(0.0);
    else return false;
  }
  const Dn t1 = 0.5 * (-b + dsqrt(det)) / a;
  out = dmax(t1, tmax);
  return true;
}

// time_from_1_node2d (ev::from_1): a copy when the member is within
// 0.01*tolerance, else the member's time plus the straight ray.  Depths az
// (the member) and zu (the node) are inputs: interface nodes move with their
// interface.
__device__ Dn from1_dual(const Mem& a, const Dn& aT, const Dn& av, const Dn& az, double xu,
                         const Dn& zu, const Dn& vu, double tol, bool& offered) {
  const double dxu = xu - a.x;
  const Dn dzu = zu - az;
  const Dn dist = dsqrt(dxu * dxu + dzu * dzu);
  if (dist.v < 0.01 * tol) {
    offered = !a.copied;
    return aT;
  }
  offered = true;
  const Dn tt = dist / (0.5 * (vu + av));
  return aT + tt;
}

// time_from_2_nodes2d (ev::from_2): the first candidate it offers whose
// value is `target` (the one the best-candidate rule kept).
__device__ bool from2_dual(const Mem& n1, const Mem& n2, const Dn& T1, const Dn& T2,
                           const Dn& v1, const Dn& v2, const Dn& z1, const Dn& z2, double xu,
                           const Dn& zu, const Dn& vu, double tol, double target, Dn& out) {
  const double r1x = n1.x - xu;
  const Dn r1z = z1 - zu;
  const double r2x = n2.x - xu;
  const Dn r2z = z2 - zu;
  if (sqrt(r1x * r1x + r1z.v * r1z.v) < 0.01 * tol) {
    out = T1;
    return !n1.copied && out.v == target;
  }
  if (sqrt(r2x * r2x + r2z.v * r2z.v) < 0.01 * tol) {
    out = T2;
    return !n2.copied && out.v == target;
  }
  const double ex = n2.x - n1.x;
  const double ez = z2.v - z1.v;
  if (sqrt(ex * ex + ez * ez) < 0.01 * tol) {
    bool offered = false;
    out = from1_dual(n1, T1, v1, z1, xu, zu, vu, tol, offered);
    return offered && out.v == target;
  }
  const Dn v12 = 0.5 * (v1 + v2);
  const Dn dx_ = (n1.x - n2.x) / v12, dz_ = (z1 - z2) / v12;
  const Dn dd = dx_ * dx_ + dz_ * dz_;
  const Dn px = (T1 - T2) / dd * dx_;
  const Dn pz = (T1 - T2) / dd * dz_;
  const Dn qx = -dz_, qz = dx_;
  const Dn ae = qx * qx + qz * qz;
  const Dn be = 2.0 * (px * qx + pz * qz);
  const Dn ce = px * px + pz * pz - 1.0;
  const Dn det = be * be - 4.0 * ae * ce;
  if (det.v < 0.0) return false;
  const Dn u1 = 0.5 * (-be + dsqrt(det)) / ae;
  const Dn u2 = 0.5 * (-be - dsqrt(det)) / ae;
  double m1x = -r1z.v, m1z = r1x;
  double l = sqrt(m1x * m1x + m1z * m1z);
  m1x /= l;
  m1z /= l;
  if (m1x * r2x + m1z * r2z.v < 0.0) { m1x = -m1x; m1z = -m1z; }
  double m2x = -r2z.v, m2z = r2x;
  l = sqrt(m2x * m2x + m2z * m2z);
  m2x /= l;
  m2z /= l;
  if (m2x * r1x + m2z * r1z.v < 0.0) { m2x = -m2x; m2z = -m2z; }
  for (int k = 0; k < 2; ++k) {
    const Dn& u = k == 0 ? u1 : u2;
    const Dn wx = px + u * qx, wz = pz + u * qz;
    if (wx.v * m1x + wz.v * m1z <= 0.0 && wx.v * m2x + wz.v * m2z <= 0.0) {
      const Dn at = T1 - (wx * r1x + wz * r1z) / (0.5 * (vu + v1));
      if (at.v >= T1.v && at.v == target) {
        out = at;
        return true;
      }
    }
  }
  return false;
}

// ------------------------------------------------ which candidate wins
__device__ inline bool takes(const Cand& best, const Cand& c) {
  return c.t < best.t || (c.t == best.t && ev::earlier(c.trig, c.ord, best));
}
__device__ inline bool changed(const Cand& a, const Cand& b) {
  return a.t != b.t || a.trig != b.trig || a.ord != b.ord;
}

// Identity of the best candidate: a regular quadrant (nb index of its x and
// z neighbours, -1 unused) or a cut-cell event (cell, triggering member p,
// earlier member q of a time_from_2 event).
struct Win {
  int kind = kAdjNone;
  int x = -1, z = -1;
  int cell = -1, p = -1, q = -1;
};

// ev::quadrant, noting the candidate that becomes the best.
__device__ void quad_t(const RNb* nb, int ix, int iz, int ord, Cand& best, Win& w) {
  const RNb& X = nb[ix];
  const RNb& Z = nb[iz];
  Cand c;
  c.ord = ord;
  if (X.ok && Z.ok) {
    const bool xlow = X.T <= Z.T;
    const RNb& lo = xlow ? X : Z;
    if (lo.single_ok && ev::reg_cand(&lo, nullptr, c)) {
      c.trig = lo.T;
      if (takes(best, c)) {
        best = c;
        w = Win();
        w.kind = kAdjRegular;
        if (xlow) w.x = ix; else w.z = iz;
      }
    }
    if (ev::reg_cand(&X, &Z, c)) {
      c.trig = fmax(X.T, Z.T);
      if (takes(best, c)) {
        best = c;
        w = Win();
        w.kind = kAdjRegular;
        w.x = ix;
        w.z = iz;
      }
    }
  } else if (X.ok) {
    if (X.single_ok && ev::reg_cand(&X, nullptr, c)) {
      c.trig = X.T;
      if (takes(best, c)) {
        best = c;
        w = Win();
        w.kind = kAdjRegular;
        w.x = ix;
      }
    }
  } else if (Z.ok) {
    if (Z.single_ok && ev::reg_cand(&Z, nullptr, c)) {
      c.trig = Z.T;
      if (takes(best, c)) {
        best = c;
        w = Win();
        w.kind = kAdjRegular;
        w.z = iz;
      }
    }
  }
}

// ev::cut_member, noting the event that becomes the best.
__device__ void cut_member_t(const Mem* m, int nm, int p, double xu, double zu, double vu,
                             double tol, int cbase, CutAcc& A, int cell, Win& w) {
  if (!m[p].single_ok) return;
  int lst[6], n = 0, pp = 0;
  for (int q = 0; q < nm; ++q) {
    const bool before = q == p || m[q].T < m[p].T || (m[q].T == m[p].T && q < p);
    if (!before) continue;
    if (q == p) pp = n;
    lst[n++] = q;
  }
  Cand b0 = A.best;
  ev::from_1(m[p], xu, zu, vu, tol, m[p].T, cbase, A);
  if (changed(b0, A.best)) {
    w = Win();
    w.kind = kAdjRay;
    w.cell = cell;
    w.p = p;
  }
  for (int k = 1; k < n; ++k) {
    const int q = (k == pp) ? lst[0] : lst[k];
    b0 = A.best;
    ev::from_2(m[p], m[q], xu, zu, vu, tol, cbase + k, A);
    if (changed(b0, A.best)) {
      w = Win();
      w.kind = kAdjPlane;
      w.cell = cell;
      w.p = p;
      w.q = q;
    }
  }
}

// ev::cell_members with the members' slots.
__device__ int cell_members_s(const Fld64& F, int r, int c, uint32_t code, int q, Mem* m,
                              int* ms) {
  const int ci = r - ((q & 1) ? 1 : 0), cj = c - (q >= 2 ? 1 : 0);
  int nm = 0;
  if ((code & (1u << (12 + q))) && ev::member_iface(F, 0, cj, m[nm])) ms[nm++] = F.H * F.pitch + cj;
  if ((code & (1u << (16 + q))) && ev::member_iface(F, 1, cj, m[nm]))
    ms[nm++] = (F.H + 1) * F.pitch + cj;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      const int rr = ci + b, cc = cj + a;
      if (rr == r && cc == c) continue;
      if (ev::member_at(F, rr, cc, m[nm])) ms[nm++] = rr * F.pitch + cc;
    }
  return nm;
}

// The members ev::update_iface uses for interface node `col` of `side`.
__device__ int iface_members_s(const Fld64& F, int side, int col, uint32_t code, Mem* m, int* ms) {
  int nm = 0;
  const int o = side ^ 1;
  const bool has_o = o == 0 ? (code & (1u << 12)) : (code & (1u << 16));
  if (has_o && ev::member_iface(F, o, col, m[nm])) ms[nm++] = (F.H + o) * F.pitch + col;
  const int br = FMT_RO(F.izc + side * F.pitch + col) - F.z_lo;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      if (ev::member_at(F, br + b, col + a, m[nm])) ms[nm++] = (br + b) * F.pitch + col + a;
  return nm;
}

// The direct neighbour `dir` of grid node (r, c) (rnb4's order L, R, U, D)
// in dual form; inputs are appended from index k.
__device__ DNb dual_nb(const Fld64& F, const RNb& n, int r, int c, int dir, const Dn& vu,
                       int& k, Inputs& in) {
  const int dr[4] = {0, 0, -1, 1}, dc[4] = {-1, 1, 0, 0};
  const int s1 = (r + dr[dir]) * F.pitch + (c + dc[dir]);
  const int s2 = (r + 2 * dr[dir]) * F.pitch + (c + 2 * dc[dir]);
  DNb o;
  o.dirx = n.dirx;
  o.second = n.second;
  in.tslot[k] = s1;
  o.T = dvar(n.T, k++);
  if (n.second) {
    in.tslot[k] = s2;
    o.T2 = dvar(n.T2, k++);
  } else {
    o.T2 = dconst(0.0);
  }
  in.vslot[k] = s1;
  const Dn v1 = dvar(FMT_RO(F.vel + s1), k++);
  const Dn velx = 0.5 * (vu + v1);
  const Dn dd = velx / F.dx;
  o.d2 = dd * dd;
  return o;
}

// Seed of slot s in dual form (k_init_source, k_seed_iface).
__device__ bool seed_dual(const AdjField& A, int s, int row, int col, Dn& val, Inputs& in,
                          int& kind) {
  const Fld64& F = A.F;
  const double h = F.dx;
  if (!A.seed.src_T) {
    if (row >= F.H) return false;
    const int iz = F.z_lo + row;
    const double ddx = (F.x0 + col * h) - A.sx, ddz = iz * h - A.sz;
    const double dist = sqrt(ddx * ddx + ddz * ddz);
    if (dist < 0.01 * F.tol) {
      val = dconst(0.0);
      kind = kAdjFixed;
      return true;
    }
    const double v = FMT_RO(F.vel + s);
    Dn vd;
    if (v < 0.01) {
      vd = dconst(0.01);
    } else {
      in.vslot[0] = s;
      vd = dvar(v, 0);
    }
    val = dist / vd;
    kind = kAdjSource;
    return true;
  }
  const Seed64& D = A.seed;
  if (row == F.H + D.dst_side) {
    const int ps = D.src_row * D.src_pitch + col;
    in.xslot[0] = ps;
    val = dvar(D.src_T[ps], 0);
    kind = kAdjHandOff;
    return true;
  }
  if (row >= F.H) return false;
  // the first interface node n (columns col-1..col+1) whose rows hold the node
  const int r = F.z_lo + row;
  for (int n = col - 1; n <= col + 1; ++n) {
    if (n < 0 || n >= F.nx) continue;
    const int izf = D.ifc.izc[n];
    if (izf < 0) continue;
    int r_a, r_b, st;
    if (D.dst_side == 1) { r_a = izf; r_b = max(0, izf - 2); st = -1; }
    else { r_a = izf + 1; r_b = min(F.nz - 1, izf + 3); st = 1; }
    for (int rr = r_a; st > 0 ? rr <= r_b : rr >= r_b; rr += st) {
      if (rr < D.r0[col] || rr > D.r1[col]) continue;
      if (rr != r) continue;
      const int ps = D.src_row * D.src_pitch + n;
      const double xm = F.ifx[n];
      in.zkey[2] = A.seed_iface * 65536 + n;
      const Dn zm = dvar(D.ifc.z[n], 2);
      const double ddx = (F.x0 + col * h) - xm;
      const Dn ddz = r * h - zm;
      const Dn dist = dsqrt(ddx * ddx + ddz * ddz);
      const double v = FMT_RO(F.vel + s);
      in.xslot[0] = ps;
      const Dn Tn = dvar(D.src_T[ps], 0);
      Dn vd;
      if (v < 0.01) {
        vd = dconst(0.01);
      } else {
        in.vslot[1] = s;
        vd = dvar(v, 1);
      }
      val = Tn + dist / vd;
      kind = kAdjHandOff;
      return true;
    }
  }
  return false;
}

// The link of slot s (see the file comment).  Returns false for a slot
// without one (outside the region or unreached).
__device__ bool derive(const AdjField& A, int s, AdjLink& L) {
  const Fld64& F = A.F;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    L.t[j] = -1;
    L.v[j] = -1;
    L.wt[j] = 0.0;
    L.wv[j] = 0.0;
  }
  L.xref = -1;
  L.xw = 0.0;
  L.kind = kAdjNone;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    L.z[j] = -1;
    L.wz[j] = 0.0;
  }
  const uint32_t code = FMT_RO(F.code + s);
  const double Ts = F.T[s];
  if (!(code & kInRegion) || !(Ts < kReachD)) return false;
  const int row = s / F.pitch, col = s - row * F.pitch;
  const bool grid = row < F.H;
  const double vu = FMT_RO(F.vel + s);
  Cand best = ev::no_cand();
  Win w;
  RNb nb[4];
  double xu = 0.0, zu = 0.0;
  const bool upd = (code & kUpdatable) && s != F.frozen_slot;
  if (upd && grid) {
    xu = ev::xg(F, col);
    zu = ev::zg(F, row);
    ev::rnb4(F, row, col, vu, nb);
    if (code & kFullyRegular) {
      quad_t(nb, 0, 2, 0, best, w);
      quad_t(nb, 1, 2, 1, best, w);
      quad_t(nb, 0, 3, 2, best, w);
      quad_t(nb, 1, 3, 3, best, w);
    } else {
      Cand rb = ev::no_cand();
      Win rw;
      for (int q = 0; q < 4; ++q) {
        if (!(code & (1u << (4 + q))) || (code & (1u << (8 + q)))) continue;
        quad_t(nb, (q >= 2) ? 0 : 1, (q & 1) ? 2 : 3, q * 32, rb, rw);
      }
      CutAcc Ac;
      Ac.best = ev::no_cand();
      Ac.pre_min = kHugeD;
      Ac.rtrig = rb.trig;
      Ac.rord = rb.ord;
      Win cw;
      for (int q = 0; q < 4; ++q) {
        if (!(code & (1u << (4 + q))) || !(code & (1u << (8 + q)))) continue;
        Mem m[6];
        int ms[6];
        const int nm = cell_members_s(F, row, col, code, q, m, ms);
        for (int p = 0; p < nm; ++p) cut_member_t(m, nm, p, xu, zu, vu, F.tol, q * 32, Ac, q, cw);
      }
      const bool reg_wins =
          rb.t < Ac.best.t || (rb.t == Ac.best.t && ev::earlier(rb.trig, rb.ord, Ac.best));
      best = reg_wins ? rb : Ac.best;
      w = reg_wins ? rw : cw;
    }
  } else if (upd) {
    const int side = row - F.H;
    if (FMT_RO(F.izc + side * F.pitch + col) >= 0) {
      xu = FMT_RO(F.ifx + col);
      zu = FMT_RO(F.ifz + side * F.pitch + col);
      Mem m[6];
      int ms[6];
      const int nm = iface_members_s(F, side, col, code, m, ms);
      CutAcc Ac;
      Ac.best = ev::no_cand();
      Ac.pre_min = kHugeD;
      Ac.rtrig = -kHugeD;
      Ac.rord = -1;
      Win cw;
      for (int p = 0; p < nm; ++p) cut_member_t(m, nm, p, xu, zu, vu, F.tol, 0, Ac, 0, cw);
      best = Ac.best;
      w = cw;
    }
  }
  // a seed at or below the best candidate is kept (ev::finish)
  double T = best.t < kReachD ? best.t : kHugeD;
  bool seeded = false;
  if (F.fl[s] & kFlSeed) {
    const double4 sd = F.seed[s];
    if (sd.x < kReachD && (T >= kReachD || sd.x <= T)) seeded = true;
  }
  Dn val = dconst(kHugeD);
  Inputs in;
  in.clear();
  int kind = kAdjMismatch;
  bool ok = false;
  if (seeded) {
    ok = seed_dual(A, s, row, col, val, in, kind);
  } else if (w.kind == kAdjRegular) {
    int k = 0;
    in.vslot[k] = s;
    const Dn vud = dvar(vu, k++);
    DNb dx_, dz_;
    const DNb* P = nullptr;
    const DNb* Q = nullptr;
    if (w.x >= 0) { dx_ = dual_nb(F, nb[w.x], row, col, w.x, vud, k, in); P = &dx_; }
    if (w.z >= 0) {
      dz_ = dual_nb(F, nb[w.z], row, col, w.z, vud, k, in);
      if (P) Q = &dz_; else P = &dz_;
    }
    ok = reg_dual(P, Q, val);
    kind = kAdjRegular;
  } else if (w.kind == kAdjRay || w.kind == kAdjPlane) {
    Mem m[6];
    int ms[6];
    if (grid) cell_members_s(F, row, col, code, w.cell, m, ms);
    else iface_members_s(F, row - F.H, col, code, m, ms);
    const Mem& a = m[w.p];
    // an interface node's depth is an input (interface id * 65536 + column)
    auto zkey = [&](int slot) {
      const int rr = slot / F.pitch;
      if (rr < F.H) return -1;
      return (rr == F.H ? A.itop : A.ibot) * 65536 + (slot - rr * F.pitch);
    };
    auto zin = [&](double z, int slot, int k) {
      const int key = zkey(slot);
      if (key < 0) return dconst(z);
      in.zkey[k] = key;
      return dvar(z, k);
    };
    const Dn zud = zin(zu, s, 7);
    if (w.kind == kAdjRay) {
      in.tslot[0] = ms[w.p];
      in.vslot[1] = ms[w.p];
      in.vslot[2] = s;
      bool offered = false;
      val = from1_dual(a, dvar(a.T, 0), dvar(a.v, 1), zin(a.z, ms[w.p], 3), xu, zud, dvar(vu, 2),
                       F.tol, offered);
      ok = offered;
      const double dxu = xu - a.x, dzu = zu - a.z;
      kind = sqrt(dxu * dxu + dzu * dzu) < 0.01 * F.tol ? kAdjCopy : kAdjRay;
    } else {
      const Mem& b = m[w.q];
      in.tslot[0] = ms[w.p];
      in.tslot[1] = ms[w.q];
      in.vslot[2] = ms[w.p];
      in.vslot[3] = ms[w.q];
      in.vslot[4] = s;
      ok = from2_dual(a, b, dvar(a.T, 0), dvar(b.T, 1), dvar(a.v, 2), dvar(b.v, 3),
                      zin(a.z, ms[w.p], 5), zin(b.z, ms[w.q], 6), xu, zud, dvar(vu, 4), F.tol,
                      best.t, val);
      kind = kAdjPlane;
    }
  }
  if (!ok || __double_as_longlong(val.v) != __double_as_longlong(Ts)) {
    L.kind = kAdjMismatch;
    return true;
  }
  L.kind = kind;
  int nt = 0, nv = 0, nzr = 0;
  for (int k = 0; k < kND; ++k) {
    if (in.tslot[k] >= 0 && nt < 4) { L.t[nt] = in.tslot[k]; L.wt[nt++] = val.d[k]; }
    if (in.vslot[k] >= 0 && nv < 4) { L.v[nv] = in.vslot[k]; L.wv[nv++] = val.d[k]; }
    if (in.xslot[k] >= 0) { L.xref = in.xslot[k]; L.xw = val.d[k]; }
    if (in.zkey[k] >= 0 && nzr < 3) { L.z[nzr] = in.zkey[k]; L.wz[nzr++] = val.d[k]; }
  }
  return true;
}

__global__ void __launch_bounds__(256) k_adj_links(AdjField* fs, int nf) {
  AdjField& A = fs[blockIdx.y];
  const int ns = A.F.nslots();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ unsigned n_reach, n_bad, n_unl;
  if (threadIdx.x == 0) { n_reach = 0; n_bad = 0; n_unl = 0; }
  __syncthreads();
  if (s < ns) {
    AdjLink L;
    if (derive(A, s, L)) {
      atomicAdd(&n_reach, 1u);
      if (L.kind == kAdjMismatch) atomicAdd(&n_bad, 1u);
      for (int j = 0; j < 4; ++j) {
        const int t = L.t[j];
        if (t < 0) continue;
        atomicAdd(&A.cnt[t], 1u);
        // the reverse sweep finds a node's readers among its spread targets
        bool listed = false;
        for (int q = 0; q < 16; ++q) listed = listed || ev::spread_target_at(A.F, t, q) == s;
        if (!listed) atomicAdd(&n_unl, 1u);
      }
    }
    A.link[s] = L;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (n_reach) atomicAdd(&A.ctr[kAdjCtrReached], n_reach);
    if (n_bad) atomicAdd(&A.ctr[kAdjCtrMismatch], n_bad);
    if (n_unl) atomicAdd(&A.ctr[kAdjCtrUnlisted], n_unl);
  }
}

// Nodes no link reads start the reverse sweep.
__global__ void k_adj_front(AdjField* fs, int nf) {
  AdjField& A = fs[blockIdx.y];
  const int ns = A.F.nslots();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int kind = A.link[s].kind;
  if (kind == kAdjNone || A.cnt[s] != 0u) return;
  A.fa[atomicAdd(&A.ctr[kAdjCtrFront], 1u)] = (unsigned)s;
}

// The readers of slot s (the links that read its time, found among its
// spread targets in their fixed order) with their weights, written at
// roff[s]: the order the sweep sums them in.
__global__ void k_adj_readers(AdjField* fs, int nf, int* rk, double* rw) {
  AdjField& A = fs[blockIdx.y];
  const int ns = A.F.nslots();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns || A.rcnt[s] == 0u) return;
  unsigned o = A.roff[s];
  const unsigned end = o + A.rcnt[s];
  for (int q = 0; q < 16 && o < end; ++q) {
    const int k = ev::spread_target_at(A.F, s, q);
    if (k < 0) continue;
    const AdjLink& K = A.link[k];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (K.t[j] == s && o < end) {
        rk[o] = k;
        rw[o] = K.wt[j];
        ++o;
      }
  }
}

// Reverse sweep of one field per block: a node is processed once every link
// reading it has been (its count reaches zero), so each node is listed once
// and the loop ends after at most one round per node.  lam[s] = d[s] + the
// sum over its readers, in list order, of weight * lam[reader].
__global__ void __launch_bounds__(1024) k_adj_sweep(AdjField* fs, int nf, const int* rk,
                                                    const double* rw) {
  AdjField& A = fs[blockIdx.x];
  __shared__ unsigned n_in, n_out;
  unsigned* fin = A.fa;
  unsigned* fout = A.fb;
  if (threadIdx.x == 0) {
    n_in = A.ctr[kAdjCtrFront];
    n_out = 0;
  }
  __syncthreads();
  unsigned done = 0, rounds = 0;
  for (;;) {
    const unsigned n = n_in;
    if (n == 0) break;
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
      const int s = (int)fin[i];
      double l = A.d[s];
      const unsigned o = A.roff[s], c = A.rcnt[s];
      for (unsigned e = 0; e < c; ++e) l += rw[o + e] * A.lam[rk[o + e]];
      A.lam[s] = l;
      const int* ts = A.link[s].t;   // a link is 8-byte aligned: plain int loads
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int t = ts[j];
        if (t < 0) continue;
        if (atomicSub(&A.cnt[t], 1u) == 1u) fout[atomicAdd(&n_out, 1u)] = (unsigned)t;
      }
    }
    __syncthreads();
    done += n;
    ++rounds;
    if (threadIdx.x == 0) {
      n_in = n_out;
      n_out = 0;
    }
    unsigned* tmp = fin;
    fin = fout;
    fout = tmp;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    A.ctr[kAdjCtrDone] = done;
    A.ctr[kAdjCtrRounds] = rounds;
  }
}

// gv[j] += sum over the links reading slot j's velocity (the node itself,
// then its spread targets in order) of weight * lam[reader] (the head-wave
// reversal may have added its terms first).
__global__ void k_adj_gv(AdjField* fs, int nf) {
  AdjField& A = fs[blockIdx.y];
  const int ns = A.F.nslots();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  double g = 0.0;
  for (int q = -1; q < 16; ++q) {
    const int k = q < 0 ? j : ev::spread_target_at(A.F, j, q);
    if (k < 0) continue;
    const AdjLink& K = A.link[k];
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (K.v[r] == j) g += K.wv[r] * A.lam[k];
  }
  A.gv[j] += g;
}

// Hand-off: parent interface node n gets the adjoint of the child's seeds
// that read it (the child's interface node n, then the grid nodes of columns
// n-1..n+1 in the rows a hand-off can seed), in that fixed order.
__global__ void k_adj_handoff(AdjField* fs, const int* child, const int* parent, int npair,
                              int nx) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nx) return;
  const AdjField& C = fs[child[blockIdx.y]];
  AdjField& P = fs[parent[blockIdx.y]];
  const Seed64& D = C.seed;
  const Fld64& F = C.F;
  const int ps = D.src_row * D.src_pitch + n;
  double acc = 0.0;
  {
    const int s = (F.H + D.dst_side) * F.pitch + n;
    const AdjLink& L = C.link[s];
    if (L.xref == ps) acc += L.xw * C.lam[s];
  }
  const int izf = D.ifc.izc[n];
  if (izf >= 0) {
    for (int c = n - 1; c <= n + 1; ++c) {
      if (c < 0 || c >= nx) continue;
      for (int r = izf - 2; r <= izf + 3; ++r) {
        const int br = r - F.z_lo;
        if (br < 0 || br >= F.H) continue;
        const int s = br * F.pitch + c;
        const AdjLink& L = C.link[s];
        if (L.xref == ps) acc += L.xw * C.lam[s];
      }
    }
  }
  if (acc != 0.0) P.d[ps] += acc;
}

// The head-wave sweep reversed, one field per thread (k_headwave's order).
// scratch: per field, nx doubles and 2*nx bytes.
__global__ void k_adj_headwave(AdjField* fs, const int* which, int nsel, const int* hw_slot,
                               const double* hw_v, const int* hw_vslot, double* const* pre,
                               double dx_if, int nx, double* scratch) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsel) return;
  AdjField& A = fs[which[q]];
  double* th = scratch + (size_t)q * nx;
  uint8_t* fwd = reinterpret_cast<uint8_t*>(scratch + (size_t)nsel * nx) + (size_t)q * 2 * nx;
  uint8_t* bwd = fwd + nx;
  const double* p = pre[q];
  for (int n = 0; n < nx; ++n) th[n] = hw_slot[n] >= 0 ? p[n] : kHugeD;
  for (int n = 0; n < nx; ++n) { fwd[n] = 0; bwd[n] = 0; }
  for (int n = 1; n < nx; ++n)
    if (hw_v[n] > 0.0) {
      const double c = th[n - 1] + dx_if / hw_v[n];
      if (c < th[n]) fwd[n] = 1;
      th[n] = fmin(th[n], c);
    }
  for (int n = nx - 2; n >= 0; --n)
    if (hw_v[n] > 0.0) {
      const double c = th[n + 1] + dx_if / hw_v[n];
      if (c < th[n]) bwd[n] = 1;
      th[n] = fmin(th[n], c);
    }
  // th now holds the sweep's values; reuse it for their adjoint
  for (int n = 0; n < nx; ++n) {
    const int s = hw_slot[n];
    double g = 0.0;
    if (s >= 0 && th[n] < p[n] - 1.0e-10) {
      g = A.d[s];
      A.d[s] = 0.0;
    }
    th[n] = g;
  }
  for (int n = 0; n <= nx - 2; ++n)
    if (bwd[n]) {
      th[n + 1] += th[n];
      const int vs = hw_vslot[n];
      if (vs >= 0) A.gv[vs] += th[n] * (-dx_if / (hw_v[n] * hw_v[n]));
      th[n] = 0.0;
    }
  for (int n = nx - 1; n >= 1; --n)
    if (fwd[n]) {
      th[n - 1] += th[n];
      const int vs = hw_vslot[n];
      if (vs >= 0) A.gv[vs] += th[n] * (-dx_if / (hw_v[n] * hw_v[n]));
      th[n] = 0.0;
    }
  for (int n = 0; n < nx; ++n)
    if (hw_slot[n] >= 0 && th[n] != 0.0) A.d[hw_slot[n]] += th[n];
}

__global__ void k_adj_swap_pre(AdjField* fs, const int* which, int nsel, const int* hw_slot,
                               double* const* pre, int nx) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nx || hw_slot[n] < 0) return;
  AdjField& A = fs[which[blockIdx.y]];
  double* p = pre[blockIdx.y];
  const double t = A.F.T[hw_slot[n]];
  A.F.T[hw_slot[n]] = p[n];
  p[n] = t;
}

// Depth gradient of field A's interface nodes in column c: the links that
// read the depth of the region's top / bottom interface node (the node
// itself and its spread targets; hand-off seeds excluded), the hand-off seeds
// that read the parent interface's node (the child's seed band, columns
// c-1..c+1), and the slots whose velocity is sampled off the interface.
__global__ void k_adj_gz(AdjField* fs, int nf, int nx) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nx) return;
  AdjField& A = fs[blockIdx.y];
  const Fld64& F = A.F;
  double g[3] = {0.0, 0.0, 0.0};
  for (int side = 0; side < 2; ++side) {
    const int S = (F.H + side) * F.pitch + c;
    const int key = (side == 0 ? A.itop : A.ibot) * 65536 + c;
    for (int q = -1; q < 16; ++q) {
      const int k = q < 0 ? S : ev::spread_target_at(F, S, q);
      if (k < 0) continue;
      const AdjLink& L = A.link[k];
      if (L.kind == kAdjHandOff) continue;
#pragma unroll
      for (int r = 0; r < 3; ++r)
        if (L.z[r] == key) g[side] += L.wz[r] * A.lam[k];
    }
  }
  if (A.level > 0) {
    const int key = A.seed_iface * 65536 + c;
    const int izf = A.seed.ifc.izc[c];
    if (izf >= 0)
      for (int cc = c - 1; cc <= c + 1; ++cc) {
        if (cc < 0 || cc >= nx) continue;
        for (int r = izf - 2; r <= izf + 3; ++r) {
          const int br = r - F.z_lo;
          if (br < 0 || br >= F.H) continue;
          const int k = br * F.pitch + cc;
          const AdjLink& L = A.link[k];
          if (L.kind != kAdjHandOff) continue;
#pragma unroll
          for (int j = 0; j < 3; ++j)
            if (L.z[j] == key) g[2] += L.wz[j] * A.lam[k];
        }
      }
  }
  for (int e = A.zrp[c]; e < A.zrp[c + 1]; ++e) g[A.zside[e]] += A.gv[A.zslot[e]] * A.zdv[e];
  A.gzf[c] = g[0];
  A.gzf[nx + c] = g[1];
  A.gzf[2 * (size_t)nx + c] = g[2];
}

// giface[(i - 1) * nx + c] += the fields' terms for interface i, fields in order.
__global__ void k_adj_gz_sum(const AdjField* fs, int nf, int nx, double* giface) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y + 1;
  if (c >= nx) return;
  double g = giface[(size_t)(i - 1) * nx + c];
  for (int k = 0; k < nf; ++k) {
    const AdjField& A = fs[k];
    if (A.itop == i) g += A.gzf[c];
    if (A.ibot == i) g += A.gzf[nx + c];
    if (A.level > 0 && A.seed_iface == i) g += A.gzf[2 * (size_t)nx + c];
  }
  giface[(size_t)(i - 1) * nx + c] = g;
}

__global__ void k_adj_grid(const AdjField* fs, int nf, const int* const* rp,
                           const int* const* slot, const double* const* w, size_t nnode,
                           double* gvel) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnode) return;
  double g = gvel[i];
  for (int k = 0; k < nf; ++k) {
    const double* gv = fs[k].gv;
    for (int e = rp[k][i]; e < rp[k][i + 1]; ++e) g += w[k][e] * gv[slot[k][e]];
  }
  gvel[i] = g;
}

}  // namespace

void adj_links(AdjField* f, int nf, size_t max_slots, cudaStream_t st) {
  if (nf <= 0) return;
  const dim3 grid((unsigned)((max_slots + 255) / 256), nf);
  k_adj_links<<<grid, 256, 0, st>>>(f, nf);
}

void adj_readers(AdjField* f, int nf, size_t max_slots, int* rk, double* rw, cudaStream_t st) {
  if (nf <= 0) return;
  const dim3 grid((unsigned)((max_slots + 255) / 256), nf);
  k_adj_readers<<<grid, 256, 0, st>>>(f, nf, rk, rw);
}

void adj_sweep(AdjField* f, int nf, size_t max_slots, const int* rk, const double* rw,
               cudaStream_t st) {
  if (nf <= 0) return;
  const dim3 grid((unsigned)((max_slots + 255) / 256), nf);
  k_adj_front<<<grid, 256, 0, st>>>(f, nf);
  k_adj_sweep<<<nf, 1024, 0, st>>>(f, nf, rk, rw);
  k_adj_gv<<<grid, 256, 0, st>>>(f, nf);
}

void adj_handoff(AdjField* f, const int* child, const int* parent, int npair, int nx,
                 cudaStream_t st) {
  if (npair <= 0) return;
  k_adj_handoff<<<dim3((nx + 127) / 128, npair), 128, 0, st>>>(f, child, parent, npair, nx);
}

void adj_headwave(AdjField* f, const int* which, int nsel, const int* hw_slot, const double* hw_v,
                  const int* hw_vslot, double* const* pre, double dx_if, int nx,
                  double* scratch, cudaStream_t st) {
  if (nsel <= 0) return;
  k_adj_headwave<<<(nsel + 31) / 32, 32, 0, st>>>(f, which, nsel, hw_slot, hw_v, hw_vslot, pre,
                                                  dx_if, nx, scratch);
}

void adj_swap_pre(AdjField* f, const int* which, int nsel, const int* hw_slot,
                  double* const* pre, int nx, cudaStream_t st) {
  if (nsel <= 0) return;
  k_adj_swap_pre<<<dim3((nx + 127) / 128, nsel), 128, 0, st>>>(f, which, nsel, hw_slot, pre, nx);
}

void adj_depth(AdjField* f, int nf, int nx, double* giface, cudaStream_t st) {
  if (nf <= 0) return;
  k_adj_gz<<<dim3((nx + 127) / 128, nf), 128, 0, st>>>(f, nf, nx);
  k_adj_gz_sum<<<dim3((nx + 127) / 128, 5), 128, 0, st>>>(f, nf, nx, giface);
}

void adj_to_grid(const AdjField* f, int nf, const int* const* map_rp, const int* const* map_slot,
                 const double* const* map_w, size_t nnode, double* gvel, cudaStream_t st) {
  if (nf <= 0 || nnode == 0) return;
  k_adj_grid<<<(unsigned)((nnode + 255) / 256), 256, 0, st>>>(f, nf, map_rp, map_slot, map_w,
                                                              nnode, gvel);
}

}  // namespace fmt2d

// ------------------------------------------------------------------ host
#include "engine.h"
#include "rays.cuh"
#include <cub/cub.cuh>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

namespace fmt2d {

namespace {

// The corner k_init_source fixes at the source (within 0.01*tolerance), or -1.
int frozen_corner(const Model& m, const Region& G, double sx, double sz) {
  const double h = m.dx;
  int ix0 = (int)std::floor((sx - m.x0) / h);
  int iz0 = (int)std::floor((sz - 0.0) / h);
  ix0 = std::max(0, std::min(m.nx - 2, ix0));
  iz0 = std::max(0, std::min(m.nz - 2, iz0));
  int frozen = -1;
  for (int ix = ix0; ix <= ix0 + 1; ++ix)
    for (int iz = iz0; iz <= iz0 + 1; ++iz) {
      const int br = iz - G.z_lo;
      if (br < 0 || br >= G.H) continue;
      const int s = br * G.pitch + ix;
      if (!(G.code[s] & kInRegion)) continue;
      const double ddx = (m.x0 + ix * h) - sx, ddz = iz * h - sz;
      if (std::sqrt(ddx * ddx + ddz * ddz) < 0.01 * m.tolerance) frozen = s;
    }
  return frozen;
}

template <class T>
std::string adj_put(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (!b.p) return "device allocation failed (adjoint)";
  if (!v.empty() &&
      cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st) !=
          cudaSuccess)
    return "cudaMemcpyAsync failed (adjoint)";
  // the host vector may go out of scope before the copy runs
  if (cudaStreamSynchronize(st) != cudaSuccess) return "cudaStreamSynchronize failed (adjoint)";
  return std::string();
}

// phase -> terminal time field (Pg, PsedP, PmP, Pg_ss, Pg_ss2)
constexpr int kTerminal[6] = {0, 1, 3, 5, 8, 12};
inline bool terminal_tf(int tf) { return tf == 1 || tf == 3 || tf == 5 || tf == 8 || tf == 12; }

}  // namespace

#define ACK(x)                                                                \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_); \
  } while (0)

std::string Engine::misfit_gradient(const int* src, const int* phase, const double* rx,
                                    const double* rz, const double* t_obs, const double* sigma,
                                    int npick, double* misfit, double* t_calc, int* valid,
                                    double* grad_vel, double* grad_iface, double* info) {
  cudaSetDevice(device_);
  if (m_.nx == 0) return "no model uploaded";
  if (npick < 0) return "negative pick count";
  for (int p = 0; p < npick; ++p) {
    if (phase[p] < 1 || phase[p] > 5) return "pick phase out of range";
    if (!(sigma[p] > 0.0)) return "pick sigma must be positive";
  }
  {
    std::vector<int> hs;
    for (int s : hw_slot_h_)
      if (s >= 0) hs.push_back(s);
    std::sort(hs.begin(), hs.end());
    if (std::adjacent_find(hs.begin(), hs.end()) != hs.end())
      return "head-wave sweep nodes share a slot (not covered by the adjoint)";
  }
  const auto t0 = std::chrono::steady_clock::now();
  long long nnz = 0;
  std::string e = trace(src, phase, rx, rz, npick, t_calc, valid, &nnz, /*rows=*/false);
  if (!e.empty()) return e;
  const int ns = nsrc();
  std::vector<double> coef(std::max(npick, 1), 0.0);
  std::vector<char> need((size_t)std::max(ns, 1) * 13, 0);
  double J = 0.0;
  for (int p = 0; p < npick; ++p) {
    if (!valid[p] || !(t_obs[p] >= 0.0)) continue;
    const double r = t_calc[p] - t_obs[p];
    J += 0.5 * (r / sigma[p]) * (r / sigma[p]);
    coef[p] = r / (sigma[p] * sigma[p]);
    for (int tf = kTerminal[phase[p]]; tf > 0; tf = kTf[tf].level > 0 ? kTf[tf].parent : 0)
      need[(size_t)src[p] * 13 + tf] = 1;
  }
  *misfit = J;
  // the picks of each (source, terminal field), in pick order
  std::vector<std::vector<int>> picks_of((size_t)std::max(ns, 1) * 13);
  for (int p = 0; p < npick; ++p)
    if (coef[p] != 0.0) picks_of[(size_t)src[p] * 13 + kTerminal[phase[p]]].push_back(p);
  const size_t nnode = (size_t)m_.nx * m_.nz;
  DevBuf d_coef, d_gvel, d_giface;
  if (!(e = adj_put(d_coef, coef, stream_)).empty()) return e;
  d_gvel.alloc(nnode * sizeof(double));
  d_giface.alloc((size_t)5 * m_.nx * sizeof(double));
  if (!d_gvel.p || !d_giface.p) return "device allocation failed (gradient)";
  ACK(cudaMemsetAsync(d_gvel.p, 0, nnode * sizeof(double), stream_));
  ACK(cudaMemsetAsync(d_giface.p, 0, (size_t)5 * m_.nx * sizeof(double), stream_));
  // slot -> grid velocity maps of the regions in use, and their slots sampled
  // off an interface (depth slopes), built once per uploaded model
  for (int tf = 1; tf <= 12; ++tf) {
    bool used = false;
    for (int s = 0; s < ns; ++s) used = used || need[(size_t)s * 13 + tf];
    const int r = kTf[tf].reg;
    if (!used || adj_map_version_[r] == model_version_) continue;
    std::vector<int> rp, sl, zrp, zsl, zsd;
    std::vector<double> w, zdv;
    if (!(e = slot_velocity_map(m_, r, rp, sl, w, &zrp, &zsl, &zsd, &zdv)).empty()) return e;
    DevBuf* M = adj_map_[r];
    if (!(e = adj_put(M[0], rp, stream_)).empty()) return e;
    if (!(e = adj_put(M[1], sl, stream_)).empty()) return e;
    if (!(e = adj_put(M[2], w, stream_)).empty()) return e;
    if (!(e = adj_put(M[3], zrp, stream_)).empty()) return e;
    if (!(e = adj_put(M[4], zsl, stream_)).empty()) return e;
    if (!(e = adj_put(M[5], zsd, stream_)).empty()) return e;
    if (!(e = adj_put(M[6], zdv, stream_)).empty()) return e;
    adj_map_version_[r] = model_version_;
  }
  DevBuf d_hwvslot;
  if (!(e = adj_put(d_hwvslot, hw_vslot_h_, stream_)).empty()) return e;
  // sources in chunks that fit in device memory
  // per slot: link, counts, adjoint, direct term, velocity gradient, work
  // lists, reader count and offset, and up to 4 reader entries
  constexpr size_t kPerSlot = sizeof(AdjLink) + 2 * sizeof(unsigned) + 3 * sizeof(double) +
                              2 * sizeof(unsigned) + 2 * sizeof(unsigned) +
                              4 * (sizeof(int) + sizeof(double));
  size_t free_b = 0, total_b = 0;
  ACK(cudaMemGetInfo(&free_b, &total_b));
  const size_t budget = free_b / 2;
  unsigned long long cnt_bad = 0, cnt_unl = 0, cnt_left = 0, cnt_reach = 0, cnt_fields = 0;
  unsigned max_rounds = 0;
  int s0 = 0;
  while (s0 < ns) {
    // [s0, s1): the sources of this chunk
    size_t bytes = 0;
    int s1 = s0;
    while (s1 < ns) {
      size_t b = 0;
      for (int tf = 1; tf <= 12; ++tf)
        if (need[(size_t)s1 * 13 + tf]) b += reg_[kTf[tf].reg].nslots * kPerSlot;
      if (s1 > s0 && bytes + b > budget) break;
      bytes += b;
      ++s1;
    }
    // fields of the chunk, deepest stage level first
    struct Item { int s, tf, level; };
    std::vector<Item> items;
    for (int s = s0; s < s1; ++s)
      for (int tf = 1; tf <= 12; ++tf)
        if (need[(size_t)s * 13 + tf]) {
          if (!fields_[s][tf].solved) return "time field not solved (run the forward first)";
          items.push_back({s, tf, kTf[tf].level});
        }
    s0 = s1;
    if (items.empty()) continue;
    std::stable_sort(items.begin(), items.end(),
                     [](const Item& a, const Item& b) { return a.level > b.level; });
    const int nf = (int)items.size();
    std::vector<size_t> off(nf + 1, 0);
    for (int i = 0; i < nf; ++i) off[i + 1] = off[i] + reg_[kTf[items[i].tf].reg].nslots;
    const size_t tot = off[nf];
    DevBuf b_link, b_cnt, b_lam, b_d, b_gv, b_fa, b_fb, b_ctr, b_gz, b_rcnt, b_roff;
    b_rcnt.alloc(tot * sizeof(unsigned));
    b_roff.alloc(tot * sizeof(unsigned));
    b_gz.alloc((size_t)nf * 3 * m_.nx * sizeof(double));
    b_link.alloc(tot * sizeof(AdjLink));
    b_cnt.alloc(tot * sizeof(unsigned));
    b_lam.alloc(tot * sizeof(double));
    b_d.alloc(tot * sizeof(double));
    b_gv.alloc(tot * sizeof(double));
    b_fa.alloc(tot * sizeof(unsigned));
    b_fb.alloc(tot * sizeof(unsigned));
    b_ctr.alloc((size_t)nf * kAdjCtrN * sizeof(unsigned));
    if (!b_link.p || !b_cnt.p || !b_lam.p || !b_d.p || !b_gv.p || !b_fa.p || !b_fb.p || !b_ctr.p ||
        !b_gz.p || !b_rcnt.p || !b_roff.p)
      return "device allocation failed (adjoint state)";
    ACK(cudaMemsetAsync(b_cnt.p, 0, tot * sizeof(unsigned), stream_));
    ACK(cudaMemsetAsync(b_lam.p, 0, tot * sizeof(double), stream_));
    ACK(cudaMemsetAsync(b_d.p, 0, tot * sizeof(double), stream_));
    ACK(cudaMemsetAsync(b_gv.p, 0, tot * sizeof(double), stream_));
    ACK(cudaMemsetAsync(b_ctr.p, 0, (size_t)nf * kAdjCtrN * sizeof(unsigned), stream_));
    std::vector<AdjField> hf(nf);
    for (int i = 0; i < nf; ++i) {
      const int s = items[i].s, tf = items[i].tf;
      const TfInfo& I = kTf[tf];
      AdjField& A = hf[i];
      A.F = field_view(s, tf);
      A.link = b_link.as<AdjLink>() + off[i];
      A.cnt = b_cnt.as<unsigned>() + off[i];
      A.lam = b_lam.as<double>() + off[i];
      A.d = b_d.as<double>() + off[i];
      A.gv = b_gv.as<double>() + off[i];
      A.fa = b_fa.as<unsigned>() + off[i];
      A.fb = b_fb.as<unsigned>() + off[i];
      A.ctr = b_ctr.as<unsigned>() + (size_t)i * kAdjCtrN;
      A.level = I.level;
      A.itop = m_.reg[I.reg].itop;
      A.ibot = m_.reg[I.reg].ibot;
      A.seed_iface = I.level > 0 ? I.istart : 0;
      A.gzf = b_gz.as<double>() + (size_t)i * 3 * m_.nx;
      A.rcnt = b_rcnt.as<unsigned>() + off[i];
      A.roff = b_roff.as<unsigned>() + off[i];
      A.zrp = adj_map_[I.reg][3].as<int>();
      A.zslot = adj_map_[I.reg][4].as<int>();
      A.zside = adj_map_[I.reg][5].as<int>();
      A.zdv = adj_map_[I.reg][6].as<double>();
      A.sx = src_x_[s];
      A.sz = src_z_[s];
      if (I.level == 0) {
        A.F.frozen_slot = frozen_corner(m_, m_.reg[I.reg], A.sx, A.sz);
      } else {
        const Region& PR = m_.reg[kTf[I.parent].reg];
        Seed64& d = A.seed;
        d.dst = i;
        d.src_T = fields_[s][I.parent].T.as<double>();
        d.src_G = fields_[s][I.parent].Gout.as<double2>();
        d.src_row = PR.H + (I.istart == PR.itop ? 0 : 1);
        d.src_pitch = PR.pitch;
        d.ifc = ifc_[I.istart];
        d.r0 = reg_[I.reg].r0.as<int>();
        d.r1 = reg_[I.reg].r1.as<int>();
        d.dst_side = I.dst_side;
        d.reflect = I.reflect;
        d.target_side = I.target_side;
      }
    }
    DevBuf d_adj;
    if (!(e = adj_put(d_adj, hf, stream_)).empty()) return e;
    AdjField* dA = d_adj.as<AdjField>();
    auto index_of = [&](int s, int tf) {
      for (int i = 0; i < nf; ++i)
        if (items[i].s == s && items[i].tf == tf) return i;
      return -1;
    };
    const double dx_if = m_.xpos[1] - m_.xpos[0];
    for (int i0 = 0; i0 < nf;) {
      const int level = items[i0].level;
      int i1 = i0;
      while (i1 < nf && items[i1].level == level) ++i1;
      size_t max_slots = 0;
      for (int i = i0; i < i1; ++i) max_slots = std::max(max_slots, reg_[kTf[items[i].tf].reg].nslots);
      // hand-off terms from the children (one level deeper, already swept)
      std::vector<int> child, parent;
      for (int i = 0; i < i0; ++i)
        if (items[i].level == level + 1) {
          const int p = index_of(items[i].s, kTf[items[i].tf].parent);
          if (p < 0) return "adjoint: parent field missing";
          child.push_back(i);
          parent.push_back(p);
        }
      DevBuf d_child, d_parent;
      if (!child.empty()) {
        if (!(e = adj_put(d_child, child, stream_)).empty()) return e;
        if (!(e = adj_put(d_parent, parent, stream_)).empty()) return e;
        adj_handoff(dA, d_child.as<int>(), d_parent.as<int>(), (int)child.size(), m_.nx, stream_);
        ACK(cudaGetLastError());
      }
      // the picks' terms on the terminal fields
      // each target field's picks (valid, observed), in pick order
      std::vector<int> tgt, tp(1, 0), tpk;
      std::vector<double*> dptr;
      for (int i = i0; i < i1; ++i)
        if (terminal_tf(items[i].tf)) {
          tgt.push_back(items[i].s * 13 + items[i].tf);
          dptr.push_back(hf[i].d);
          const std::vector<int>& pl = picks_of[(size_t)items[i].s * 13 + items[i].tf];
          tpk.insert(tpk.end(), pl.begin(), pl.end());
          tp.push_back((int)tpk.size());
        }
      DevBuf d_tgt, d_dptr, d_tp, d_tpk;
      if (!tgt.empty() && !tpk.empty()) {
        if (!(e = adj_put(d_tgt, tgt, stream_)).empty()) return e;
        if (!(e = adj_put(d_dptr, dptr, stream_)).empty()) return e;
        if (!(e = adj_put(d_tp, tp, stream_)).empty()) return e;
        if (!(e = adj_put(d_tpk, tpk, stream_)).empty()) return e;
        tr_adj_picks(d_trmodel_.as<TrModel>(), d_trfields_.as<TrField>(), d_picks_.as<TrPick>(),
                     d_entry_.as<double>(), d_coef.as<double>(), d_tgt.as<int>(), d_tp.as<int>(),
                     d_tpk.as<int>(), d_dptr.as<double* const>(), (int)tgt.size(), stream_);
        ACK(cudaGetLastError());
      }
      // the head-wave sweep of the PmP up-going fields, reversed; their
      // links are derived on the solved (pre-sweep) times
      std::vector<int> hw;
      std::vector<double*> pre;
      for (int i = i0; i < i1; ++i)
        if (items[i].tf == 5) {
          FieldStore& S = fields_[items[i].s][5];
          if (!S.hwpre.p) return "adjoint: head-wave times of the PmP field missing";
          hw.push_back(i);
          pre.push_back(S.hwpre.as<double>());
        }
      DevBuf d_hw, d_pre, d_scr;
      if (!hw.empty()) {
        if (!(e = adj_put(d_hw, hw, stream_)).empty()) return e;
        if (!(e = adj_put(d_pre, pre, stream_)).empty()) return e;
        d_scr.alloc(hw.size() * (size_t)m_.nx * (sizeof(double) + 2));
        if (!d_scr.p) return "device allocation failed (head-wave scratch)";
        adj_headwave(dA, d_hw.as<int>(), (int)hw.size(), hw_slot_.as<int>(), hw_v_.as<double>(),
                     d_hwvslot.as<int>(), d_pre.as<double* const>(), dx_if, m_.nx,
                     d_scr.as<double>(), stream_);
        adj_swap_pre(dA, d_hw.as<int>(), (int)hw.size(), hw_slot_.as<int>(),
                     d_pre.as<double* const>(), m_.nx, stream_);
        ACK(cudaGetLastError());
      }
      // the swept times go back into the fields on every way out of this
      // level (after its links and sweep, or on an error return)
      struct SwapBack {
        AdjField* f;
        const int* which;
        int n;
        const int* slot;
        double* const* pre;
        int nx;
        cudaStream_t st;
        ~SwapBack() {
          if (n > 0) {
            adj_swap_pre(f, which, n, slot, pre, nx, st);
            cudaStreamSynchronize(st);
          }
        }
      } swap_back{dA, d_hw.as<int>(), (int)hw.size(), hw_slot_.as<int>(),
                  d_pre.as<double* const>(), m_.nx, stream_};
      adj_links(dA + i0, i1 - i0, max_slots, stream_);
      ACK(cudaGetLastError());
      // reader lists of the level: counts, offsets (relative to the level's
      // first slot), then the lists
      const size_t a0 = off[i0], n0 = off[i1] - off[i0];
      unsigned* rc = b_rcnt.as<unsigned>() + a0;
      unsigned* ro = b_roff.as<unsigned>() + a0;
      ACK(cudaMemcpyAsync(rc, b_cnt.as<unsigned>() + a0, n0 * sizeof(unsigned),
                          cudaMemcpyDeviceToDevice, stream_));
      size_t scan_b = 0;
      ACK(cub::DeviceScan::ExclusiveSum(nullptr, scan_b, rc, ro, (int)n0, stream_));
      DevBuf scan_tmp;
      scan_tmp.alloc(std::max<size_t>(scan_b, 16));
      if (!scan_tmp.p) return "device allocation failed (reader scan)";
      ACK(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_b, rc, ro, (int)n0, stream_));
      unsigned last[2] = {0u, 0u};
      ACK(cudaMemcpyAsync(&last[0], ro + n0 - 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
                          stream_));
      ACK(cudaMemcpyAsync(&last[1], rc + n0 - 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
                          stream_));
      ACK(cudaStreamSynchronize(stream_));
      const size_t nref = (size_t)last[0] + last[1];
      DevBuf b_rk, b_rw;
      b_rk.alloc(std::max<size_t>(nref, 1) * sizeof(int));
      b_rw.alloc(std::max<size_t>(nref, 1) * sizeof(double));
      if (!b_rk.p || !b_rw.p) return "device allocation failed (reader lists)";
      adj_readers(dA + i0, i1 - i0, max_slots, b_rk.as<int>(), b_rw.as<double>(), stream_);
      adj_sweep(dA + i0, i1 - i0, max_slots, b_rk.as<int>(), b_rw.as<double>(), stream_);
      ACK(cudaGetLastError());
      ACK(cudaStreamSynchronize(stream_));
      i0 = i1;
    }
    // onto the propagation grid, fields in order
    std::vector<const int*> mrp(nf), msl(nf);
    std::vector<const double*> mw(nf);
    for (int i = 0; i < nf; ++i) {
      const int r = kTf[items[i].tf].reg;
      mrp[i] = adj_map_[r][0].as<int>();
      msl[i] = adj_map_[r][1].as<int>();
      mw[i] = adj_map_[r][2].as<double>();
    }
    DevBuf d_mrp, d_msl, d_mw;
    if (!(e = adj_put(d_mrp, mrp, stream_)).empty()) return e;
    if (!(e = adj_put(d_msl, msl, stream_)).empty()) return e;
    if (!(e = adj_put(d_mw, mw, stream_)).empty()) return e;
    adj_to_grid(dA, nf, d_mrp.as<const int* const>(), d_msl.as<const int* const>(),
                d_mw.as<const double* const>(), nnode, d_gvel.as<double>(), stream_);
    adj_depth(dA, nf, m_.nx, d_giface.as<double>(), stream_);
    ACK(cudaGetLastError());
    std::vector<unsigned> ctr((size_t)nf * kAdjCtrN);
    ACK(cudaMemcpyAsync(ctr.data(), b_ctr.p, ctr.size() * sizeof(unsigned),
                        cudaMemcpyDeviceToHost, stream_));
    ACK(cudaStreamSynchronize(stream_));
    for (int i = 0; i < nf; ++i) {
      const unsigned* c = &ctr[(size_t)i * kAdjCtrN];
      cnt_bad += c[kAdjCtrMismatch];
      cnt_unl += c[kAdjCtrUnlisted];
      cnt_reach += c[kAdjCtrReached];
      cnt_left += c[kAdjCtrReached] - std::min(c[kAdjCtrReached], c[kAdjCtrDone]);
      max_rounds = std::max(max_rounds, c[kAdjCtrRounds]);
    }
    cnt_fields += nf;
  }
  if (grad_vel)
    ACK(cudaMemcpyAsync(grad_vel, d_gvel.p, nnode * sizeof(double), cudaMemcpyDeviceToHost,
                        stream_));
  if (grad_iface)
    ACK(cudaMemcpyAsync(grad_iface, d_giface.p, (size_t)5 * m_.nx * sizeof(double),
                        cudaMemcpyDeviceToHost, stream_));
  ACK(cudaStreamSynchronize(stream_));
  if (info) {
    info[0] = (double)cnt_bad;
    info[1] = (double)cnt_unl;
    info[2] = (double)cnt_left;
    info[3] = (double)max_rounds;
    info[4] = (double)cnt_fields;
    info[5] = (double)cnt_reach;
    info[6] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                  .count();
    info[7] = 0.0;
  }
  return std::string();
}

}  // namespace fmt2d
