// Device functions of the tiled eikonal solver (stencil, cut-cell updates,
// tile staging).  Included by the solver kernels only.
#pragma once
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

// A candidate time offset with the event that produces it in the reference.
// Fast marching accepts nodes in time order and an update replaces a value
// only when it is strictly smaller, so of equal candidates the one computed
// first survives: the one with the earlier trigger (the latest-accepted
// member of the update), then the earlier one in the reference's order of
// updates within one trigger (ord).
struct Cand {
  float t, trig;
  int ord;
  float gx, gz;
  bool suspect, copy;
};

__device__ __forceinline__ Cand no_cand() {
  Cand c;
  c.t = kHugeF; c.trig = kHugeF; c.ord = 0x7fffffff;
  c.gx = 0.0f; c.gz = 0.0f; c.suspect = false; c.copy = false;
  return c;
}

// (trig, ord) of a precedes b's in the reference's event order
__device__ __forceinline__ bool earlier_event(float trig, int ord, const Cand& b) {
  return trig < b.trig || (trig == b.trig && ord < b.ord);
}

__device__ __forceinline__ void take(Cand& best, float t, float trig, int ord, float gx, float gz,
                                     bool sus, bool copy) {
  if (t < best.t || (t == best.t && earlier_event(trig, ord, best))) {
    best.t = t; best.trig = trig; best.ord = ord; best.gx = gx; best.gz = gz;
    best.suspect = sus; best.copy = copy;
  }
}

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

// Candidates of one regular quadrant: the one-sided update from the earlier
// neighbour (triggered by it while the other was not yet accepted) and the
// two-sided update (triggered by the later one).
__device__ __forceinline__ void quadrant(const Nb& X, const Nb& Z, int ord, Cand& best) {
  if (X.ok && Z.ok) {
    const bool xlow = X.tau <= Z.tau;
    const Nb& lo = xlow ? X : Z;
    if (lo.single_ok) {
      const float t = single_t(lo);
      if (xlow) take(best, t, lo.tau, ord, axis_grad(X, t), 0.0f, true, false);
      else take(best, t, lo.tau, ord, 0.0f, axis_grad(Z, t), true, false);
    }
    const float t = pair_t(X, Z);
    take(best, t, fmaxf(X.tau, Z.tau), ord, axis_grad(X, t), axis_grad(Z, t), false, false);
  } else if (X.ok) {
    if (X.single_ok) {
      const float t = single_t(X);
      take(best, t, X.tau, ord, axis_grad(X, t), 0.0f, true, false);
    }
  } else if (Z.ok) {
    if (Z.single_ok) {
      const float t = single_t(Z);
      take(best, t, Z.tau, ord, 0.0f, axis_grad(Z, t), true, false);
    }
  }
}

// ---------------------------------------------------------------------------
// Cut-cell updates (time_from_1_node2d / time_from_2_nodes2d) on positions
// relative to the updated node and times relative to a reference time of the
// neighbourhood.
struct Member {
  float x, z, tau;   // position relative to the updated node, time offset
  float gx, gz, v;
  bool single_ok, copied;
};

// Candidates of the cut cells of a node.  pre_min tracks the smallest cut-cell
// candidate that the reference computes before the best regular candidate
// (rtrig, rord): the reference's suspect flag is only written by regular
// updates, so a node keeps the flag of the last regular update that lowered it.
struct CutAcc {
  Cand best;
  float pre_min, rtrig;
  int rord;
};

__device__ __forceinline__ void offer(CutAcc& A, float t, float trig, int ord, float gx, float gz,
                                      bool copy) {
  take(A.best, t, trig, ord, gx, gz, false, copy);
  if (trig < A.rtrig || (trig == A.rtrig && ord < A.rord)) A.pre_min = fminf(A.pre_min, t);
}

// tol2 = (0.01 * tolerance)^2: members closer than that hand their time over.
__device__ __forceinline__ void from_1(const Member& a, float vu, float tol2, int ord, CutAcc& A) {
  const float d2 = a.x * a.x + a.z * a.z;
  if (d2 < tol2) {
    if (!a.copied) offer(A, a.tau, a.tau, ord, a.gx, a.gz, true);
    return;
  }
  const float dist = sqrtf(d2);
  const float t = a.tau + dist * (2.0f * rcp(vu + a.v));
  const float ig = rcp(dist * vu);
  offer(A, t, a.tau, ord, -a.x * ig, -a.z * ig, false);
}

// The planar-front update is evaluated in FP64: its root and cone tests
// (det >= 0, w.n <= 0, t >= t1) decide near-grazing fronts by small margins,
// where FP32 rounding would drop candidates the reference keeps.  Pairs whose
// later member is not earlier than the best candidate so far are skipped: a
// planar-front time is never earlier than that member's.
__device__ void from_2(const Member& A_, const Member& B_, int ord, float vu, float tol2,
                       CutAcc& A) {
  const bool swap = A_.tau < B_.tau;           // later (larger time) node first
  const Member& n1 = swap ? B_ : A_;
  const Member& n2 = swap ? A_ : B_;
  const float trig = n1.tau;
  if (n1.x * n1.x + n1.z * n1.z < tol2) {
    if (!n1.copied) offer(A, n1.tau, trig, ord, n1.gx, n1.gz, true);
    return;
  }
  if (n2.x * n2.x + n2.z * n2.z < tol2) {
    if (!n2.copied) offer(A, n2.tau, trig, ord, n2.gx, n2.gz, true);
    return;
  }
  if (n1.tau > A.best.t && n1.tau > A.pre_min) return;
  {
    const float ex = n2.x - n1.x, ez = n2.z - n1.z;
    if (ex * ex + ez * ez < tol2) {
      // time_from_1_node2d of the later member, in this pair's event slot
      const float dist = sqrtf(n1.x * n1.x + n1.z * n1.z);
      const float t = n1.tau + dist * (2.0f * rcp(vu + n1.v));
      const float ig = rcp(dist * vu);
      offer(A, t, trig, ord, -n1.x * ig, -n1.z * ig, false);
      return;
    }
  }
  const double r1x = n1.x, r1z = n1.z, r2x = n2.x, r2z = n2.z;
  const double t1 = n1.tau, t2 = n2.tau;
  const double v12 = 0.5 * ((double)n1.v + (double)n2.v);
  const double dx = (r1x - r2x) / v12, dz = (r1z - r2z) / v12;
  const double s = (t1 - t2) / (dx * dx + dz * dz);
  const double px = s * dx, pz = s * dz;
  const double qx = -dz, qz = dx;
  const double ae = qx * qx + qz * qz, be = 2.0 * (px * qx + pz * qz);
  const double ce = px * px + pz * pz - 1.0;
  const double det = be * be - 4.0 * ae * ce;
  if (det < 0.0) return;
  const double sq = sqrt(det), ia = 0.5 / ae;
  double n1x = -r1z, n1z = r1x;
  double l = rsqrt(n1x * n1x + n1z * n1z);
  n1x *= l; n1z *= l;
  if (n1x * r2x + n1z * r2z < 0.0) { n1x = -n1x; n1z = -n1z; }
  double n2x = -r2z, n2z = r2x;
  l = rsqrt(n2x * n2x + n2z * n2z);
  n2x *= l; n2z *= l;
  if (n2x * r1x + n2z * r1z < 0.0) { n2x = -n2x; n2z = -n2z; }
  const double ivb = 2.0 / ((double)vu + (double)n1.v);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double uu = (-be + (k == 0 ? sq : -sq)) * ia;
    const double wx = px + uu * qx, wz = pz + uu * qz;
    if (wx * n1x + wz * n1z <= 0.0 && wx * n2x + wz * n2z <= 0.0) {
      const double t = t1 - (wx * r1x + wz * r1z) * ivb;
      if (t >= t1) {
        const float ig = rsqrtf((float)(wx * wx + wz * wz)) * rcp(n1.v);
        offer(A, (float)t, trig, ord, (float)wx * ig, (float)wz * ig, false);
      }
    }
  }
}

// All candidates of one cut cell whose members are listed in the reference's
// connected-node order; within one trigger the reference evaluates the point
// update of the trigger first, then its pairs with the earlier members.
__device__ __forceinline__ void cell_generic(const Member* mem, int nm, float vu, float tol2,
                                             int cbase, CutAcc& A) {
  for (int a = 0; a < nm; ++a)
    if (mem[a].single_ok) from_1(mem[a], vu, tol2, cbase, A);
  for (int a = 0; a < nm; ++a)
    for (int b = a + 1; b < nm; ++b) {
      const int early = mem[a].tau < mem[b].tau ? a : b;
      from_2(mem[a], mem[b], cbase + 1 + early, vu, tol2, A);
    }
}

struct TileCtx {
  const DevField* F;
  int c0, r0;          // tile origin (column, bbox row)
  int frozen_local;    // smem index of the frozen node, -1 if none here
  int z_lo;            // band's first grid row
  float h, tol2;
  bool mono;           // only accept decreases (tiles revisited many times)
};

// (hi, lo) = tref + tau exactly (TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& hi, float& lo) {
  hi = a + b;
  const float bb = hi - a;
  lo = (a - (hi - bb)) + (b - bb);
}

// Members of an irregular cell as seen from a grid node at smem (i,j), in the
// reference's connected-node order: top-interface node, bottom-interface
// node, then the grid corners (x outer, z inner).
__device__ int gather_cell_grid(const TileSmem& S, const TileCtx& C, uint32_t code, int c,
                                int i, int j, float tref, Member* mem) {
  const int ci = i - ((c & 1) ? 1 : 0), cj = j - (c >= 2 ? 1 : 0);
  const float h = C.h;
  int nm = 0;
  const int kk = cj;  // interface entry of the cell's column
  const int zrow_u = C.r0 - kHalo + i + C.z_lo;   // absolute row of the node
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const bool has = side == 0 ? (code & (1u << (12 + c))) : (code & (1u << (16 + c)));
    if (!has) continue;
    if (S.iTh[side][kk] >= kReachedF) continue;
    Member& m = mem[nm++];
    m.x = (float)(kk - j) * h;
    m.z = (float)(S.izc[side][kk] - zrow_u) * h + S.idz[side][kk];
    m.tau = (S.iTh[side][kk] - tref) + S.iTl[side][kk];
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
      m.x = (float)(jj - j) * h;
      m.z = (float)(ii - i) * h;
      m.tau = (S.Th[s] - tref) + S.Tl[s];
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

__device__ __forceinline__ NewV no_change() {
  NewV v;
  v.sig = 0; v.write = false; v.th = kHugeF; v.tl = 0.0f; v.gx = 0.0f; v.gz = 0.0f;
  v.suspect = false; v.copy = false;
  return v;
}

// New value = min(seed, tref + best offset), classified against the current
// (hi, lo) value.  Seeds are stored as (hi, lo, gx, gz) and precede every
// candidate in the reference's order.  sus_t: offset of the regular candidate
// whose suspect flag the node would keep (a seed at or below it means that
// update never happened).  In monotone mode only decreases are taken.
__device__ __forceinline__ NewV finish(float tref, const Cand& w, bool sus, float sus_t,
                                       const float4* seedp, float cur_h, float cur_l,
                                       bool cur_copy, bool mono) {
  NewV out = no_change();
  float th = kHugeF, tl = 0.0f, gx = w.gx, gz = w.gz;
  bool su = sus, cp = w.copy;
  if (w.t < kReachedF && tref < kReachedF) two_sum(tref, w.t, th, tl);
  if (seedp) {
    const float4 sd = *seedp;
    if (sd.x < kReachedF) {
      if (th >= kReachedF || (sd.x - th) + (sd.y - tl) <= 0.0f) {
        th = sd.x; tl = sd.y; gx = sd.z; gz = sd.w; su = false; cp = false;
      } else if (su && (sd.x - tref) + sd.y <= sus_t) {
        su = false;
      }
    }
  }
  if (th >= kReachedF) {
    // nothing reaches the node (any more)
    if (cur_h < kReachedF && !mono) { out.write = true; out.sig = 2; }
    return out;
  }
  if (cur_h >= kReachedF) {
    out.th = th; out.tl = tl; out.gx = gx; out.gz = gz; out.suspect = su; out.copy = cp;
    out.write = true; out.sig = 2;
    return out;
  }
  const float d = (th - cur_h) + (tl - cur_l);
  if (mono && !(d < 0.0f)) return out;
  out.th = th; out.tl = tl; out.gx = gx; out.gz = gz; out.suspect = su; out.copy = cp;
  const float ad = fabsf(d);
  out.write = th != cur_h || tl != cur_l || cp != cur_copy;
  out.sig = ad > kSigDT ? 2 : (ad > (float)kLocalDT ? 1 : 0);
  return out;
}

// Update of a grid node at smem (i,j); reads shared memory only (plus the
// seed of a seeded node).
__device__ NewV update_grid(const TileSmem& S, const TileCtx& C, int i, int j, uint32_t code,
                            int slot) {
  const int s = i * kSP + j;
  if (!(code & kUpdatable) || s == C.frozen_local) return no_change();
  const float vu = S.vel[s];
  const float h = C.h;
  float tref = kHugeF;
  tref = fminf(tref, S.vel[s - 1] > 0.0f ? S.Th[s - 1] : kHugeF);
  tref = fminf(tref, S.vel[s + 1] > 0.0f ? S.Th[s + 1] : kHugeF);
  tref = fminf(tref, S.vel[s - kSP] > 0.0f ? S.Th[s - kSP] : kHugeF);
  tref = fminf(tref, S.vel[s + kSP] > 0.0f ? S.Th[s + kSP] : kHugeF);
  const bool any_irr = (code & 0xF00u) != 0;
  const float4* seedp = (S.fl[s] & kFlagSeed) ? C.F->seed + slot : nullptr;
  const bool cur_copy = (S.fl[s] & kFlagCopy) != 0;
  if (any_irr) {
    // interface members of the cut cells can be the only reached neighbours
    const int kk0 = j - 1, kk1 = j;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      tref = fminf(tref, S.iTh[side][kk0]);
      tref = fminf(tref, S.iTh[side][kk1]);
    }
    tref = fminf(tref, fminf(fminf(S.Th[s - kSP - 1], S.Th[s - kSP + 1]),
                             fminf(S.Th[s + kSP - 1], S.Th[s + kSP + 1])));
  }
  if (tref >= kReachedF)
    return finish(kHugeF, no_cand(), false, kHugeF, seedp, S.Th[s], S.Tl[s], cur_copy, C.mono);
  const float two_h = 2.0f * h, ih = 1.0f / h;
  Nb L, R, U, D;
  nb_eval(S, s - 1, s - 2, vu, tref, two_h, +ih, C.frozen_local, L);
  nb_eval(S, s + 1, s + 2, vu, tref, two_h, -ih, C.frozen_local, R);
  nb_eval(S, s - kSP, s - 2 * kSP, vu, tref, two_h, +ih, C.frozen_local, U);
  nb_eval(S, s + kSP, s + 2 * kSP, vu, tref, two_h, -ih, C.frozen_local, D);
  // cells: c0 = (R,D), c1 = (R,U), c2 = (L,D), c3 = (L,U)
  if (!any_irr) {
    // update_time2d's quadrant loop: (L,U), (R,U), (L,D), (R,D)
    Cand best = no_cand();
    if (code & (1u << 7)) quadrant(L, U, 0, best);
    if (code & (1u << 5)) quadrant(R, U, 1, best);
    if (code & (1u << 6)) quadrant(L, D, 2, best);
    if (code & (1u << 4)) quadrant(R, D, 3, best);
    return finish(tref, best, best.suspect, best.t, seedp, S.Th[s], S.Tl[s], cur_copy, C.mono);
  }
  // next to a cut cell of the region's own interfaces: connected cells in the
  // order c0..c3; regular cells first (their best sets the suspect rule)
  Cand rb = no_cand();
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (!(code & (1u << (4 + c))) || (code & (1u << (8 + c)))) continue;
    quadrant((c >= 2) ? L : R, (c & 1) ? U : D, c * 32, rb);
  }
  CutAcc A;
  A.best = no_cand();
  A.pre_min = kHugeF;
  A.rtrig = rb.trig;
  A.rord = rb.ord;
#pragma unroll 1
  for (int c = 0; c < 4; ++c) {
    if (!(code & (1u << (4 + c))) || !(code & (1u << (8 + c)))) continue;
    Member mem[6];
    const int nm = gather_cell_grid(S, C, code, c, i, j, tref, mem);
    cell_generic(mem, nm, vu, C.tol2, c * 32, A);
  }
  const bool reg_wins = rb.t < A.best.t || (rb.t == A.best.t && earlier_event(rb.trig, rb.ord, A.best));
  const Cand& w = reg_wins ? rb : A.best;
  const bool sus = rb.suspect && (reg_wins || rb.t < A.pre_min);
  return finish(tref, w, sus, rb.t, seedp, S.Th[s], S.Tl[s], cur_copy, C.mono);
}

// Update of an interface node (side, smem interface entry k) owned by the tile.
__device__ NewV update_iface(const TileSmem& S, const TileCtx& C, int side, int k, int slot) {
  const uint32_t code = S.icode[side][k];
  if (!(code & kUpdatable)) return no_change();
  const int izc = S.izc[side][k];
  const float h = C.h;
  const int ci = izc - C.z_lo - C.r0 + kHalo;   // smem row of the cell's top
  const int cj = k;                              // smem column of the cell's left
  const float zu = S.idz[side][k];               // node depth relative to z(izc)
  // reference time: smallest member time
  float tref = kHugeF;
  const int o = side ^ 1;
  const bool has_o = o == 0 ? (code & (1u << 12)) : (code & (1u << 16));
  if (has_o) tref = fminf(tref, S.iTh[o][k]);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int ii = ci + b, jj = cj + a;
      if (ii < 0 || ii >= kSR || jj < 0 || jj >= kSP - 1) continue;
      const int s = ii * kSP + jj;
      if (S.vel[s] > 0.0f) tref = fminf(tref, S.Th[s]);
    }
  const float4* seedp = (S.ifl[side][k] & kFlagSeed) ? C.F->seed + slot : nullptr;
  const bool cur_copy = (S.ifl[side][k] & kFlagCopy) != 0;
  if (tref >= kReachedF)
    return finish(kHugeF, no_cand(), false, kHugeF, seedp, S.iTh[side][k], S.iTl[side][k],
                  cur_copy, C.mono);
  // members in connected-node order: the other interface's node, then the
  // grid corners (x outer, z inner)
  Member mem[6];
  int nm = 0;
  if (has_o && S.iTh[o][k] < kReachedF) {
    Member& m = mem[nm++];
    m.x = 0.0f;
    m.z = (float)(S.izc[o][k] - izc) * h + S.idz[o][k] - zu;
    m.tau = (S.iTh[o][k] - tref) + S.iTl[o][k];
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
      m.x = (float)a * h;
      m.z = (float)b * h - zu;
      m.tau = (S.Th[s] - tref) + S.Tl[s];
      m.gx = S.gx[s];
      m.gz = S.gz[s];
      m.v = S.vel[s];
      m.single_ok = (s != C.frozen_local);
      m.copied = (S.fl[s] & kFlagCopy) != 0;
    }
  CutAcc A;
  A.best = no_cand();
  A.pre_min = kHugeF;
  A.rtrig = -kHugeF;
  A.rord = -1;
  if (nm > 0) cell_generic(mem, nm, S.ivel[side][k], C.tol2, 0, A);
  return finish(tref, A.best, false, kHugeF, seedp, S.iTh[side][k], S.iTl[side][k], cur_copy,
                C.mono);
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

}  // namespace fmt2d
