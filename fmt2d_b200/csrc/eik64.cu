// FP64 eikonal solver: the reference's fast-marching stencil solved to its
// fixed point by data-parallel relaxation, one thread block per time field.
//
// The candidate arithmetic (eik_eval.cuh) gives every node the smallest of
// its seed and of the candidate times its fast-marching update events
// produce.  The solve is a fast iterative method over a field's active list:
// each step evaluates every listed node once (a thread per node), commits the
// new values and lists the nodes a changed node can move.  A time window
// bounds what may be committed: a node whose new time lies beyond it waits
// (it records the time and stays listed; until an input changes or the
// window reaches that time, listing it costs a compare), and the window moves
// on only after a step in which nothing inside it changed, so nodes settle in
// time slices as the heap accepts them.  When the list is empty every node is
// at the fixed point; a separate check of every node (k_verify) re-lists any
// that is not.
//
// One thread block owns a field for the whole solve: the lists, the
// "listed" bitset and the window live in shared memory, steps are separated
// by block barriers instead of kernel launches, and the field's front stays
// in the SM's L1.  A step has four phases separated by barriers: evaluate
// (reads committed state only, stages new values per slot), arbitrate,
// commit, spread.  Evaluations never see a value of the same step, so the
// result does not depend on thread timing: a forward is bit-identical run to
// run.
//
// Arithmetic is FP64 with the reference's expression order; this file is
// compiled with --fmad=false so candidate times are bit-identical to the
// FP64 restatement's.
#include <algorithm>
#include <climits>
#include <mutex>
#include "eik64.cuh"
#include "eik_eval.cuh"
#include "model.h"

namespace fmt2d {

namespace {

using namespace ev;

// ---------------------------------------------------------------- field solve
// Threads of a field's solve block: k_solve is instantiated for each size;
// the result does not depend on it (no evaluation sees a value of its own
// step), only the time does, so a context may pick the fastest for its
// workload (e64_solve_sizes, fmt2d_autotune).
constexpr int kSolveSizes[3] = {256, 384, 512};
constexpr int kSolveDefault = 384;
constexpr unsigned kLCap = 4096;          // entries of each list held in shared memory
constexpr unsigned kCCap = 2048;          // commit entries held in shared memory
constexpr int kTileRows = 8;              // a tile: 8 slot rows x 32 slot columns (one bitset word per row)
constexpr int kTilesMax = 12288;          // tiles per field (tile minima live in shared memory)
constexpr size_t kSmemMax = 227 * 1024;   // dynamic shared memory of the solve block
constexpr unsigned kSpreadBit = 0x80000000u;   // commit entry: the node moved
constexpr unsigned kLostBit = 0x40000000u;     // commit entry: lost arbitration, listed again
constexpr unsigned kSlotMask = 0x3fffffffu;
constexpr unsigned long long kNone = ULLONG_MAX;

struct SolveShared {
  Fld64 F;
  unsigned cnt[2];                 // list lengths
  unsigned nc[2];                  // commit list length, by step parity
  int changed[2];                  // a committed write moved a node, by step parity
  int cutstep[2];                  // the step evaluated a node next to an interface
  unsigned nready[2];              // tiles to release, by release parity
  unsigned long long gmin[2];      // earliest waiting time (bits of a positive double)
  int err;
};

__device__ __forceinline__ unsigned get_entry(const unsigned* sl, const unsigned* ov, unsigned i) {
  return i < kLCap ? sl[i] : ov[i - kLCap];
}

// List slot s unless it is listed already (bits: one bit per slot).
__device__ __forceinline__ void push(unsigned* bits, unsigned* sl, unsigned* ov, unsigned* cnt,
                                     unsigned s) {
  const unsigned bit = 1u << (s & 31);
  if (atomicOr(bits + (s >> 5), bit) & bit) return;
  const unsigned p = atomicAdd(cnt, 1u);
  if (p < kLCap) sl[p] = s;
  else ov[p - kLCap] = s;
}

__device__ __forceinline__ unsigned long long dbits(double d) {
  return (unsigned long long)__double_as_longlong(d);
}

__host__ __device__ inline int tiles_of(const Fld64& F) {
  return ((F.H + 2 + kTileRows - 1) / kTileRows) * (F.pitch / 32);
}

// Solve every field of the batch from its list_in (one block per field).
//
// Waiting nodes: a node whose new time lies beyond the window records it in
// pend and sets its bit in the waiting bitset; each tile of 8 x 32 slots
// keeps the smallest waiting time of its nodes.  When the window moves on,
// the tiles it has reached are scanned (a warp per tile) and their nodes
// that are due are listed, so a waiting node costs nothing until then.  A
// waiting node whose input changes is listed at once (its recorded time was
// computed from the old value).
//
// Shared memory: the two lists, the commit list, the tile minima and the
// list of tiles to scan, and (when they fit) the listed and waiting bitsets;
// smem_bits is the bitset size in words that fits, larger fields use their
// global bitsets.
template <int kSolveThreads>
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_solve(Fld64* fields, int nf, int smem_bits, int nsmem, int tiles_cap, long long max_steps,
            unsigned long long* ctr) {
  constexpr int kSolveWarps = kSolveThreads / 32;
  constexpr int kHalfWarps = kSolveThreads / 16;
  extern __shared__ __align__(16) unsigned char dsm_raw[];
  __shared__ SolveShared sh;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int hw = tid >> 4, hl = tid & 15;                 // half-warp, its lane
  const unsigned hmask = 0xffffu << (16 * (hw & 1));
  if (tid == 0) {
    sh.F = fields[blockIdx.x];
    sh.cnt[0] = sh.cnt[1] = 0u;
    sh.nc[0] = sh.nc[1] = 0u;
    sh.changed[0] = sh.changed[1] = 0;
    sh.cutstep[0] = sh.cutstep[1] = 0;
    sh.nready[0] = sh.nready[1] = 0u;
    sh.gmin[0] = sh.gmin[1] = kNone;
    sh.err = 0;
  }
  __syncthreads();
  const Fld64& F = sh.F;
  const unsigned ns = (unsigned)F.nslots();
  const unsigned nbw = (ns + 31u) >> 5;
  const int tcols = F.pitch / 32, ntiles = tiles_of(F);
  unsigned long long* tmin = reinterpret_cast<unsigned long long*>(dsm_raw);
  unsigned* sl[2];
  sl[0] = reinterpret_cast<unsigned*>(tmin + tiles_cap);
  sl[1] = sl[0] + kLCap;
  unsigned* scl = sl[1] + kLCap;
  unsigned short* ready = reinterpret_cast<unsigned short*>(scl + kCCap);
  unsigned* sbits = reinterpret_cast<unsigned*>(ready + tiles_cap);
  // the bitsets in shared memory, as many as fit in order of use: listed
  // (atomics on every push), moving (read by arbitration), waiting
  const int nloc = nbw <= (unsigned)smem_bits ? nsmem : 0;
  unsigned* bits = nloc >= 1 ? sbits : F.inq;
  unsigned* mbits = nloc >= 2 ? sbits + smem_bits : F.moving;
  unsigned* wbits = nloc >= 3 ? sbits + 2 * smem_bits : F.wait;
  // a field without a window never holds a node back: nothing waits
  const bool windowed = F.clock[1] < kReachD;
  unsigned* ov[2] = {F.over, F.over + ns};
  unsigned* cov = F.over + 2 * (size_t)ns;
  for (unsigned w = tid; w < nbw; w += kSolveThreads) {
    bits[w] = 0u;
    wbits[w] = 0u;
    mbits[w] = 0u;
  }
  for (int t = tid; t < ntiles; t += kSolveThreads) tmin[t] = kNone;
  __syncthreads();
  {
    const unsigned n0 = F.cnt[0];
    for (unsigned i = tid; i < n0; i += kSolveThreads)
      push(bits, sl[0], ov[0], &sh.cnt[0], F.list_in[i]);
  }
  __syncthreads();
  double W = F.clock[0];
  const double wstep = F.clock[1];
  unsigned long long n_eval = 0, n_write = 0, n_rel = 0, n_cut = 0;
  unsigned long long cyc[5] = {0, 0, 0, 0, 0};   // thread 0: cycles per phase
  unsigned long long steps_cut = 0;
  long long c0 = clock64();
  int cur = 0, rp = 0;
  long long it = 0;
  for (;; ++it) {
    const unsigned n = sh.cnt[cur];
    if (n == 0u) break;
    if (it >= max_steps) {
      if (tid == 0) sh.err = 1;
      break;
    }
    const int par = (int)(it & 1), nxt = cur ^ 1;
    // evaluate: read committed state only, stage what changes
    for (unsigned i = tid; i < n; i += kSolveThreads) {
      const unsigned s = get_entry(sl[cur], ov[cur], i);
      atomicAnd(bits + (s >> 5), ~(1u << (s & 31)));
      const uint32_t code = FMT_RO(F.code + s);
      const NewV nv = evaluate(F, (int)s);
      ++n_eval;
      if (!(code & kFullyRegular)) {
        ++n_cut;
        sh.cutstep[par] = 1;
      }
      if (!nv.write) {
        F.pend[s] = -1.0;
        continue;
      }
      if (nv.T < kReachD && nv.T > W) {   // beyond the window: wait for it
        F.pend[s] = nv.T;
        atomicOr(wbits + (s >> 5), 1u << (s & 31));
        const int row = (int)(s / (unsigned)F.pitch), col = (int)(s - (unsigned)row * F.pitch);
        atomicMin(tmin + (row / kTileRows) * tcols + (col >> 5), dbits(nv.T));
        continue;
      }
      F.pend[s] = -1.0;
      F.Tn[s] = nv.T;
      F.Gn[s] = make_double2(nv.gx, nv.gz);
      F.fln[s] = (uint8_t)((F.fl[s] & kFlSeed) | (nv.copy ? kFlCopy : 0) | (nv.sus ? kFlSusp : 0));
      const unsigned p = atomicAdd(&sh.nc[par], 1u);
      const unsigned e = s | (nv.spread ? kSpreadBit : 0u);
      if (p < kCCap) scl[p] = e;
      else cov[p - kCCap] = e;
      if (nv.spread) {
        sh.changed[par] = 1;
        F.claim[s] = dbits(nv.T);
        atomicOr(mbits + (s >> 5), 1u << (s & 31));
      }
    }
    __syncthreads();
    if (tid == 0) {
      const long long c1 = clock64();
      cyc[0] += (unsigned long long)(c1 - c0);
      if (sh.cutstep[par]) {
        cyc[2] += (unsigned long long)(c1 - c0);
        ++steps_cut;
      }
      c0 = c1;
    }
    // arbitrate: a moving node commits only if no node that reads it (the
    // nodes it reads are among them) moves to a smaller (time, slot) in the
    // same step; the others are listed again.  Of two nodes that feed each
    // other the earlier goes first, as the heap accepts them, so a pair that
    // hands a time back and forth (a zero-increment update) cannot swap
    // values forever.
    const unsigned nc = sh.nc[par];
    if (tid == 0) {
      sh.cnt[cur] = 0u;
      sh.nc[par ^ 1] = 0u;
      sh.changed[par ^ 1] = 0;
      sh.cutstep[par ^ 1] = 0;
    }
    // (a half-warp per moved node, a lane per node that reads it); a winner
    // commits at once (nothing reads committed times in this phase; the old
    // time stays in Tn for the spread threshold)
    for (unsigned j = hw; j < nc; j += kHalfWarps) {
      const unsigned e = j < kCCap ? scl[j] : cov[j - kCCap];
      const int s = (int)(e & kSlotMask);
      bool lose = false;
      if (e & kSpreadBit) {
        // only neighbours that move this step hold a claim (moving bitset)
        const int t = neighbour_slot(F, s, hl);
        bool l = false;
        if (t >= 0 && ((mbits[t >> 5] >> (t & 31)) & 1u)) {
          const unsigned long long ks = F.claim[s], kt = F.claim[t];
          l = kt < ks || (kt == ks && t < s);
        }
        lose = (__ballot_sync(hmask, l) & hmask) != 0u;
      }
      if (hl == 0) {
        if (lose) {
          if (j < kCCap) scl[j] = e | kLostBit;
          else cov[j - kCCap] = e | kLostBit;
          push(bits, sl[nxt], ov[nxt], &sh.cnt[nxt], (unsigned)s);
        } else {
          if (e & kSpreadBit) ++n_write;
          const double old = F.T[s];
          F.T[s] = F.Tn[s];
          F.Tn[s] = old;
          F.G[s] = F.Gn[s];
          F.fl[s] = F.fln[s];
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      const long long c1 = clock64();
      cyc[1] += (unsigned long long)(c1 - c0);
      c0 = c1;
    }
    // spread: every candidate of a node u that involves node v is at or above
    // v's time, so a change of v from a to b can only move nodes at or above
    // min(a, b); those below are not listed unless they wait with a time
    // computed from the old value, which is dropped
    for (unsigned j = hw; j < nc; j += kHalfWarps) {
      const unsigned e = j < kCCap ? scl[j] : cov[j - kCCap];
      if (!(e & kSpreadBit)) continue;
      const int s = (int)(e & kSlotMask);
      if (hl == 0) atomicAnd(mbits + (s >> 5), ~(1u << (s & 31)));   // readers are done
      if (e & kLostBit) continue;
      const int t = spread_target_at(F, s, hl);
      if (t < 0) continue;
      const double thr = fmin(F.Tn[s], F.T[s]);
      // a waiting target (its bit may be stale) drops the time it waits with
      const bool waiting = windowed && ((wbits[t >> 5] >> (t & 31)) & 1u);
      if (waiting) F.pend[t] = -1.0;
      if (waiting || !(F.T[t] < thr)) push(bits, sl[nxt], ov[nxt], &sh.cnt[nxt], (unsigned)t);
    }
    __syncthreads();
    if (tid == 0) {
      const long long c1 = clock64();
      cyc[3] += (unsigned long long)(c1 - c0);
      c0 = c1;
    }
    // the window moves on after a step that changed nothing inside it (or
    // listed nothing); the tiles it reaches release their due nodes, and when
    // none is due it jumps to the earliest waiting time
    const bool chg = sh.changed[par] != 0;
    if (!chg || sh.cnt[nxt] == 0u) {
      if (!chg) W += wstep;
      for (;;) {
        const int q = rp & 1;
        ++rp;
        for (int t = tid; t < ntiles; t += kSolveThreads)
          if (tmin[t] != kNone && __longlong_as_double((long long)tmin[t]) <= W)
            ready[atomicAdd(&sh.nready[q], 1u)] = (unsigned short)t;
        __syncthreads();
        const unsigned nr = sh.nready[q];
        if (tid == 0) {
          sh.nready[q ^ 1] = 0u;
          sh.gmin[q ^ 1] = kNone;
        }
        for (unsigned k = warp; k < nr; k += kSolveWarps) {
          const int t = ready[k];
          const int r0 = (t / tcols) * kTileRows, c0 = (t % tcols) * 32;
          // lane l takes column c0 + l of the tile's rows; the rows' loads
          // are issued together
          unsigned word[kTileRows];
          double pd[kTileRows];
#pragma unroll
          for (int rr = 0; rr < kTileRows; ++rr)
            word[rr] = r0 + rr < F.H + 2 ? wbits[(unsigned)((r0 + rr) * F.pitch + c0) >> 5] : 0u;
#pragma unroll
          for (int rr = 0; rr < kTileRows; ++rr)
            pd[rr] = (word[rr] >> lane) & 1u ? F.pend[(r0 + rr) * F.pitch + c0 + lane] : 0.0;
          unsigned long long m = kNone;
#pragma unroll
          for (int rr = 0; rr < kTileRows; ++rr) {
            const bool set = (word[rr] >> lane) & 1u;
            bool clear = false;
            if (set) {
              if (pd[rr] < 0.0) {
                clear = true;                 // listed since (an input changed)
              } else if (pd[rr] <= W) {
                clear = true;
                push(bits, sl[nxt], ov[nxt], &sh.cnt[nxt], (unsigned)((r0 + rr) * F.pitch + c0 + lane));
                ++n_rel;
              } else {
                m = min(m, dbits(pd[rr]));
              }
            }
            const unsigned cm = __ballot_sync(0xffffffffu, clear);
            if (lane == 0 && cm) wbits[(unsigned)((r0 + rr) * F.pitch + c0) >> 5] = word[rr] & ~cm;
          }
#pragma unroll
          for (int o = 16; o; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
          if (lane == 0) tmin[t] = m;
        }
        __syncthreads();
        if (sh.cnt[nxt] != 0u) break;
        // nothing due: the earliest waiting time, if any
        unsigned long long m = kNone;
        for (int t = tid; t < ntiles; t += kSolveThreads) m = min(m, tmin[t]);
        if (m != kNone) atomicMin(&sh.gmin[q], m);
        __syncthreads();
        const unsigned long long g = sh.gmin[q];
        if (g == kNone) break;
        W = fmax(W, __longlong_as_double((long long)g));
      }
      if (tid == 0) {
        const long long c1 = clock64();
        cyc[4] += (unsigned long long)(c1 - c0);
        c0 = c1;
      }
    }
    cur = nxt;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    n_eval += __shfl_xor_sync(0xffffffffu, n_eval, o);
    n_write += __shfl_xor_sync(0xffffffffu, n_write, o);
    n_rel += __shfl_xor_sync(0xffffffffu, n_rel, o);
    n_cut += __shfl_xor_sync(0xffffffffu, n_cut, o);
  }
  if (lane == 0 && ctr) {
    atomicAdd(ctr + kCtrCut, n_cut);
    atomicAdd(ctr + kCtrEval, n_eval);
    atomicAdd(ctr + kCtrWrite, n_write);
    atomicAdd(ctr + kCtrPass, n_rel);
  }
  __syncthreads();
  if (tid == 0) {
    F.clock[0] = W;
    F.cnt[0] = 0u;   // start list consumed; the check refills it
    F.cnt[1] = 0u;
    F.cnt[3] = (unsigned)(it < 0xffffffffll ? it : 0xffffffffll);
    if (sh.err) F.cnt[2] = 1u;
    if (ctr) {
      for (int k = 0; k < 5; ++k) atomicAdd(ctr + kCtrCycEval + k, cyc[k]);
      atomicAdd(ctr + kCtrStepsCut, steps_cut);
      atomicAdd(ctr + kCtrSteps, (unsigned long long)it);
      atomicMax(ctr + kCtrMaxSteps, (unsigned long long)it);
    }
  }
}

// Append slot s to the field's start list unless it is there already
// (F.inq zeroed before the kernel that appends).
__device__ __forceinline__ void list_start(const Fld64& F, unsigned s) {
  const unsigned bit = 1u << (s & 31);
  if (atomicOr(F.inq + (s >> 5), bit) & bit) return;
  F.list_in[atomicAdd(F.cnt, 1u)] = s;
}

// Fixed-point check of every node (window ignored): a node whose update
// would change it is listed and counted.
__global__ void k_verify(Fld64* fields, int nf) {
  const Fld64& F = fields[blockIdx.y];
  const int ns = F.nslots();
  unsigned nbad = 0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    if ((s % F.pitch) >= F.nx) continue;
    const NewV nv = evaluate(F, s);
    if (nv.write) {
      ++nbad;
      list_start(F, (unsigned)s);
    }
  }
  if (nbad) atomicAdd(F.cnt + 1, nbad);
}

// List every seeded node and the nodes around it.
__global__ void k_queue_seeds(Fld64* fields, int nf) {
  const Fld64& F = fields[blockIdx.y];
  const int ns = F.nslots();
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    if ((s % F.pitch) >= F.nx || !(F.fl[s] & kFlSeed)) continue;
    list_start(F, (unsigned)s);
    int t[16];
    const int k = spread_targets(F, s, t);
    for (int q = 0; q < k; ++q) list_start(F, (unsigned)t[q]);
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
    F.pend[i] = -1.0;
    F.claim[i] = ULLONG_MAX;
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
  }
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
// The solved times the sweep replaces are saved first (pre, nx per field:
// the adjoint re-derives each node's winning update from them).
__global__ void k_headwave(Fld64* fields, const int* hw_slot, const double* hw_v, double dx_if,
                           int nx, double* scratch, const int* which, int nsel,
                           double* const* pre) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsel) return;
  Fld64& F = fields[which[q]];
  double* th = scratch + (size_t)q * nx;
  for (int n = 0; n < nx; ++n) th[n] = hw_slot[n] >= 0 ? F.T[hw_slot[n]] : kHugeD;
  if (pre && pre[q])
    for (int n = 0; n < nx; ++n) pre[q][n] = th[n];
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
void e64_start(Fld64* f, int nf, size_t max_slots, const double* step, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 256);
  k_queue_seeds<<<dim3(bx, nf), 256, 0, st>>>(f, nf);
  k_clock<<<nf, 256, 0, st>>>(f, nf, step);
}
// Dynamic shared memory of k_solve for a batch whose largest field has
// max_slots slots and max_tiles tiles (tiles_cap rounded up to a multiple of
// 8); smem_bits: words of each bitset kept in shared memory, nsmem: how many
// of the three bitsets (listed, moving, waiting, in that order) fit there
// (0: all in global memory).
static size_t solve_smem(size_t max_slots, int max_tiles, int* smem_bits, int* nsmem,
                         int* tiles_cap) {
  const int cap = (max_tiles + 7) / 8 * 8;
  const size_t fixed = (size_t)cap * sizeof(unsigned long long) +
                       (2 * (size_t)kLCap + kCCap) * sizeof(unsigned) +
                       (size_t)cap * sizeof(unsigned short);
  const size_t nbw = (max_slots + 31) / 32;
  const size_t room = fixed + 1024 < kSmemMax ? (kSmemMax - fixed - 1024) / sizeof(unsigned) : 0;
  const int n = nbw == 0 ? 0 : (int)std::min<size_t>(3, room / nbw);
  *smem_bits = n > 0 ? (int)nbw : 0;
  *nsmem = n;
  *tiles_cap = cap;
  return fixed + (size_t)n * nbw * sizeof(unsigned);
}
int e64_tiles(const Fld64& f) { return tiles_of(f); }
int e64_tiles_max() { return kTilesMax; }
// k_solve may use up to kSmemMax of dynamic shared memory.  The attribute is
// set once per device and instantiation: changing a kernel's attributes while
// it runs (a solve of another stage chain on another stream) waits for that
// kernel to finish, which would serialise the chains.
template <int NT>
static void solve_attr_once() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  // the opt-in limit covers static and dynamic shared memory together
  int optin = 0;
  cudaFuncAttributes fa;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, k_solve<NT>) != cudaSuccess)
    return;
  const int dyn = std::min<int>((int)kSmemMax, optin - (int)fa.sharedSizeBytes);
  if (cudaFuncSetAttribute(k_solve<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ==
      cudaSuccess)
    done[dev] = true;
}

template <int NT>
static void solve_launch(Fld64* f, int nf, int smem_bits, int nsmem, int cap, size_t bytes,
                         long long max_steps, unsigned long long* ctr, cudaStream_t st) {
  solve_attr_once<NT>();
  k_solve<NT><<<nf, NT, bytes, st>>>(f, nf, smem_bits, nsmem, cap, max_steps, ctr);
}

const int* e64_solve_sizes(int* n) {
  *n = 3;
  return kSolveSizes;
}

void e64_solve(Fld64* f, int nf, size_t max_slots, int max_tiles, long long max_steps,
               unsigned long long* ctr, int threads, cudaStream_t st) {
  int smem_bits = 0, nsmem = 0, cap = 0;
  const size_t bytes = solve_smem(max_slots, max_tiles, &smem_bits, &nsmem, &cap);
  if (threads == 256)
    solve_launch<256>(f, nf, smem_bits, nsmem, cap, bytes, max_steps, ctr, st);
  else if (threads == 512)
    solve_launch<512>(f, nf, smem_bits, nsmem, cap, bytes, max_steps, ctr, st);
  else
    solve_launch<kSolveDefault>(f, nf, smem_bits, nsmem, cap, bytes, max_steps, ctr, st);
}
void e64_verify(Fld64* f, int nf, size_t max_slots, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 512);
  k_verify<<<dim3(bx, nf), 256, 0, st>>>(f, nf);
}
void e64_finish(Fld64* f, int nf, size_t max_slots, const int* water_up, cudaStream_t st) {
  const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 512);
  k_final_grad<<<dim3(bx, nf), 256, 0, st>>>(f, nf);
  k_water_fix<<<dim3(64, nf), 128, 0, st>>>(f, water_up, nf);
}
void e64_headwave(Fld64* f, const int* hw_slot, const double* hw_v, double dx_if, int nx,
                  double* scratch, const int* which, int nsel, double* const* pre,
                  cudaStream_t st) {
  k_headwave<<<(nsel + 31) / 32, 32, 0, st>>>(f, hw_slot, hw_v, dx_if, nx, scratch, which, nsel, pre);
}
void e64_export(const double* T, const double2* G, const int* slot_of_node, int nnode, double* oT,
                double* ogx, double* ogz, cudaStream_t st) {
  k_export<<<(nnode + 255) / 256, 256, 0, st>>>(T, G, slot_of_node, nnode, oT, ogx, ogz);
}

}  // namespace fmt2d
