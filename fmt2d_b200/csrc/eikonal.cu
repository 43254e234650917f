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
// candidate of the current neighbour state) without a heap.
//
// Work is organised like a windowed Dijkstra over 32x32 tiles ("narrow band"):
//   * every tile keeps a bit mask of nodes whose inputs moved and a key, the
//     smallest time among them;
//   * each round a field's front is its smallest key, and only tiles with a
//     key inside [front, front + band] are visited (eik_front, eik_select);
//   * a visit (eik_visit, one warp, tile staged in shared memory with a 2-node
//     halo) relaxes its active nodes by directional Gauss-Seidel sweeps; a node
//     whose new time lies beyond the band is deferred (kept active, not
//     propagated), a changed node inside the band activates its stencil
//     neighbours, across the tile edge by setting bits in the neighbour tile.
// Values are replaced, not min-ed with their history, because the 2nd-order
// switch depends on neighbour gradients that are only final at the fixed
// point; a copy is only taken from a node whose own value is not a copy,
// which is what the heap's acceptance order guarantees for coincident nodes.
#include "eikonal_dev.cuh"

namespace fmt2d {

namespace {

__device__ __forceinline__ unsigned* tile_mask(const DevField& F, int t) {
  return F.act + (size_t)t * kTileWords;
}

// Mark nodes of a neighbour tile active and lower its key.
__device__ __forceinline__ void nb_activate(const DevField& F, int tx, int ty, int word,
                                            unsigned bits, unsigned key) {
  const DevRegion& R = F.R;
  if (!bits || tx < 0 || ty < 0 || tx >= R.tiles_x || ty >= R.tiles_y) return;
  const int t = ty * R.tiles_x + tx;
  atomicOr(tile_mask(F, t) + word, bits);
  atomicMin(F.tkey + t, key);
}

__device__ __forceinline__ unsigned dil1(unsigned m) { return m | (m << 1) | (m >> 1); }

}  // namespace

// Per field: the front (smallest pending key over its tiles) and the number
// of tiles with pending work (summed into *n_pending).
__global__ void eik_front(const DevField* fields, int nf, unsigned* n_pending) {
  const DevField& F = fields[blockIdx.x];
  const int nt = F.R.tiles_x * F.R.tiles_y;
  unsigned mn = kKeyNone, cnt = 0u;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    const unsigned k = F.tkey[t];
    if (k != kKeyNone) { mn = min(mn, k); ++cnt; }
  }
  mn = __reduce_min_sync(0xffffffffu, mn);
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  __shared__ unsigned smn[32], scnt[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { smn[w] = mn; scnt[w] = cnt; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    mn = l < nw ? smn[l] : kKeyNone;
    cnt = l < nw ? scnt[l] : 0u;
    mn = __reduce_min_sync(0xffffffffu, mn);
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if (l == 0) {
      *F.front = mn == kKeyNone ? kHugeF : __uint_as_float(mn);
      if (cnt) atomicAdd(n_pending, cnt);
    }
  }
}

// Queue every tile whose key lies inside its field's band.
__global__ void eik_select(const DevField* fields, int nf, int total_tiles, unsigned* queue,
                           unsigned* qlen) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total_tiles) return;
  const int fi = find_field(fields, nf, b);
  const DevField& F = fields[fi];
  const int t = b - F.tile_base;
  if (t >= F.R.tiles_x * F.R.tiles_y) return;
  const unsigned k = F.tkey[t];
  if (k == kKeyNone) return;
  const float lim = *F.front + F.band;
  if (k <= key_of(lim)) queue[atomicAdd(qlen, 1u)] = (unsigned)b;
}

// Persistent visits of the queued tiles.
__global__ void __launch_bounds__(32, 4) eik_visit(const DevField* __restrict__ fields, int nf,
                                                   const unsigned* queue, const unsigned* qlen,
                                                   unsigned* qhead, int max_passes,
                                                   unsigned long long* counters) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem& S = *reinterpret_cast<TileSmem*>(smem_raw);
  const int lane = threadIdx.x;
  const unsigned n_queued = *qlen;
  for (;;) {
    unsigned idx = 0;
    if (lane == 0) idx = atomicAdd(qhead, 1u);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= n_queued) break;
    const int b = (int)queue[idx];
    const int fi = find_field(fields, nf, b);
    const DevField& F = fields[fi];
    const DevRegion& R = F.R;
    const int t = b - F.tile_base;
    const int tx = t % R.tiles_x, ty = t / R.tiles_x;
    TileCtx C;
    C.F = &F;
    C.c0 = tx * kTW;
    C.r0 = ty * kTH;
    C.h = (float)R.dx;
    C.z_lo = R.z_lo;
    C.tol2 = (float)((0.01 * R.tol) * (0.01 * R.tol));
    C.frozen_local = -1;
    unsigned nvis = 0;
    if (lane == 0) nvis = F.tvis[t]++;
    C.mono = __shfl_sync(0xffffffffu, nvis, 0) >= kMonoVisits;
    const float band_end = *F.front + F.band;
    // take the pending work: key first, then the masks (a neighbour that adds
    // bits after this also lowers the key again)
    if (lane == 0) atomicExch(F.tkey + t, kKeyNone);
    __syncwarp();
    unsigned* gm = tile_mask(F, t);
    unsigned act = atomicExch(gm + lane, 0u);
    unsigned iw = lane < 2 ? atomicExch(gm + kTH + lane, 0u) : 0u;
    unsigned iact[2] = {__shfl_sync(0xffffffffu, iw, 0), __shfl_sync(0xffffffffu, iw, 1)};
    load_tile(S, C, F, lane);
    unsigned own[2];
    owned_ifaces(S, C, F, lane, own);
    const int nrows = min(kTH, R.H - C.r0);
    const unsigned cols = (C.c0 + kTW <= R.nx) ? 0xffffffffu : ((1u << (R.nx - C.c0)) - 1u);
    act = lane < nrows ? (act & cols) : 0u;
    iact[0] &= own[0];
    iact[1] &= own[1];
    unsigned defer = 0u, idefer[2] = {0u, 0u};
    unsigned defer_key = kKeyNone;
    // edge records: nodes that moved significantly next to each tile edge
    unsigned e_left = 0u, e_right = 0u, e_top = 0u, e_bot = 0u;   // rows / columns
    unsigned e_key = kKeyNone;
    bool e_tl = false, e_tr = false, e_bl = false, e_br = false;
    bool converged = false;
    unsigned n_pass = 0, n_steps = 0, n_upd = 0;
    for (int pass = 0; pass < max_passes; ++pass) {
      const unsigned rows_act = __ballot_sync(0xffffffffu, act != 0u);
      if (rows_act == 0u && iact[0] == 0u && iact[1] == 0u) { converged = true; break; }
      ++n_pass;
      const int dir = pass & 3;
      if (dir < 2) {
        // z sweep: lane = column, rows in sweep order
        unsigned todo = rows_act;
        while (todo) {
          const int r = dir == 0 ? __ffs(todo) - 1 : 31 - __clz(todo);
          const int slot = (C.r0 + r) * R.pitch + C.c0 + lane;
          for (int rep = 0; rep < 3; ++rep) {
            const unsigned m = __shfl_sync(0xffffffffu, act, r);
            if (!m) break;
            ++n_steps;
            n_upd += __popc(m);
            NewV nv = no_change();
            const bool mine = (m >> lane) & 1u;
            if (mine) {
              const uint32_t code = R.code[slot];
              if (code & kInRegion) nv = update_grid(S, C, r + kHalo, lane + kHalo, code, slot);
            }
            __syncwarp();
            if (nv.write) write_node(S, (r + kHalo) * kSP + lane + kHalo, nv);
            __syncwarp();
            const bool late = mine && nv.th < kReachedF && nv.th > band_end;
            const bool moved = mine && !late && nv.sig >= 1;
            const bool big = moved && nv.sig == 2;
            const unsigned dfr = __ballot_sync(0xffffffffu, late);
            const unsigned chg = __ballot_sync(0xffffffffu, moved);
            const unsigned sig = __ballot_sync(0xffffffffu, big);
            if (late) defer_key = min(defer_key, key_of(nv.th));
            if (big && (r < 2 || r >= kTH - 2 || lane < 2 || lane >= kTW - 2))
              e_key = min(e_key, key_of(nv.th));
            const int d = lane - r;
            if (d == 0) { act = (act & ~m) | (nb_x(chg) & cols); defer |= dfr; }
            else if (d == 1 || d == -1) act |= dil1(chg) & cols;
            else if (d == 2 || d == -2) act |= chg & cols;
            if (lane >= nrows) act = 0u;
            if (chg) { iact[0] |= dil1(chg) & own[0]; iact[1] |= dil1(chg) & own[1]; }
            if (sig) {
              if (r < 2) e_top |= sig;
              if (r >= kTH - 2) e_bot |= sig;
              if (sig & 0x3u) e_left |= 1u << r;
              if (sig & 0xC0000000u) e_right |= 1u << r;
              if (r < 2) { e_tl = e_tl || (sig & 0x3u); e_tr = e_tr || (sig & 0xC0000000u); }
              if (r >= kTH - 2) { e_bl = e_bl || (sig & 0x3u); e_br = e_br || (sig & 0xC0000000u); }
            }
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
          const int slot = (C.r0 + lane) * R.pitch + C.c0 + c;
          const unsigned bit = 1u << c;
          for (int rep = 0; rep < 3; ++rep) {
            const bool mine = (act >> c) & 1u;
            const unsigned mb = __ballot_sync(0xffffffffu, mine);
            if (!mb) break;
            ++n_steps;
            n_upd += __popc(mb);
            NewV nv = no_change();
            if (mine) {
              const uint32_t code = R.code[slot];
              if (code & kInRegion) nv = update_grid(S, C, lane + kHalo, c + kHalo, code, slot);
            }
            __syncwarp();
            if (nv.write) write_node(S, (lane + kHalo) * kSP + c + kHalo, nv);
            __syncwarp();
            const bool late = mine && nv.th < kReachedF && nv.th > band_end;
            const bool ch = mine && !late && nv.sig >= 1;
            const bool big = ch && nv.sig == 2;
            if (mine) act &= ~bit;
            if (late) { defer |= bit; defer_key = min(defer_key, key_of(nv.th)); }
            if (ch) act |= nb_x(bit) & cols;
            const bool u1 = __shfl_up_sync(0xffffffffu, ch, 1) && lane >= 1;
            const bool u2 = __shfl_up_sync(0xffffffffu, ch, 2) && lane >= 2;
            const bool d1 = __shfl_down_sync(0xffffffffu, ch, 1) && lane <= 30;
            const bool d2 = __shfl_down_sync(0xffffffffu, ch, 2) && lane <= 29;
            if (u1 || d1) act |= dil1(bit) & cols;
            if (u2 || d2) act |= bit & cols;
            if (lane >= nrows) act = 0u;
            if (__any_sync(0xffffffffu, ch)) {
              iact[0] |= (bit | (bit >> 1)) & own[0];
              iact[1] |= (bit | (bit >> 1)) & own[1];
            }
            const unsigned sg = __ballot_sync(0xffffffffu, big);
            if (sg) {
              if (c < 2) e_left |= sg;
              if (c >= kTW - 2) e_right |= sg;
              if (sg & 0x3u) e_top |= bit;
              if (sg & 0xC0000000u) e_bot |= bit;
              if (c < 2) { e_tl = e_tl || (sg & 0x3u); e_bl = e_bl || (sg & 0xC0000000u); }
              if (c >= kTW - 2) { e_tr = e_tr || (sg & 0x3u); e_br = e_br || (sg & 0xC0000000u); }
            }
            if (big && (lane < 2 || lane >= kTH - 2 || c < 2 || c >= kTW - 2))
              e_key = min(e_key, key_of(nv.th));
          }
          const unsigned nxt = __reduce_or_sync(0xffffffffu, act);
          if (dir == 2) todo = c >= 31 ? 0u : (nxt & ~((2u << c) - 1u));
          else todo = c == 0 ? 0u : (nxt & ((1u << c) - 1u));
        }
      }
      // interface nodes owned by the tile (lane = column)
      for (int rep = 0; rep < 2; ++rep) {
        if (!iact[0] && !iact[1]) break;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          NewV nv = no_change();
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
          const bool late = mine && nv.th < kReachedF && nv.th > band_end;
          const bool moved = mine && !late && nv.sig >= 1;
          const bool big = moved && nv.sig == 2;
          iact[side] &= ~__ballot_sync(0xffffffffu, mine);
          idefer[side] |= __ballot_sync(0xffffffffu, late);
          if (late) defer_key = min(defer_key, key_of(nv.th));
          const unsigned chg = __ballot_sync(0xffffffffu, moved);
          const unsigned sig = __ballot_sync(0xffffffffu, big);
          // a moved interface node re-activates the grid nodes around its cut cell
          const int rr_l = S.izc[side][k] - R.z_lo - C.r0;   // tile row of the cell's top
          unsigned todo = chg;
          while (todo) {
            const int q = __ffs(todo) - 1;
            todo &= todo - 1u;
            const int rr = __shfl_sync(0xffffffffu, rr_l, q);
            const int d = lane - rr;
            if (d >= -1 && d <= 2 && lane < nrows) {
              const unsigned qb = 1u << q;
              act |= (qb | (qb >> 1) | (qb << 1) | (qb << 2)) & cols;
            }
          }
          iact[side ^ 1] |= chg & own[side ^ 1];
          if (big) e_key = min(e_key, key_of(nv.th));
          // edges touched by the moved node's cut cell (rows rr..rr+1, columns k..k+1)
          if (sig) {
            const bool top_ = big && rr_l <= 1, bot_ = big && rr_l >= kTH - 3;
            const unsigned tops = __ballot_sync(0xffffffffu, top_);
            const unsigned bots = __ballot_sync(0xffffffffu, bot_);
            e_top |= dil1(tops);
            e_bot |= dil1(bots);
            if (sig & 0xC0000000u) {
              const int rq = __shfl_sync(0xffffffffu, rr_l, 31 - __clz(sig & 0xC0000000u));
              if (rq >= -1 && rq <= kTH - 1) e_right |= (0x3u << max(rq, 0)) | (rq < 0 ? 1u : 0u);
            }
            if (sig & 0x1u) {
              const int rq = __shfl_sync(0xffffffffu, rr_l, 0);
              if (rq >= -1 && rq <= kTH - 1) e_left |= (0x3u << max(rq, 0)) | (rq < 0 ? 1u : 0u);
            }
            e_tr = e_tr || (tops & 0xC0000000u);
            e_br = e_br || (bots & 0xC0000000u);
            e_tl = e_tl || (tops & 0x1u);
            e_bl = e_bl || (bots & 0x1u);
          }
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
    __syncwarp();
    // ---- pending work back into the tile: unconverged and deferred nodes
    if (!converged) {
      // the tile's key becomes the earliest time among its still-active nodes
      for (unsigned m = act; m; m &= m - 1u)
        defer_key = min(defer_key, key_of(S.Th[(lane + kHalo) * kSP + __ffs(m) - 1 + kHalo]));
#pragma unroll
      for (int side = 0; side < 2; ++side)
        if ((iact[side] >> lane) & 1u) defer_key = min(defer_key, key_of(S.iTh[side][lane + kHalo]));
      defer |= act;
      idefer[0] |= iact[0];
      idefer[1] |= iact[1];
    }
    const unsigned dk = __reduce_min_sync(0xffffffffu, defer_key);
    if (defer) atomicOr(gm + lane, defer);
    if (lane < 2 && idefer[lane]) atomicOr(gm + kTH + lane, idefer[lane]);
    const bool any_defer = __any_sync(0xffffffffu, defer != 0u) || idefer[0] || idefer[1];
    if (lane == 0 && any_defer) atomicMin(F.tkey + t, dk == kKeyNone ? key_of(band_end) : dk);
    // ---- neighbour tiles whose halo moved
    const unsigned ek = __reduce_min_sync(0xffffffffu, e_key);
    if (lane == 0) {
      const unsigned key = ek;
      const unsigned el = dil1(e_left), er = dil1(e_right);
      const unsigned et = dil1(e_top), eb = dil1(e_bot);
      if (et) {
        nb_activate(F, tx, ty - 1, kTH - 2, et, key);
        nb_activate(F, tx, ty - 1, kTH - 1, et, key);
        nb_activate(F, tx, ty - 1, kTH, et, key);      // its interface nodes
        nb_activate(F, tx, ty - 1, kTH + 1, et, key);
      }
      if (eb) {
        nb_activate(F, tx, ty + 1, 0, eb, key);
        nb_activate(F, tx, ty + 1, 1, eb, key);
      }
      if (el) {
        for (unsigned m = el; m; m &= m - 1u) nb_activate(F, tx - 1, ty, __ffs(m) - 1, 0xC0000000u, key);
        nb_activate(F, tx - 1, ty, kTH, 0x80000000u, key);
        nb_activate(F, tx - 1, ty, kTH + 1, 0x80000000u, key);
      }
      if (er)
        for (unsigned m = er; m; m &= m - 1u) nb_activate(F, tx + 1, ty, __ffs(m) - 1, 0x3u, key);
      if (e_tl) {
        nb_activate(F, tx - 1, ty - 1, kTH - 2, 0xC0000000u, key);
        nb_activate(F, tx - 1, ty - 1, kTH - 1, 0xC0000000u, key);
        nb_activate(F, tx - 1, ty - 1, kTH, 0x80000000u, key);
        nb_activate(F, tx - 1, ty - 1, kTH + 1, 0x80000000u, key);
      }
      if (e_tr) {
        nb_activate(F, tx + 1, ty - 1, kTH - 2, 0x3u, key);
        nb_activate(F, tx + 1, ty - 1, kTH - 1, 0x3u, key);
      }
      if (e_bl) {
        nb_activate(F, tx - 1, ty + 1, 0, 0xC0000000u, key);
        nb_activate(F, tx - 1, ty + 1, 1, 0xC0000000u, key);
      }
      if (e_br) {
        nb_activate(F, tx + 1, ty + 1, 0, 0x3u, key);
        nb_activate(F, tx + 1, ty + 1, 1, 0x3u, key);
      }
      if (counters) {
        atomicAdd(counters + 0, (unsigned long long)n_pass);
        atomicAdd(counters + 1, (unsigned long long)n_steps);
        atomicAdd(counters + 2, (unsigned long long)(converged ? 0 : 1));
        atomicAdd(counters + 3, (unsigned long long)n_upd);
      }
    }
    __syncwarp();
  }
}

// Final gradient pass over every tile of every field: re-evaluates each node
// on the converged field, writes the selected value's gradient and suspect
// flag (single-axis winner, refitted afterwards as the reference does when
// its heap is empty), and re-queues tiles where a node would still move by
// more than kSigDT (n_bad counts them; the caller then runs more rounds).
__global__ void __launch_bounds__(32, 4) eik_final(const DevField* __restrict__ fields, int nf,
                                                   float* const* gout, uint8_t* const* susp,
                                                   unsigned* n_bad) {
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
  C.h = (float)R.dx;
  C.z_lo = R.z_lo;
  C.tol2 = (float)((0.01 * R.tol) * (0.01 * R.tol));
  C.frozen_local = -1;
  C.mono = F.tvis[t] >= kMonoVisits;
  load_tile(S, C, F, lane);
  unsigned own[2];
  owned_ifaces(S, C, F, lane, own);
  float2* G = reinterpret_cast<float2*>(gout[fi]);
  uint8_t* SU = susp[fi];
  bool bad = false;
  unsigned bad_key = kKeyNone;
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
      if (nv.sig == 2) { bad = true; bad_key = min(bad_key, key_of(fminf(nv.th, S.Th[s]))); }
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
      if (nv.sig == 2) { bad = true; bad_key = min(bad_key, key_of(fminf(nv.th, S.iTh[side][k]))); }
    }
    G[slot] = g;
    SU[slot] = 0;
  }
  const unsigned bk = __reduce_min_sync(0xffffffffu, bad_key);
  if (__any_sync(0xffffffffu, bad)) {
    unsigned* gm = tile_mask(F, t);
    atomicOr(gm + lane, 0xffffffffu);
    if (lane < 2) atomicOr(gm + kTH + lane, 0xffffffffu);
    if (lane == 0) {
      atomicMin(F.tkey + t, bk);
      atomicAdd(n_bad, 1u);
    }
  }
}

size_t eik_round_smem() { return sizeof(TileSmem); }

}  // namespace fmt2d
