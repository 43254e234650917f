// Host engine: model upload and the batched forward solve (all sources' time
// fields of one stage level are solved together in one round loop).
#include "engine.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <thread>

namespace fmt2d {

//                     reg istart parent level dst_side target_side reflect water_up
const TfInfo kTf[13] = {{0, 0, 0, -1, 0, 0, 0, -1},
                        {5, 2, 0, 0, 0, 0, 0, -1},    // tf1  Pg, point source
                        {2, 2, 0, 0, 0, 0, 0, -1},    // tf2  PsedP down
                        {2, 3, 2, 1, 1, -1, 1, -1},   // tf3  PsedP up from the sediment base
                        {6, 2, 0, 0, 0, 0, 0, -1},    // tf4  PmP down
                        {6, 4, 4, 1, 1, -1, 1, -1},   // tf5  PmP up from the Moho
                        {1, 2, 1, 1, 1, -1, 1, 1},    // tf6  Pg_ss water up
                        {1, 1, 6, 2, 0, 1, 1, 0},     // tf7  Pg_ss water down
                        {1, 2, 7, 3, 1, -1, 1, 1},    // tf8  Pg_ss water up
                        {1, 2, 0, 0, 0, 0, 0, 1},     // tf9  Pg_ss2 water up, point source
                        {1, 1, 9, 1, 0, 1, 1, 0},     // tf10 Pg_ss2 water down
                        {5, 2, 10, 2, 0, 1, 1, -1},   // tf11 Pg_ss2 solid
                        {1, 2, 11, 3, 1, -1, 1, 1}};  // tf12 Pg_ss2 water up

unsigned phase_fields(int mask) {
  unsigned f = 0;
  if (mask & 1) f |= 1u << 1;
  if (mask & 2) f |= (1u << 2) | (1u << 3);
  if (mask & 4) f |= (1u << 4) | (1u << 5);
  if (mask & 8) f |= (1u << 1) | (1u << 6) | (1u << 7) | (1u << 8);
  if (mask & 16) f |= (1u << 9) | (1u << 10) | (1u << 11) | (1u << 12);
  return f;
}

#define CK(x)                                                                 \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_); \
  } while (0)

void DevBuf::alloc(size_t n) {
  if (n <= bytes && p) return;
  free_();
  if (cudaMalloc(&p, n < 16 ? 16 : n) != cudaSuccess) { p = nullptr; bytes = 0; return; }
  bytes = n;
}

void DevBuf::free_() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

namespace {
template <class T>
std::string put(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.alloc(v.size() * sizeof(T));
  if (!b.p) return "device allocation failed";
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return std::string();
}

template <class T>
std::string put_raw(DevBuf& b, const T* v, size_t n, cudaStream_t st) {
  b.alloc(n * sizeof(T));
  if (!b.p) return "device allocation failed";
  if (n) CK(cudaMemcpyAsync(b.p, v, n * sizeof(T), cudaMemcpyHostToDevice, st));
  return std::string();
}

// Pinned staging of a lane: make room for n bytes (the lane's stream must be
// idle: the old area may be freed), then hand out 256-byte aligned pieces.
std::string lane_reserve(SolveLane& L, size_t n) {
  L.pin_used = 0;
  if (n <= L.pin_cap && L.pin) return std::string();
  if (L.pin) cudaFreeHost(L.pin);
  L.pin = nullptr;
  L.pin_cap = 0;
  const size_t cap = std::max<size_t>(n, 1 << 16);
  if (cudaMallocHost(&L.pin, cap) != cudaSuccess) {
    L.pin = nullptr;
    return "pinned host allocation failed";
  }
  L.pin_cap = cap;
  return std::string();
}

void* lane_take(SolveLane& L, size_t n) {
  const size_t a = (L.pin_used + 255) / 256 * 256;
  if (a + n > L.pin_cap) return nullptr;
  L.pin_used = a + n;
  return L.pin + a;
}

// put() through the lane's pinned staging (the copy is stream-ordered; the
// staging piece is not reused before the lane's stream is idle again).
template <class T>
std::string put_lane(SolveLane& L, DevBuf& b, const std::vector<T>& v) {
  b.alloc(v.size() * sizeof(T));
  if (!b.p) return "device allocation failed";
  if (v.empty()) return std::string();
  void* h = lane_take(L, v.size() * sizeof(T));
  if (!h) return "pinned staging too small";
  std::memcpy(h, v.data(), v.size() * sizeof(T));
  CK(cudaMemcpyAsync(b.p, h, v.size() * sizeof(T), cudaMemcpyHostToDevice, L.st));
  return std::string();
}

// invert2d_main.f90:906-931: depth of the seafloor interface under x.
double seafloor_at(const Model& m, double px) {
  const std::vector<double>& z = m.ifc[2].z;
  const int n = m.nx;
  const double dx = m.xpos[1] - m.xpos[0];
  const int k = (int)std::floor((px - m.xpos[0]) / dx);
  if (k < 0) return z[0];
  if (k >= n - 1) return z[n - 1];
  const double w = std::min(1.0, std::max(0.0, (px - m.xpos[k]) / dx));
  return (1.0 - w) * z[k] + w * z[k + 1];
}
}  // namespace

Engine::Engine(int device) : device_(device) {
  cudaSetDevice(device_);
  cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&ev_start_, cudaEventDisableTiming);
  for (SolveLane& L : lanes_) {
    cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming);
  }
  cudaMallocHost(&h_count_, 4 * sizeof(unsigned));
}

Engine::~Engine() {
  cudaSetDevice(device_);
  fields_.clear();
  if (h_count_) cudaFreeHost(h_count_);
  for (SolveLane& L : lanes_) {
    L.free_all();
    if (L.done) cudaEventDestroy(L.done);
    if (L.st) cudaStreamDestroy(L.st);
  }
  if (ev_start_) cudaEventDestroy(ev_start_);
  if (stream_) cudaStreamDestroy(stream_);
}

std::string Engine::upload(const Model& m) {
  cudaSetDevice(device_);
  m_ = m;
  // the field stores stay allocated (a store grows when a region does);
  // every field is unsolved until the next forward
  for (auto& src : fields_)
    for (FieldStore& f : src) f.solved = false;
  std::string e;
  for (int r = 1; r <= 6; ++r) {
    const Region& G = m.reg[r];
    DevRegionStore& D = reg_[r];
    std::vector<int> izc(2 * G.pitch, -1);
    std::vector<double> ix(G.pitch, 0.0), iz(2 * G.pitch, 0.0);
    for (int k = 0; k < m.nx; ++k) {
      izc[k] = G.izc_top[k];
      izc[G.pitch + k] = G.izc_bot[k];
      ix[k] = m.xpos[k];
      iz[k] = m.ifc[G.itop].z[k];
      iz[G.pitch + k] = m.ifc[G.ibot].z[k];
    }
    if (!(e = put(D.code, G.code, stream_)).empty()) return e;
    if (!(e = put(D.vel64, G.vel64, stream_)).empty()) return e;
    if (!(e = put(D.izc, izc, stream_)).empty()) return e;
    if (!(e = put(D.iface_x, ix, stream_)).empty()) return e;
    if (!(e = put(D.iface_z, iz, stream_)).empty()) return e;
    if (!(e = put(D.r0, G.r0, stream_)).empty()) return e;
    if (!(e = put(D.r1, G.r1, stream_)).empty()) return e;
    if (!(e = put(D.slot_of_node, G.slot_of_node, stream_)).empty()) return e;
    D.nslots = G.nslots();
    double vm = 0.0;
    for (size_t s2 = 0; s2 < G.vel64.size(); ++s2) vm = std::max(vm, G.vel64[s2]);
    D.vmax = vm > 0.0 ? vm : 1.0;
  }
  for (int k = 1; k <= 5; ++k) {
    const Interface& f = m.ifc[k];
    if (!(e = put(ifc_buf_[k][0], f.z, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][1], f.nrm_x, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][2], f.nrm_z, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][3], f.vel_top, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][4], f.vel_bot, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][5], f.izc, stream_)).empty()) return e;
    Ifc64& I = ifc_[k];
    I.z = ifc_buf_[k][0].as<double>();
    I.nrm_x = ifc_buf_[k][1].as<double>();
    I.nrm_z = ifc_buf_[k][2].as<double>();
    I.vel_top = ifc_buf_[k][3].as<double>();
    I.vel_bot = ifc_buf_[k][4].as<double>();
    I.izc = ifc_buf_[k][5].as<int>();
  }
  // Head-wave sweep tables of the up-going PmP field (inversion2d.f90:4294-
  // 4348): node n of the Moho intersection maps through the intersection's
  // rright table (else rleft) into region 6, as the reference indexes it.
  {
    const Region& R6 = m.reg[6];
    const Interface& moho = m.ifc[4];
    std::vector<int> hs(m.nx, -1), hvs(m.nx, -1);   // sweep node; slot whose velocity hv is
    std::vector<double> hv(m.nx, 0.0);
    for (int n = 0; n < m.nx; ++n) {
      int id = 0;
      if (!m.rright[4].empty()) id = m.rright[4][n];
      if (id == 0 && !m.rleft[4].empty()) id = m.rleft[4][n];
      if (id < 1 || id > R6.nnode) continue;
      const int slot = R6.slot_of_node[id - 1];
      hs[n] = slot;
      if (id - 1 >= R6.ngnode) {
        const int k3 = (id - 1 - R6.ngnode) % m.nx;
        const int c = moho.izc[k3];
        if (c < 0) continue;
        for (int ii = 0; ii <= 1; ++ii)
          for (int jj = 0; jj <= 1; ++jj) {
            const int a = k3 + ii, b = c + jj;
            if (a >= m.nx || b >= m.nz) continue;
            if (m.node_region[m.g(a, b)] != 6) continue;
            const int q = m.rnode_id[m.g(a, b)];
            if (q < 1 || q > R6.ngnode) continue;
            if (b * m.dx > moho.z[n] + 0.5 * m.dx) {
              const int sq = R6.slot_of_node[q - 1];
              if (R6.vel64[sq] > hv[n]) { hv[n] = R6.vel64[sq]; hvs[n] = sq; }
            }
          }
      } else {
        hv[n] = R6.vel64[slot];
        hvs[n] = slot;
      }
    }
    if (!(e = put(hw_slot_, hs, stream_)).empty()) return e;
    if (!(e = put(hw_v_, hv, stream_)).empty()) return e;
    hw_slot_h_ = hs;
    hw_vslot_h_ = hvs;
  }
  if (!(e = upload_trace_tables()).empty()) return e;
  npick_ = -1;
  ++model_version_;   // cached per-model tables (the adjoint's velocity maps) are stale
  CK(cudaStreamSynchronize(stream_));
  return std::string();
}

void Engine::ensure_sources(int nsrc) {
  if ((int)fields_.size() < nsrc) fields_.resize(nsrc);
  src_x_.resize(std::max<size_t>(src_x_.size(), nsrc));
  src_z_.resize(std::max<size_t>(src_z_.size(), nsrc));
}

std::string Engine::forward(const double* sx, int nsrc, int phase_mask) {
  cudaSetDevice(device_);
  if (m_.nx == 0) return "no model uploaded";
  if (nsrc <= 0) return "no sources";
  ensure_sources(nsrc);
  const unsigned need = phase_fields(phase_mask);
  for (int s = 0; s < nsrc; ++s) {
    src_x_[s] = sx[s];
    src_z_[s] = seafloor_at(m_, sx[s]);
    for (int tf = 1; tf <= 12; ++tf) {
      FieldStore& F = fields_[s][tf];
      F.solved = false;
      if (!(need & (1u << tf))) continue;
      const DevRegionStore& D = reg_[kTf[tf].reg];
      F.T.alloc(D.nslots * 8);
      F.G.alloc(D.nslots * 16);
      F.Gout.alloc(D.nslots * 16);
      F.fl.alloc(D.nslots);
      F.seed.alloc(D.nslots * 32);
      F.clock.alloc(32);
      if (!F.T.p || !F.G.p || !F.Gout.p || !F.fl.p || !F.seed.p || !F.clock.p)
        return "device allocation failed for the time fields";
    }
  }
  stats_ = SolveStats();
  not_converged_ = false;
  // the stage chains (Pg -> Pg_ss, PsedP, PmP, Pg_ss2) are independent: each
  // runs on its own stream, driven by its own host thread, after the work
  // already queued on the context's stream and before anything queued on it
  // later
  bool active[kChains] = {};
  for (int tf = 1; tf <= 12; ++tf)
    if (need & (1u << tf)) active[chain_of(tf)] = true;
  CK(cudaEventRecord(ev_start_, stream_));
  std::string errs[kChains];
  auto run_chain = [&](int c) {
    cudaSetDevice(device_);
    SolveLane& L = lanes_[c];
    L.stats = SolveStats();
    L.not_converged = false;
    cudaStreamWaitEvent(L.st, ev_start_, 0);
    for (int level = 0; level <= 3 && errs[c].empty(); ++level) {
      std::vector<std::pair<int, int>> items;
      for (int tf = 1; tf <= 12; ++tf)
        if ((need & (1u << tf)) && kTf[tf].level == level && chain_of(tf) == c)
          for (int s = 0; s < nsrc; ++s) items.emplace_back(s, tf);
      if (!items.empty()) errs[c] = solve_level(L, items);
    }
    cudaEventRecord(L.done, L.st);
  };
  std::vector<std::thread> threads;
  int nact = 0, last = -1;
  for (int c = 0; c < kChains; ++c)
    if (active[c]) {
      ++nact;
      last = c;
    }
  for (int c = 0; c < kChains; ++c)
    if (active[c] && c != last) threads.emplace_back(run_chain, c);
  if (last >= 0) run_chain(last);
  for (std::thread& t : threads) t.join();
  std::string err;
  for (int c = 0; c < kChains; ++c) {
    if (!active[c]) continue;
    const SolveStats& q = lanes_[c].stats;
    stats_.rounds = std::max(stats_.rounds, q.rounds);
    stats_.round_ms = std::max(stats_.round_ms, q.round_ms);
    stats_.steps_sum += q.steps_sum;
    stats_.batches += q.batches;
    stats_.final_passes += q.final_passes;
    stats_.evals += q.evals;
    stats_.writes += q.writes;
    stats_.passed += q.passed;
    stats_.unsettled += q.unsettled;
    stats_.capped += q.capped;
    stats_.launches += q.launches;
    stats_.nodes += q.nodes;
    for (int k = 0; k < 5; ++k) stats_.cycles[k] += q.cycles[k];
    stats_.cut_evals += q.cut_evals;
    stats_.cut_steps += q.cut_steps;
    not_converged_ = not_converged_ || lanes_[c].not_converged;
    cudaStreamWaitEvent(stream_, lanes_[c].done, 0);
    if (err.empty() && !errs[c].empty()) err = errs[c];
  }
  if (!err.empty()) return err;
  CK(cudaStreamSynchronize(stream_));
  return std::string();
}

Fld64 Engine::field_view(int src, int tf) const {
  const Region& G = m_.reg[kTf[tf].reg];
  const DevRegionStore& D = reg_[kTf[tf].reg];
  const FieldStore& S = fields_[src][tf];
  Fld64 f;
  f.code = D.code.as<uint32_t>();
  f.vel = D.vel64.as<double>();
  f.izc = D.izc.as<int>();
  f.ifx = D.iface_x.as<double>();
  f.ifz = D.iface_z.as<double>();
  f.H = G.H;
  f.pitch = G.pitch;
  f.z_lo = G.z_lo;
  f.nx = m_.nx;
  f.nz = m_.nz;
  f.x0 = m_.x0;
  f.dx = m_.dx;
  f.tol = m_.tolerance;
  f.T = S.T.as<double>();
  f.G = S.G.as<double2>();
  f.Gout = S.Gout.as<double2>();
  f.fl = S.fl.as<uint8_t>();
  f.seed = S.seed.as<double4>();
  f.clock = S.clock.as<double>();
  return f;
}

std::string Engine::solve_level(SolveLane& L, const std::vector<std::pair<int, int>>& items) {
  const int nf = (int)items.size();
  std::vector<Fld64> hf(nf);
  std::vector<int> up(nf, -1), hw;
  std::vector<double> wstep(nf);
  size_t total = 0, max_slots = 0;
  for (int i = 0; i < nf; ++i) {
    const int tf = items[i].second;
    const DevRegionStore& D = reg_[kTf[tf].reg];
    total += D.nslots;
    max_slots = std::max(max_slots, D.nslots);
  }
  if (max_slots >= (1ull << 30)) return "region too large for the eikonal solver (2^30 slots)";
  {
    // the lane's stream is idle here (the previous level ended with a sync)
    const size_t per = sizeof(Fld64) + sizeof(Seed64) + 4 * sizeof(double) + 8 * sizeof(unsigned) +
                       sizeof(double*);
    std::string e0s = lane_reserve(L, (size_t)nf * per + kCtrN * 8 + 16 * 256);
    if (!e0s.empty()) return e0s;
  }
  // solver scratch of the batch, per slot: staged time, gradient and flags,
  // pending time, start list, list and commit overflow, listed bitset
  const size_t words = (total + 31 * (size_t)nf + 31) / 32 + (size_t)nf;
  L.sTn.alloc(total * sizeof(double));
  L.sGn.alloc(total * sizeof(double2));
  L.sfln.alloc(total);
  L.spend.alloc(total * sizeof(double));
  L.sclaim.alloc(total * sizeof(unsigned long long));
  L.slist.alloc(total * sizeof(unsigned));
  L.sover.alloc(3 * total * sizeof(unsigned));
  L.sinq.alloc(3 * words * sizeof(unsigned));
  L.scnt.alloc((size_t)nf * 4 * sizeof(unsigned));
  L.ctr.alloc(kCtrN * sizeof(unsigned long long));
  if (!L.sTn.p || !L.sGn.p || !L.sfln.p || !L.spend.p || !L.sclaim.p || !L.slist.p ||
      !L.sover.p ||
      !L.sinq.p || !L.scnt.p || !L.ctr.p)
    return "device allocation failed for the solver scratch";
  size_t base = 0, wbase = 0;
  int max_tiles = 0;
  for (int i = 0; i < nf; ++i) {
    const int s = items[i].first, tf = items[i].second;
    const DevRegionStore& D = reg_[kTf[tf].reg];
    hf[i] = field_view(s, tf);
    hf[i].Tn = L.sTn.as<double>() + base;
    hf[i].Gn = L.sGn.as<double2>() + base;
    hf[i].fln = L.sfln.as<uint8_t>() + base;
    hf[i].pend = L.spend.as<double>() + base;
    hf[i].claim = L.sclaim.as<unsigned long long>() + base;
    hf[i].list_in = L.slist.as<unsigned>() + base;
    hf[i].over = L.sover.as<unsigned>() + 3 * base;
    hf[i].inq = L.sinq.as<unsigned>() + wbase;
    hf[i].wait = L.sinq.as<unsigned>() + words + wbase;
    hf[i].moving = L.sinq.as<unsigned>() + 2 * words + wbase;
    if (e64_tiles(hf[i]) > e64_tiles_max()) return "region too large for the eikonal solver";
    max_tiles = std::max(max_tiles, e64_tiles(hf[i]));
    hf[i].cnt = L.scnt.as<unsigned>() + 4 * (size_t)i;
    base += D.nslots;
    wbase += (D.nslots + 31) / 32;
    up[i] = kTf[tf].water_up;
    // the schedule's window, or by default none for a point source and
    // kIfaceWindowCells for a stage seeded along an interface (its seeds span
    // the whole line at once; without a window far nodes take early times
    // that many later updates revise)
    const double wc = window_cells > 0.0 ? window_cells
                      : (kTf[tf].level == 0 ? 0.0 : iface_window_cells);
    wstep[i] = wc > 0.0 ? wc * m_.dx / D.vmax : kHugeD;
    if (tf == 5) hw.push_back(i);
  }
  std::string e;
  if (!(e = put_lane(L, L.fields, hf)).empty()) return e;
  if (!(e = put_lane(L, L.up, up)).empty()) return e;
  if (!(e = put_lane(L, L.step, wstep)).empty()) return e;
  unsigned long long* dctr = L.ctr.as<unsigned long long>();
  CK(cudaMemsetAsync(L.sinq.p, 0, words * sizeof(unsigned), L.st));
  CK(cudaMemsetAsync(L.scnt.p, 0, (size_t)nf * 4 * sizeof(unsigned), L.st));
  CK(cudaMemsetAsync(dctr, 0, kCtrN * sizeof(unsigned long long), L.st));
  Fld64* dF = L.fields.as<Fld64>();
  e64_fill(dF, nf, max_slots, L.st);
  ++L.stats.launches;
  CK(cudaGetLastError());
  const int level = kTf[items[0].second].level;
  if (level == 0) {
    std::vector<double> sx(nf), sz(nf);
    for (int i = 0; i < nf; ++i) { sx[i] = src_x_[items[i].first]; sz[i] = src_z_[items[i].first]; }
    if (!(e = put_lane(L, L.sx, sx)).empty()) return e;
    if (!(e = put_lane(L, L.sz, sz)).empty()) return e;
    e64_init_source(dF, L.sx.as<double>(), L.sz.as<double>(), nf, L.st);
    ++L.stats.launches;
  } else {
    std::vector<Seed64> sd(nf);
    for (int i = 0; i < nf; ++i) {
      const int s = items[i].first, tf = items[i].second;
      const TfInfo& I = kTf[tf];
      const FieldStore& P = fields_[s][I.parent];
      if (!P.solved) return "parent time field not solved";
      const Region& PR = m_.reg[kTf[I.parent].reg];
      const DevRegionStore& D = reg_[I.reg];
      Seed64& d = sd[i];
      d.dst = i;
      d.src_T = P.T.as<double>();
      d.src_G = P.Gout.as<double2>();
      d.src_row = PR.H + (I.istart == PR.itop ? 0 : 1);
      d.src_pitch = PR.pitch;
      d.ifc = ifc_[I.istart];
      d.r0 = D.r0.as<int>();
      d.r1 = D.r1.as<int>();
      d.dst_side = I.dst_side;
      d.reflect = I.reflect;
      d.target_side = I.target_side;
    }
    if (!(e = put_lane(L, L.seeds, sd)).empty()) return e;
    e64_seed_iface(dF, L.seeds.as<Seed64>(), nf, m_.nx, L.st);
    ++L.stats.launches;
  }
  e64_start(dF, nf, max_slots, L.step.as<double>(), L.st);
  L.stats.launches += 2;
  CK(cudaGetLastError());
  // solve, then check every node; nodes the check re-lists are solved again
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return "cudaEventCreate failed";
  }
  std::string err;
  unsigned* hc = static_cast<unsigned*>(lane_take(L, (size_t)nf * 4 * sizeof(unsigned)));
  unsigned long long* hctr =
      static_cast<unsigned long long*>(lane_take(L, kCtrN * sizeof(unsigned long long)));
  if (!hc || !hctr) return "pinned staging too small";
  cudaEventRecord(e0, L.st);
  unsigned long long bad = 0;
  for (int pass = 0;; ++pass) {
    e64_solve(dF, nf, max_slots, max_tiles, max_steps, dctr, solve_threads, L.st);
    ++L.stats.launches;
    ++L.stats.final_passes;
    cudaMemsetAsync(L.sinq.p, 0, words * sizeof(unsigned), L.st);
    e64_verify(dF, nf, max_slots, L.st);
    ++L.stats.launches;
    cudaError_t ce = cudaMemcpyAsync(hc, L.scnt.p, (size_t)nf * 4 * sizeof(unsigned),
                                     cudaMemcpyDeviceToHost, L.st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(L.st);
    if (ce != cudaSuccess) { err = std::string("eikonal solve: ") + cudaGetErrorString(ce); break; }
    bad = 0;
    unsigned capped = 0;
    for (int i = 0; i < nf; ++i) {
      bad += hc[4 * (size_t)i + 1];
      capped += hc[4 * (size_t)i + 2];
    }
    if (capped) {
      L.stats.capped += capped;
      L.not_converged = true;
      err = "eikonal solve reached its step cap in " + std::to_string(capped) + " fields";
      break;
    }
    if (bad == 0 || pass + 1 >= max_passes) break;
  }
  cudaEventRecord(e1, L.st);
  cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!err.empty()) return err;
  L.stats.round_ms += ms;
  {
    unsigned long long* c = hctr;
    CK(cudaMemcpyAsync(c, dctr, kCtrN * sizeof(unsigned long long), cudaMemcpyDeviceToHost, L.st));
    CK(cudaStreamSynchronize(L.st));
    L.stats.evals += c[kCtrEval];
    L.stats.writes += c[kCtrWrite];
    L.stats.passed += c[kCtrPass];
    L.stats.rounds += (long long)c[kCtrMaxSteps];
    L.stats.steps_sum += c[kCtrSteps];
    for (int k = 0; k < 5; ++k) L.stats.cycles[k] += (double)c[kCtrCycEval + k];
    L.stats.cut_evals += c[kCtrCut];
    L.stats.cut_steps += c[kCtrStepsCut];
  }
  if (bad) {
    L.stats.unsettled += bad;
    L.not_converged = true;
    return "eikonal solve did not reach its fixed point (" + std::to_string(bad) +
           " nodes still move after " + std::to_string(max_passes) + " passes)";
  }
  e64_finish(dF, nf, max_slots, L.up.as<int>(), L.st);
  L.stats.launches += 2;
  CK(cudaGetLastError());
  if (!hw.empty()) {
    if (!(e = put_lane(L, L.which, hw)).empty()) return e;
    L.hw.alloc(hw.size() * (size_t)m_.nx * sizeof(double));
    // each field keeps its solved times at the sweep nodes (for the adjoint)
    std::vector<double*> pre(hw.size());
    for (size_t q = 0; q < hw.size(); ++q) {
      FieldStore& S = fields_[items[hw[q]].first][items[hw[q]].second];
      S.hwpre.alloc((size_t)m_.nx * sizeof(double));
      if (!S.hwpre.p) return "device allocation failed (head-wave times)";
      pre[q] = S.hwpre.as<double>();
    }
    if (!(e = put_lane(L, L.hwpre, pre)).empty()) return e;
    const double dx_if = m_.xpos[1] - m_.xpos[0];
    e64_headwave(dF, hw_slot_.as<int>(), hw_v_.as<double>(), dx_if, m_.nx,
                 L.hw.as<double>(), L.which.as<int>(), (int)hw.size(), L.hwpre.as<double*>(),
                 L.st);
    ++L.stats.launches;
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(L.st));
  for (int i = 0; i < nf; ++i) {
    fields_[items[i].first][items[i].second].solved = true;
    L.stats.nodes += m_.reg[kTf[items[i].second].reg].nnode;
  }
  ++L.stats.batches;
  return std::string();
}

std::string Engine::get_field_device(int src, int tf, double* T, double* gx, double* gz) {
  cudaSetDevice(device_);
  if (src < 0 || src >= (int)fields_.size() || tf < 1 || tf > 12) return "bad field index";
  const FieldStore& F = fields_[src][tf];
  if (!F.solved) return "time field not solved";
  const Region& G = m_.reg[kTf[tf].reg];
  const DevRegionStore& D = reg_[kTf[tf].reg];
  e64_export(F.T.as<double>(), F.Gout.as<double2>(), D.slot_of_node.as<int>(), G.nnode, T, gx, gz,
             stream_);
  ++stats_.launches;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(stream_));
  return std::string();
}

std::string Engine::get_field(int src, int tf, double* T, double* gx, double* gz) {
  cudaSetDevice(device_);
  if (src < 0 || src >= (int)fields_.size() || tf < 1 || tf > 12) return "bad field index";
  const FieldStore& F = fields_[src][tf];
  if (!F.solved) return "time field not solved";
  const Region& G = m_.reg[kTf[tf].reg];
  const DevRegionStore& D = reg_[kTf[tf].reg];
  const int nn = G.nnode;
  export_.alloc((size_t)nn * 3 * sizeof(double));
  if (!export_.p) return "device allocation failed";
  double* d = export_.as<double>();
  e64_export(F.T.as<double>(), F.Gout.as<double2>(), D.slot_of_node.as<int>(), nn, d, d + nn,
             d + 2 * (size_t)nn, stream_);
  ++stats_.launches;
  CK(cudaGetLastError());
  if (T) CK(cudaMemcpyAsync(T, d, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (gx) CK(cudaMemcpyAsync(gx, d + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (gz) CK(cudaMemcpyAsync(gz, d + 2 * (size_t)nn, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return std::string();
}

}  // namespace fmt2d
