// Host engine: model upload and the batched forward solve (all sources' time
// fields of one stage level are solved together in one round loop).
#include "engine.h"
#include "kernels.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>

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
  cudaMallocHost(&h_count_, 4 * sizeof(unsigned));
  cudaFuncSetAttribute(eik_visit, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)eik_round_smem());
  cudaFuncSetAttribute(eik_final, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)eik_round_smem());
  // persistent visit blocks: as many warps as fit on the device at once
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eik_visit, 32, eik_round_smem());
  visit_blocks_ = std::max(1, nsm) * std::max(1, per_sm);
}

Engine::~Engine() {
  cudaSetDevice(device_);
  fields_.clear();
  if (h_count_) cudaFreeHost(h_count_);
  if (stream_) cudaStreamDestroy(stream_);
}

std::string Engine::upload(const Model& m) {
  cudaSetDevice(device_);
  m_ = m;
  fields_.clear();
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
    if (!(e = put(D.vel, G.vel, stream_)).empty()) return e;
    if (!(e = put(D.vel64, G.vel64, stream_)).empty()) return e;
    if (!(e = put(D.iface_dz, G.iface_dz, stream_)).empty()) return e;
    if (!(e = put(D.izc, izc, stream_)).empty()) return e;
    if (!(e = put(D.iface_x, ix, stream_)).empty()) return e;
    if (!(e = put(D.iface_z, iz, stream_)).empty()) return e;
    if (!(e = put(D.r0, G.r0, stream_)).empty()) return e;
    if (!(e = put(D.r1, G.r1, stream_)).empty()) return e;
    if (!(e = put(D.slot_of_node, G.slot_of_node, stream_)).empty()) return e;
    DevRegion& R = D.R;
    R.code = D.code.as<uint32_t>();
    R.vel = D.vel.as<float>();
    R.iface_dz = D.iface_dz.as<float>();
    R.izc = D.izc.as<int>();
    R.H = G.H;
    R.pitch = G.pitch;
    R.tiles_x = G.tiles_x;
    R.tiles_y = G.tiles_y;
    R.z_lo = G.z_lo;
    R.nx = m.nx;
    R.dx = m.dx;
    R.x0 = m.x0;
    R.tol = m.tolerance;
    DevRegionX& X = D.X;
    X.vel64 = D.vel64.as<double>();
    X.iface_x = D.iface_x.as<double>();
    X.iface_z = D.iface_z.as<double>();
    X.r0 = D.r0.as<int>();
    X.r1 = D.r1.as<int>();
    X.itop = G.itop;
    X.ibot = G.ibot;
    X.id = r;
    X.nz = m.nz;
    D.nslots = G.nslots();
    D.ntiles = G.tiles_x * G.tiles_y;
    double vs = 0.0;
    long nv = 0;
    for (size_t s = 0; s < G.vel64.size(); ++s)
      if (G.vel64[s] > 0.0) { vs += G.vel64[s]; ++nv; }
    D.vmean = nv ? vs / nv : 1.0;
  }
  for (int k = 1; k <= 5; ++k) {
    const Interface& f = m.ifc[k];
    if (!(e = put(ifc_buf_[k][0], f.z, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][1], f.nrm_x, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][2], f.nrm_z, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][3], f.vel_top, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][4], f.vel_bot, stream_)).empty()) return e;
    if (!(e = put(ifc_buf_[k][5], f.izc, stream_)).empty()) return e;
    DevIface& I = ifc_[k];
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
    std::vector<int> hs(m.nx, -1);
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
            if (b * m.dx > moho.z[n] + 0.5 * m.dx)
              hv[n] = std::max(hv[n], R6.vel64[R6.slot_of_node[q - 1]]);
          }
      } else {
        hv[n] = R6.vel64[slot];
      }
    }
    if (!(e = put(hw_slot_, hs, stream_)).empty()) return e;
    if (!(e = put(hw_v_, hv, stream_)).empty()) return e;
  }
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
      F.t2.alloc(D.nslots * 8);
      F.g2.alloc(D.nslots * 8);
      F.gout.alloc(D.nslots * 8);
      F.susp.alloc(D.nslots);
      F.act.alloc((size_t)kTileWords * D.ntiles * 4);
      F.tkey.alloc((size_t)D.ntiles * 8);   // keys, then visit counts
      F.front.alloc(16);
      F.seed.alloc(D.nslots * 16);
      F.sflag.alloc(D.nslots);
      if (!F.t2.p || !F.g2.p || !F.gout.p || !F.susp.p || !F.act.p || !F.seed.p || !F.sflag.p ||
          !F.tkey.p || !F.front.p)
        return "device allocation failed for the time fields";
    }
  }
  stats_ = SolveStats();
  for (int level = 0; level <= 3; ++level) {
    std::vector<std::pair<int, int>> items;
    for (int tf = 1; tf <= 12; ++tf)
      if ((need & (1u << tf)) && kTf[tf].level == level)
        for (int s = 0; s < nsrc; ++s) items.emplace_back(s, tf);
    if (items.empty()) continue;
    std::string e = solve_level(items);
    if (!e.empty()) return e;
  }
  CK(cudaStreamSynchronize(stream_));
  return std::string();
}

std::string Engine::solve_level(const std::vector<std::pair<int, int>>& items) {
  const int nf = (int)items.size();
  std::vector<DevField> hf(nf);
  std::vector<DevRegionX> hx(nf);
  std::vector<float*> hg(nf);
  std::vector<uint8_t*> hs(nf);
  std::vector<int> up(nf, -1);
  std::vector<int> hw;
  int total_tiles = 0;
  size_t max_slots = 0;
  for (int i = 0; i < nf; ++i) {
    const int s = items[i].first, tf = items[i].second;
    const DevRegionStore& D = reg_[kTf[tf].reg];
    FieldStore& F = fields_[s][tf];
    DevField& f = hf[i];
    f.R = D.R;
    f.Th = F.t2.as<float>();
    f.Tl = f.Th;
    f.gx = F.g2.as<float>();
    f.gz = f.gx;
    f.act = F.act.as<unsigned>();
    f.tkey = F.tkey.as<unsigned>();
    f.tvis = f.tkey + reg_[kTf[tf].reg].ntiles;
    f.front = F.front.as<float>();
    f.band = (float)(band_tiles * kTW * m_.dx / D.vmean);
    f.seed = F.seed.as<float4>();
    f.sflag = F.sflag.as<uint8_t>();
    f.frozen_slot = -1;
    f.tile_base = total_tiles;
    total_tiles += D.ntiles;
    max_slots = std::max(max_slots, D.nslots);
    hx[i] = D.X;
    hg[i] = F.gout.as<float>();
    hs[i] = F.susp.as<uint8_t>();
    up[i] = kTf[tf].water_up;
    if (tf == 5) hw.push_back(i);
  }
  std::string e;
  if (!(e = put(d_fields_, hf, stream_)).empty()) return e;
  if (!(e = put(d_xs_, hx, stream_)).empty()) return e;
  if (!(e = put(d_gout_, hg, stream_)).empty()) return e;
  if (!(e = put(d_susp_, hs, stream_)).empty()) return e;
  if (!(e = put(d_up_, up, stream_)).empty()) return e;
  DevField* dF = d_fields_.as<DevField>();
  {
    const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 1024);
    k_fill<<<dim3(bx, nf), 256, 0, stream_>>>(dF, nf, max_slots);
    ++stats_.launches;
    CK(cudaGetLastError());
  }
  const int level = kTf[items[0].second].level;
  if (level == 0) {
    std::vector<double> sx(nf), sz(nf);
    for (int i = 0; i < nf; ++i) { sx[i] = src_x_[items[i].first]; sz[i] = src_z_[items[i].first]; }
    if (!(e = put(d_sx_, sx, stream_)).empty()) return e;
    if (!(e = put(d_sz_, sz, stream_)).empty()) return e;
    k_init_source<<<(nf + 63) / 64, 64, 0, stream_>>>(dF, d_xs_.as<DevRegionX>(),
                                                       d_sx_.as<double>(), d_sz_.as<double>(),
                                                       nf, m_.nz);
    ++stats_.launches;
    CK(cudaGetLastError());
  } else {
    std::vector<SeedDesc> sd(nf);
    for (int i = 0; i < nf; ++i) {
      const int s = items[i].first, tf = items[i].second;
      const TfInfo& I = kTf[tf];
      const FieldStore& P = fields_[s][I.parent];
      if (!P.solved) return "parent time field not solved";
      const Region& PR = m_.reg[kTf[I.parent].reg];
      SeedDesc& d = sd[i];
      d.dst = hf[i];
      d.dstx = hx[i];
      d.src_t = P.t2.as<float>();
      d.src_g = P.gout.as<float>();
      d.src_row = PR.H + (I.istart == PR.itop ? 0 : 1);
      d.src_pitch = PR.pitch;
      d.ifc = ifc_[I.istart];
      d.dst_side = I.dst_side;
      d.reflect = I.reflect;
      d.target_side = I.target_side;
    }
    if (!(e = put(d_seeds_, sd, stream_)).empty()) return e;
    k_seed_iface<<<dim3((m_.nx + 127) / 128, nf), 128, 0, stream_>>>(d_seeds_.as<SeedDesc>(), nf,
                                                                    m_.nz);
    ++stats_.launches;
    CK(cudaGetLastError());
  }
  d_count_.alloc(16);
  d_counters_.alloc(4 * sizeof(unsigned long long));
  unsigned long long* dctr = d_counters_.as<unsigned long long>();
  CK(cudaMemsetAsync(dctr, 0, 4 * sizeof(unsigned long long), stream_));
  unsigned* dcount = d_count_.as<unsigned>();
  const size_t smem = eik_round_smem();
  d_queue_.alloc((size_t)total_tiles * sizeof(unsigned));
  unsigned* dq = d_queue_.as<unsigned>();
  {
    const int bx = (int)std::min<size_t>(((size_t)kTileWords * 4096 + 255) / 256, 256);
    k_seed_masks<<<dim3(bx, nf), 256, 0, stream_>>>(dF, nf);
    ++stats_.launches;
    CK(cudaGetLastError());
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int pass = 0; pass < 6; ++pass) {
    for (int round = 0; round < max_rounds; ++round) {
      // dcount: [0] tiles with pending work, [1] queued tiles, [2] queue head
      CK(cudaMemsetAsync(dcount, 0, 4 * sizeof(unsigned), stream_));
      eik_front<<<nf, 256, 0, stream_>>>(dF, nf, dcount);
      ++stats_.launches;
      eik_select<<<(total_tiles + 255) / 256, 256, 0, stream_>>>(dF, nf, total_tiles, dq,
                                                                 dcount + 1);
      ++stats_.launches;
      cudaEventRecord(e0, stream_);
      eik_visit<<<visit_blocks_, 32, smem, stream_>>>(dF, nf, dq, dcount + 1, dcount + 2,
                                                      max_passes, dctr);
      ++stats_.launches;
      cudaEventRecord(e1, stream_);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h_count_, dcount, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                         stream_));
      CK(cudaStreamSynchronize(stream_));
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      stats_.round_ms += ms;
      ++stats_.rounds;
      stats_.tile_visits += h_count_[1];
      if (h_count_[0] == 0u) break;
    }
    CK(cudaMemsetAsync(dcount, 0, 4 * sizeof(unsigned), stream_));
    eik_final<<<total_tiles, 32, smem, stream_>>>(dF, nf, d_gout_.as<float*>(),
                                                  d_susp_.as<uint8_t*>(), dcount);
    ++stats_.launches;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_count_, dcount, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    ++stats_.final_passes;
    if (h_count_[0] == 0u) break;
  }
  {
    unsigned long long c[4];
    CK(cudaMemcpy(c, dctr, sizeof(c), cudaMemcpyDeviceToHost));
    stats_.passes += c[0];
    stats_.steps += c[1];
    stats_.capped += c[2];
    stats_.updates += c[3];
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    const int bx = (int)std::min<size_t>((max_slots + 255) / 256, 512);
    k_fit_suspect<<<dim3(bx, nf), 256, 0, stream_>>>(dF, d_xs_.as<DevRegionX>(),
                                                     d_gout_.as<float*>(), d_susp_.as<uint8_t*>(),
                                                     nf);
    ++stats_.launches;
    CK(cudaGetLastError());
    k_water_fix<<<dim3((m_.nx + 127) / 128, nf), 128, 0, stream_>>>(dF, d_gout_.as<float*>(),
                                                                   d_up_.as<int>(), nf);
    ++stats_.launches;
    CK(cudaGetLastError());
  }
  if (!hw.empty()) {
    if (!(e = put(d_which_, hw, stream_)).empty()) return e;
    d_scratch_.alloc(hw.size() * (size_t)m_.nx * sizeof(double));
    const double dx_if = m_.xpos[1] - m_.xpos[0];
    k_headwave<<<((int)hw.size() + 31) / 32, 32, 0, stream_>>>(
        dF, d_xs_.as<DevRegionX>(), d_gout_.as<float*>(), hw_slot_.as<int>(), hw_v_.as<double>(),
        dx_if, m_.nx, d_scratch_.as<double>(), d_which_.as<int>(), (int)hw.size());
    ++stats_.launches;
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(stream_));
  for (int i = 0; i < nf; ++i) {
    fields_[items[i].first][items[i].second].solved = true;
    stats_.nodes += m_.reg[kTf[items[i].second].reg].nnode;
  }
  ++stats_.batches;
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
  DevBuf out;
  out.alloc((size_t)nn * 3 * sizeof(double));
  if (!out.p) return "device allocation failed";
  double* d = out.as<double>();
  k_export<<<(nn + 255) / 256, 256, 0, stream_>>>(F.t2.as<float>(), F.gout.as<float>(),
                                                  D.slot_of_node.as<int>(), nn, d, d + nn,
                                                  d + 2 * (size_t)nn);
  ++stats_.launches;
  CK(cudaGetLastError());
  if (T) CK(cudaMemcpyAsync(T, d, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (gx) CK(cudaMemcpyAsync(gx, d + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (gz) CK(cudaMemcpyAsync(gz, d + 2 * (size_t)nn, nn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return std::string();
}

}  // namespace fmt2d
