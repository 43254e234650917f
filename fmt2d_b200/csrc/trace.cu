// Host side of the ray backtrace and Frechet rows: device tables of the
// model, the two tracing passes (count, then write) and the assembly of the
// contributions into CSR rows (read_frechet_data2d's layout: one row per pick,
// columns ascending, entries with |value| <= 1e-30 dropped as
// compute_frechet_for_ray2d does, src/inversion2d.f90:4761-4768).
#include "engine.h"
#include "rays.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <algorithm>

namespace fmt2d {

#define TCK(x)                                                                \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_); \
  } while (0)

namespace {

__global__ void k_keep(const unsigned long long* keys, const double* vals, int n, int* flag,
                       int* row_cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool keep = fabs(vals[i]) > 1.0e-30;
  flag[i] = keep ? 1 : 0;
  if (keep) atomicAdd(row_cnt + (int)(keys[i] >> 32), 1);
}

__global__ void k_scatter_rows(const unsigned long long* keys, const double* vals,
                               const int* flag, const int* pos, int n, int* col, double* val) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  col[pos[i]] = (int)(keys[i] & 0xffffffffull);
  val[pos[i]] = vals[i];
}

template <class T>
std::string put_vec(DevBuf& b, const T* v, size_t n, cudaStream_t st) {
  b.alloc(std::max<size_t>(n, 1) * sizeof(T));
  if (!b.p) return "device allocation failed";
  if (n) TCK(cudaMemcpyAsync(b.p, v, n * sizeof(T), cudaMemcpyHostToDevice, st));
  return std::string();
}

}  // namespace

std::string Engine::upload_trace_tables() {
  const Model& m = m_;
  std::string e;
  if (!(e = put_vec(d_pvel_, m.vel.data(), m.vel.size(), stream_)).empty()) return e;
  if (!(e = put_vec(d_invidx_, m.inv_idx.data(), m.inv_idx.size(), stream_)).empty()) return e;
  if (!(e = put_vec(d_xpos_, m.xpos.data(), m.xpos.size(), stream_)).empty()) return e;
  TrModel t;
  t.nx = m.nx;
  t.nz = m.nz;
  t.x0 = m.x0;
  t.dx = m.dx;
  t.tol = m.tolerance;
  t.vwater = m.vwater;
  t.vel = d_pvel_.as<double>();
  t.xpos = d_xpos_.as<double>();
  for (int k = 1; k <= 5; ++k) t.ifz[k] = ifc_buf_[k][0].as<double>();
  t.inv_idx = d_invidx_.as<int>();
  t.iface_inv = m.iface_inv;
  t.iface_start = m.n_vel_parms;
  t.n_inv = m.n_inv_parms;
  for (int r = 1; r <= 6; ++r) {
    const Region& G = m.reg[r];
    TrRegion& R = t.reg[r];
    R.code = reg_[r].code.as<uint32_t>();
    R.slot_of_node = reg_[r].slot_of_node.as<int>();
    R.r0 = reg_[r].r0.as<int>();
    R.r1 = reg_[r].r1.as<int>();
    R.z_lo = G.z_lo;
    R.H = G.H;
    R.pitch = G.pitch;
    R.itop = G.itop;
    R.ibot = G.ibot;
    R.id = r;
    R.nnode = G.nnode;
  }
  return put_vec(d_trmodel_, &t, 1, stream_);
}

std::string Engine::trace(const int* src, const int* phase, const double* rx, const double* rz,
                          int npick, double* t_calc, int* valid, long long* nnz, bool rows) {
  cudaSetDevice(device_);
  if (m_.nx == 0) return "no model uploaded";
  if (npick < 0) return "negative pick count";
  const int ns = (int)fields_.size();
  std::vector<TrPick> pk(std::max(npick, 1));
  for (int i = 0; i < npick; ++i) {
    if (src[i] < 0 || src[i] >= ns) return "pick source out of range";
    if (phase[i] < 1 || phase[i] > 5) return "pick phase out of range";
    pk[i].src = src[i];
    pk[i].phase = phase[i];
    pk[i].rx = rx[i];
    pk[i].rz = rz[i];
  }
  std::vector<TrField> tf((size_t)std::max(ns, 1) * 13);
  for (int s = 0; s < ns; ++s)
    for (int k = 1; k <= 12; ++k)
      if (fields_[s][k].solved) {
        tf[(size_t)s * 13 + k].T = fields_[s][k].T.as<double>();
        tf[(size_t)s * 13 + k].G = fields_[s][k].Gout.as<double2>();
      }
  // the entry search's seafloor-node times, once per terminal field of
  // phases 1-3 (tf1, tf3, tf5) of every source
  std::vector<SfJob> jobs;
  {
    const int nsf = m_.nx;
    size_t nj = 0;
    for (int s = 0; s < ns; ++s)
      for (int k : {1, 3, 5})
        if (fields_[s][k].solved) ++nj;
    d_sft_.alloc(std::max<size_t>(nj, 1) * nsf * sizeof(double));
    if (!d_sft_.p) return "device allocation failed (seafloor times)";
    size_t j = 0;
    for (int s = 0; s < ns; ++s)
      for (int k : {1, 3, 5})
        if (fields_[s][k].solved) {
          SfJob J;
          J.T = fields_[s][k].T.as<double>();
          J.reg = kTf[k].reg;
          J.out = d_sft_.as<double>() + j * nsf;
          tf[(size_t)s * 13 + k].sft = J.out;
          jobs.push_back(J);
          ++j;
        }
  }
  std::string e;
  if (!(e = put_vec(d_picks_, pk.data(), (size_t)npick, stream_)).empty()) return e;
  if (!(e = put_vec(d_trfields_, tf.data(), tf.size(), stream_)).empty()) return e;
  if (!jobs.empty()) {
    if (!(e = put_vec(d_sfjobs_, jobs.data(), jobs.size(), stream_)).empty()) return e;
    tr_sf_times(d_trmodel_.as<TrModel>(), d_sfjobs_.as<SfJob>(), (int)jobs.size(), m_.nx, stream_);
    ++stats_.launches;
    TCK(cudaGetLastError());
  }
  if (!(e = put_vec(d_srcx_, src_x_.data(), (size_t)ns, stream_)).empty()) return e;
  if (!(e = put_vec(d_srcz_, src_z_.data(), (size_t)ns, stream_)).empty()) return e;
  const size_t np = (size_t)std::max(npick, 1);
  d_tcalc_.alloc(np * sizeof(double));
  d_valid_.alloc(np * sizeof(int));
  d_cnt_.alloc((np + 1) * sizeof(unsigned));
  d_off_.alloc((np + 1) * sizeof(unsigned long long));
  d_rowptr_.alloc((np + 1) * sizeof(int));
  d_entry_.alloc(np * 3 * sizeof(double));
  if (!d_tcalc_.p || !d_valid_.p || !d_cnt_.p || !d_off_.p || !d_rowptr_.p || !d_entry_.p)
    return "device allocation failed (picks)";
  // the timing events are released on every return
  struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    Events() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~Events() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } ev;
  cudaEventRecord(ev.a, stream_);
  rows_ = rows ? 0 : -1;
  nnz_ = 0;
  npick_ = -1;   // no rows to hand out unless this trace completes
  if (npick > 0) {
    const TrModel* M = d_trmodel_.as<TrModel>();
    unsigned* cnt = d_cnt_.as<unsigned>();
    TCK(cudaMemsetAsync(cnt, 0, (np + 1) * sizeof(unsigned), stream_));
    tr_launch(M, d_trfields_.as<TrField>(), d_srcx_.as<double>(), d_srcz_.as<double>(),
              d_picks_.as<TrPick>(), npick, d_tcalc_.as<double>(), d_valid_.as<int>(), cnt,
              nullptr, nullptr, nullptr, d_entry_.as<double>(), stream_);
    ++stats_.launches;
    TCK(cudaGetLastError());
    if (!rows) {   // times only (the line search's compute_rms_after_forward)
      TCK(cudaMemcpyAsync(t_calc, d_tcalc_.p, (size_t)npick * 8, cudaMemcpyDeviceToHost, stream_));
      TCK(cudaMemcpyAsync(valid, d_valid_.p, (size_t)npick * 4, cudaMemcpyDeviceToHost, stream_));
      cudaEventRecord(ev.b, stream_);
      TCK(cudaStreamSynchronize(stream_));
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ev.a, ev.b);
      trace_ms_ = ms;
      npick_ = npick;
      if (nnz) *nnz = 0;
      return std::string();
    }
    // offsets of each pick's contributions (64-bit: long rays times many picks)
    unsigned long long* off = d_off_.as<unsigned long long>();
    size_t tmp_bytes = 0;
    TCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, off, npick + 1, stream_));
    d_tmp_.alloc(std::max<size_t>(tmp_bytes, 16));
    TCK(cub::DeviceScan::ExclusiveSum(d_tmp_.p, tmp_bytes, cnt, off, npick + 1, stream_));
    unsigned long long total = 0;
    TCK(cudaMemcpyAsync(&total, off + npick, sizeof(total), cudaMemcpyDeviceToHost, stream_));
    TCK(cudaStreamSynchronize(stream_));
    if (total >= 0x7fffffffull) return "too many Frechet contributions for 32-bit CSR";
    const size_t nt = std::max<size_t>((size_t)total, 1);
    DevBuf keys, vals, keys2, vals2;
    keys.alloc(nt * 8);
    vals.alloc(nt * 8);
    keys2.alloc(nt * 8);
    vals2.alloc(nt * 8);
    if (!keys.p || !vals.p || !keys2.p || !vals2.p) return "device allocation failed (Frechet)";
    tr_launch(M, d_trfields_.as<TrField>(), d_srcx_.as<double>(), d_srcz_.as<double>(),
              d_picks_.as<TrPick>(), npick, d_tcalc_.as<double>(), d_valid_.as<int>(), cnt, off,
              keys.as<unsigned long long>(), vals.as<double>(), nullptr, stream_);
    ++stats_.launches;
    TCK(cudaGetLastError());
    const int n = (int)total;
    int end_bit = 32;
    while (end_bit < 63 && (1ull << (end_bit - 32)) <= (unsigned long long)npick) ++end_bit;
    // stable sort by (pick, parameter): contributions of one entry stay in
    // segment order
    size_t sb = 0;
    TCK(cub::DeviceRadixSort::SortPairs(nullptr, sb, keys.as<unsigned long long>(),
                                        keys2.as<unsigned long long>(), vals.as<double>(),
                                        vals2.as<double>(), n, 0, end_bit, stream_));
    d_tmp_.alloc(std::max<size_t>(sb, 16));
    TCK(cub::DeviceRadixSort::SortPairs(d_tmp_.p, sb, keys.as<unsigned long long>(),
                                        keys2.as<unsigned long long>(), vals.as<double>(),
                                        vals2.as<double>(), n, 0, end_bit, stream_));
    // sum equal keys
    DevBuf nruns;
    nruns.alloc(16);
    size_t rb = 0;
    TCK(cub::DeviceReduce::ReduceByKey(nullptr, rb, keys2.as<unsigned long long>(),
                                       keys.as<unsigned long long>(), vals2.as<double>(),
                                       vals.as<double>(), nruns.as<int>(), ::cuda::std::plus<>{}, n, stream_));
    d_tmp_.alloc(std::max<size_t>(rb, 16));
    TCK(cub::DeviceReduce::ReduceByKey(d_tmp_.p, rb, keys2.as<unsigned long long>(),
                                       keys.as<unsigned long long>(), vals2.as<double>(),
                                       vals.as<double>(), nruns.as<int>(), ::cuda::std::plus<>{}, n, stream_));
    int nu = 0;
    TCK(cudaMemcpyAsync(&nu, nruns.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TCK(cudaStreamSynchronize(stream_));
    // drop zero entries, count each row, place the survivors
    DevBuf flag, pos, rcnt;
    flag.alloc((size_t)std::max(nu, 1) * 4);
    pos.alloc((size_t)std::max(nu, 1) * 4);
    rcnt.alloc((np + 1) * 4);
    if (!flag.p || !pos.p || !rcnt.p) return "device allocation failed (Frechet rows)";
    TCK(cudaMemsetAsync(rcnt.p, 0, (np + 1) * 4, stream_));
    if (nu > 0)
      k_keep<<<(nu + 255) / 256, 256, 0, stream_>>>(keys.as<unsigned long long>(),
                                                     vals.as<double>(), nu, flag.as<int>(),
                                                     rcnt.as<int>());
    ++stats_.launches;
    size_t qb = 0;
    TCK(cub::DeviceScan::ExclusiveSum(nullptr, qb, flag.as<int>(), pos.as<int>(), std::max(nu, 1),
                                      stream_));
    size_t qb2 = 0;
    TCK(cub::DeviceScan::ExclusiveSum(nullptr, qb2, rcnt.as<int>(), d_rowptr_.as<int>(),
                                      npick + 1, stream_));
    d_tmp_.alloc(std::max<size_t>(std::max(qb, qb2), 16));
    if (nu > 0)
      TCK(cub::DeviceScan::ExclusiveSum(d_tmp_.p, qb, flag.as<int>(), pos.as<int>(), nu, stream_));
    TCK(cub::DeviceScan::ExclusiveSum(d_tmp_.p, qb2, rcnt.as<int>(), d_rowptr_.as<int>(),
                                      npick + 1, stream_));
    int kept = 0;
    TCK(cudaMemcpyAsync(&kept, d_rowptr_.as<int>() + npick, sizeof(int), cudaMemcpyDeviceToHost,
                        stream_));
    TCK(cudaStreamSynchronize(stream_));
    d_col_.alloc((size_t)std::max(kept, 1) * 4);
    d_val_.alloc((size_t)std::max(kept, 1) * 8);
    if (!d_col_.p || !d_val_.p) return "device allocation failed (Frechet rows)";
    if (nu > 0)
      k_scatter_rows<<<(nu + 255) / 256, 256, 0, stream_>>>(
          keys.as<unsigned long long>(), vals.as<double>(), flag.as<int>(), pos.as<int>(), nu,
          d_col_.as<int>(), d_val_.as<double>());
    ++stats_.launches;
    TCK(cudaGetLastError());
    nnz_ = kept;
    rows_ = npick;
    TCK(cudaMemcpyAsync(t_calc, d_tcalc_.p, (size_t)npick * 8, cudaMemcpyDeviceToHost, stream_));
    TCK(cudaMemcpyAsync(valid, d_valid_.p, (size_t)npick * 4, cudaMemcpyDeviceToHost, stream_));
  }
  cudaEventRecord(ev.b, stream_);
  TCK(cudaStreamSynchronize(stream_));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ev.a, ev.b);
  trace_ms_ = ms;
  npick_ = npick;
  if (nnz) *nnz = nnz_;
  return std::string();
}

std::string Engine::trace_entries(double* water_time, double* entry_x, double* entry_z) {
  cudaSetDevice(device_);
  if (npick_ < 0) return "no completed trace";
  if (npick_ == 0) return std::string();
  std::vector<double> e((size_t)npick_ * 3);
  TCK(cudaMemcpyAsync(e.data(), d_entry_.p, e.size() * sizeof(double), cudaMemcpyDeviceToHost,
                      stream_));
  TCK(cudaStreamSynchronize(stream_));
  for (int p = 0; p < npick_; ++p) {
    if (entry_x) entry_x[p] = e[3 * (size_t)p];
    if (entry_z) entry_z[p] = e[3 * (size_t)p + 1];
    if (water_time) water_time[p] = e[3 * (size_t)p + 2];
  }
  return std::string();
}

std::string Engine::frechet_rows(int* row_ptr, int* col, double* val, int base) {
  cudaSetDevice(device_);
  if (npick_ < 0) return "no picks traced";
  if (rows_ < 0) return "no picks traced with Frechet rows (the last trace computed times only)";
  if (row_ptr) {
    std::vector<int> rp(npick_ + 1, 0);
    if (npick_ > 0)
      TCK(cudaMemcpy(rp.data(), d_rowptr_.p, (size_t)(npick_ + 1) * 4, cudaMemcpyDeviceToHost));
    for (int i = 0; i <= npick_; ++i) row_ptr[i] = rp[i] + base;
  }
  if (nnz_ > 0) {
    if (col) {
      TCK(cudaMemcpy(col, d_col_.p, (size_t)nnz_ * 4, cudaMemcpyDeviceToHost));
      if (base == 0)
        for (long long k = 0; k < nnz_; ++k) col[k] -= 1;   // contributions carry 1-based ids
    }
    if (val) TCK(cudaMemcpy(val, d_val_.p, (size_t)nnz_ * 8, cudaMemcpyDeviceToHost));
  }
  return std::string();
}

}  // namespace fmt2d
