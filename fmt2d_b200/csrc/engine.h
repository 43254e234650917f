// Host engine: device copy of the model and the per-source time fields, and
// the phase/stage recipe of the forward solve.
#pragma once
#include <cuda_runtime.h>
#include <array>
#include <memory>
#include <string>
#include <vector>
#include "fields.cuh"
#include "model.h"

namespace fmt2d {

// Time fields of the five phases (inversion2d.f90:4214-4476 via the tables of
// invert2d_main.f90:564-700): region, start interface, parent field.
struct TfInfo {
  int reg, istart, parent, level, dst_side, target_side, reflect, water_up;
};
extern const TfInfo kTf[13];
// phase -> time fields it needs (bit tf)
unsigned phase_fields(int phase_mask);

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void alloc(size_t n);
  void free_();
  ~DevBuf() { free_(); }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct DevRegionStore {
  DevBuf code, vel, vel64, iface_dz, izc, iface_x, iface_z, r0, r1, slot_of_node;
  DevRegion R;
  DevRegionX X;
  size_t nslots = 0;
  int ntiles = 0;
  double vmean = 1.0;   // mean region velocity (sets the processing band)
};

struct FieldStore {
  DevBuf t2, g2, gout, susp, act, seed, sflag, tkey, front;
  bool solved = false;
};

struct SolveStats {
  int rounds = 0, batches = 0, final_passes = 0;
  long long tile_visits = 0;
  double round_ms = 0.0;     // device time of the round kernels
  // device counters: sweep passes, warp row/column steps, visits that hit
  // the pass cap, node updates
  unsigned long long passes = 0, steps = 0, capped = 0, updates = 0;
  long long launches = 0;     // kernels launched since the last forward began
  long long nodes = 0;        // region nodes of the time fields solved
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  std::string upload(const Model& m);
  // Solve all time fields of the enabled phases for sources at the given x
  // (placed on the seafloor), one slot per source.
  std::string forward(const double* sx, int nsrc, int phase_mask);
  std::string get_field(int src, int tf, double* T, double* gx, double* gz);
  const Model& model() const { return m_; }
  cudaStream_t stream() const { return stream_; }
  const SolveStats& stats() const { return stats_; }
  int max_passes = 64;     // directional sweeps per tile visit before it re-queues itself
  double band_tiles = 1.5; // processing band: this many tile widths at the mean velocity
  int max_rounds = 4000;   // safety cap on rounds per batch
  // device pointers of a solved field (float2 time, float2 gradient per slot)
  const float* field_t(int src, int tf) const { return fields_[src][tf].t2.as<float>(); }
  const float* field_g(int src, int tf) const { return fields_[src][tf].gout.as<float>(); }
  const DevRegionStore& region(int r) const { return reg_[r]; }
  double source_z(int src) const { return src_z_[src]; }
  double source_x(int src) const { return src_x_[src]; }
  int nsrc() const { return (int)fields_.size(); }

 private:
  std::string solve_level(const std::vector<std::pair<int, int>>& items);
  void ensure_sources(int nsrc);
  int device_;
  cudaStream_t stream_ = nullptr;
  Model m_;
  DevRegionStore reg_[7];
  DevBuf ifc_buf_[6][6];      // z, nx, nz, vel_top, vel_bot, izc
  DevIface ifc_[6];
  DevBuf hw_slot_, hw_v_;
  std::vector<std::array<FieldStore, 13>> fields_;
  std::vector<double> src_x_, src_z_;
  DevBuf d_fields_, d_xs_, d_seeds_, d_sx_, d_sz_, d_count_, d_gout_, d_susp_, d_up_, d_which_,
      d_scratch_, d_counters_, d_queue_;
  unsigned* h_count_ = nullptr;
  int visit_blocks_ = 1;
  SolveStats stats_;
};

}  // namespace fmt2d
