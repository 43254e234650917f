// Host engine: device copy of the model and the per-source time fields, and
// the phase/stage recipe of the forward solve.
#pragma once
#include <cuda_runtime.h>
#include <array>
#include <memory>
#include <string>
#include <vector>
#include "eik64.cuh"
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

// Owning device buffer (move-only: a copy would free the memory twice).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      free_();
      p = o.p;
      bytes = o.bytes;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  void alloc(size_t n);
  void free_();
  ~DevBuf() { free_(); }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Static device data of one region (slot layout of model.h).
struct DevRegionStore {
  DevBuf code, vel64, izc, iface_x, iface_z, r0, r1, slot_of_node;
  size_t nslots = 0;
  double vmax = 1.0;   // largest region velocity (sets the window step)
};

// One solved (source, time field): FP64 time and final gradient per slot,
// plus the solver state of the field.
struct FieldStore {
  DevBuf T, G, Gout, fl, seed, clock;
  DevBuf hwpre;   // PmP up: solved times at the head-wave sweep nodes (nx)
  bool solved = false;
};

struct SolveStats {
  long long rounds = 0;       // steps of the longest field solve, summed over batches
  unsigned long long steps_sum = 0;   // steps summed over every field
  int batches = 0, final_passes = 0;   // stage batches; solve passes (each ends in a fixed-point check)
  double round_ms = 0.0;      // device time of the step loops
  unsigned long long evals = 0, writes = 0, passed = 0;   // node evaluations; writes; deferred nodes passed over
  unsigned long long unsettled = 0;   // nodes the last fixed-point check re-listed
  unsigned long long capped = 0;      // fields that reached the step cap
  long long launches = 0;     // kernels launched since the last forward began
  long long nodes = 0;        // region nodes of the time fields solved
  double cycles[5] = {0, 0, 0, 0, 0};   // SM cycles of the solve phases, summed over fields
  unsigned long long cut_evals = 0;     // evaluations of nodes next to an interface
  unsigned long long cut_steps = 0;     // steps that evaluated such a node
};

// Stage chains solved concurrently: a stage's chain is that of its level-0
// ancestor (Pg with Pg_ss, PsedP, PmP, Pg_ss2).
constexpr int kChains = 4;
inline int chain_of(int tf) {
  static const int c[13] = {0, 0, 1, 1, 2, 2, 0, 0, 0, 3, 3, 3, 3};
  return c[tf];
}

// A stream and the solver scratch of one stage chain.
struct SolveLane {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  DevBuf fields, up, step, sx, sz, seeds, which, hw, hwpre, ctr;
  DevBuf sTn, sGn, sfln, spend, sclaim, slist, sover, sinq, scnt;
  SolveStats stats;
  bool not_converged = false;
  // pinned staging of the lane's small host <-> device copies (descriptors,
  // counters): a pageable copy goes through the driver's shared staging
  // path, where a read-back waiting for one chain's solve holds up the other
  // chains' uploads and so serialises the chains
  char* pin = nullptr;
  size_t pin_cap = 0, pin_used = 0;
  void free_all() {
    for (DevBuf* b : {&fields, &up, &step, &sx, &sz, &seeds, &which, &hw, &hwpre, &ctr, &sTn, &sGn, &sfln,
                      &spend, &sclaim, &slist, &sover, &sinq, &scnt})
      b->free_();
    if (pin) cudaFreeHost(pin);
    pin = nullptr;
    pin_cap = pin_used = 0;
  }
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
  // the same into device memory of the caller (any may be null)
  std::string get_field_device(int src, int tf, double* T, double* gx, double* gz);
  // Ray backtrace and Frechet rows of npick picks (source index, phase 1..5,
  // receiver x, z) on the fields of the last forward; the rows stay on the
  // device until frechet_rows copies them out (CSR over all picks, invalid
  // picks empty, columns 1-based parameter ids unless base 0).
  // rows = false: receiver times and valid flags only (no Frechet rows).
  std::string trace(const int* src, const int* phase, const double* rx, const double* rz,
                    int npick, double* t_calc, int* valid, long long* nnz, bool rows = true);
  std::string frechet_rows(int* row_ptr, int* col, double* val, int base);
  // per pick of the last trace: the ray's receiver end (seafloor entry point
  // of an in-water pick of phases 1-3, else the receiver) and the water time
  std::string trace_entries(double* water_time, double* entry_x, double* entry_z);
  // Misfit 0.5*sum(((t_calc - t_obs)/sigma)^2) over the valid picks with
  // t_obs >= 0 (phases 1-5) on the fields of the last forward (traced here:
  // t_calc, valid), and its gradient w.r.t. the propagation-grid velocity
  // (nx*nz, ix fastest; may be null) and the interface node depths (5*nx,
  // interfaces 1..5; may be null) by the discrete adjoint of the fields.
  // info (8 values, may be null): re-derived values that differ from the
  // stored times, links outside their node's reader list, nodes the reverse
  // sweep did not reach, its most rounds, fields, reached nodes, ms.
  std::string misfit_gradient(const int* src, const int* phase, const double* rx,
                              const double* rz, const double* t_obs, const double* sigma,
                              int npick, double* misfit, double* t_calc, int* valid,
                              double* grad_vel, double* grad_iface, double* info);
  double trace_ms() const { return trace_ms_; }
  long long frechet_nnz() const { return nnz_; }
  const Model& model() const { return m_; }
  cudaStream_t stream() const { return stream_; }
  const SolveStats& stats() const { return stats_; }
  // the last forward failed because a field did not reach its fixed point
  bool not_converged() const { return not_converged_; }
  // window step in cells at the region's largest velocity; 0: none for point
  // sources, kIfaceWindowCells for stages seeded along an interface
  double window_cells = 0.0;
  static constexpr double kIfaceWindowCells = 32.0;
  // the default window of stages seeded along an interface (cells; 0: none)
  double iface_window_cells = kIfaceWindowCells;
  static constexpr long long kDefaultMaxSteps = 4000000;
  long long max_steps = kDefaultMaxSteps;  // safety cap on the steps of one field's solve
  int max_passes = 6;             // solve passes (each followed by a check of every node)
  int solve_threads = 0;          // threads of a field's solve block (0: the default)
  // device pointers of a solved field (FP64 time, double2 final gradient per slot)
  const double* field_t(int src, int tf) const { return fields_[src][tf].T.as<double>(); }
  const double2* field_g(int src, int tf) const { return fields_[src][tf].Gout.as<double2>(); }
  const DevRegionStore& region(int r) const { return reg_[r]; }
  double source_z(int src) const { return src_z_[src]; }
  double source_x(int src) const { return src_x_[src]; }
  int nsrc() const { return (int)fields_.size(); }

 private:
  std::string solve_level(SolveLane& L, const std::vector<std::pair<int, int>>& items);
  std::string upload_trace_tables();
  void ensure_sources(int nsrc);
  Fld64 field_view(int src, int tf) const;
  int device_;
  cudaStream_t stream_ = nullptr;
  Model m_;
  DevRegionStore reg_[7];
  DevBuf ifc_buf_[6][6];      // z, nx, nz, vel_top, vel_bot, izc
  Ifc64 ifc_[6];
  DevBuf hw_slot_, hw_v_;
  std::vector<int> hw_slot_h_, hw_vslot_h_;   // host copies; the slot each hw_v value comes from
  long long model_version_ = 0;               // bumped by every upload
  // the adjoint's slot -> grid velocity maps per region (slot_velocity_map:
  // rp, slot, w, zrp, zslot, zside, zdv) and the model version they belong to
  DevBuf adj_map_[7][7];
  long long adj_map_version_[7] = {-1, -1, -1, -1, -1, -1, -1};
  std::vector<std::array<FieldStore, 13>> fields_;
  std::vector<double> src_x_, src_z_;
  DevBuf export_;             // region-order copy of a field being read back
  SolveLane lanes_[kChains];
  cudaEvent_t ev_start_ = nullptr;
  DevBuf d_pvel_, d_invidx_, d_xpos_, d_trmodel_, d_picks_, d_trfields_, d_srcx_, d_srcz_,
      d_tcalc_, d_valid_, d_cnt_, d_off_, d_rowptr_, d_tmp_, d_col_, d_val_, d_sft_, d_sfjobs_,
      d_entry_;
  int npick_ = -1, rows_ = 0;
  long long nnz_ = 0;
  double trace_ms_ = 0.0;
  unsigned* h_count_ = nullptr;
  SolveStats stats_;
  bool not_converged_ = false;
};

}  // namespace fmt2d
