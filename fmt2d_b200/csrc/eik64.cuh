// FP64 eikonal solver: device data of the fields being solved and the
// kernels that seed, solve and post-process them.
//
// Times and gradients are FP64 on the device so that every candidate time is
// the same IEEE double the reference's FP64 fast marching computes (the
// stencil keeps the reference's expression order and is compiled without FMA
// contraction).  The reference's acceptance order decides exact ties and
// near-threshold second-order switches by the last bit of those doubles; an
// FP32 field cannot reproduce them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fmt2d {

constexpr double kHugeD = 1.0e20;     // mod_fmt2d.f90:616 huge_time
constexpr double kReachD = 1.0e19;    // a time below this is reached
constexpr uint8_t kFlSeed = 1, kFlCopy = 2, kFlSusp = 4;

// One time field being solved (static region data, state and solver scratch).
struct Fld64 {
  const uint32_t* code = nullptr;   // per slot (model.h bits)
  const double* vel = nullptr;      // per slot, FP64
  const int* izc = nullptr;         // 2*pitch: cut-cell top row (absolute) of the interface nodes
  const double* ifx = nullptr;      // pitch: interface node x
  const double* ifz = nullptr;      // 2*pitch: interface node z (top, bottom)
  int H = 0, pitch = 0, z_lo = 0, nx = 0, nz = 0;
  double x0 = 0, dx = 0, tol = 0;
  double eps = 0.0;                 // change threshold (0: solve to the last bit)
  double* T = nullptr;              // per slot
  double2* G = nullptr;             // per slot: gradient of the winning candidate
  double2* Gout = nullptr;          // per slot: final gradient (suspect nodes refitted)
  uint8_t* fl = nullptr;            // per slot: kFlSeed | kFlCopy | kFlSusp
  double4* seed = nullptr;          // per slot: seeded (T, gx, gz, -)
  double* clock = nullptr;          // [0] window end, [1] window step
  int frozen_slot = -1;             // node fixed at the source (never a trigger)
  // solver scratch (per slot unless stated)
  double* Tn = nullptr;             // new time staged by the evaluation phase
  double2* Gn = nullptr;            // new gradient staged
  uint8_t* fln = nullptr;           // new flags staged
  double* pend = nullptr;           // time a deferred node waits with (< 0: none)
  unsigned long long* claim = nullptr;   // bits of the new time of a node moving this step
  unsigned* list_in = nullptr;      // nodes to start from (seeds, re-listed nodes)
  unsigned* over = nullptr;         // 3*nslots: list overflow (two lists) and commit overflow
  unsigned* inq = nullptr;          // bitset over slots: listed (when not in shared memory)
  unsigned* wait = nullptr;         // bitset over slots: waiting (when not in shared memory)
  unsigned* moving = nullptr;       // bitset over slots: moving this step (when not in shared memory)
  unsigned* cnt = nullptr;          // [0] list_in length, [1] unsettled nodes found by a check,
                                    // [2] error (1: step cap), [3] steps of the last solve
#if defined(__CUDACC__)
  __host__ __device__
#endif
  int nslots() const { return (H + 2) * pitch; }
};

// Interface data used by the seeding of a stage (FP64, nx nodes).
struct Ifc64 {
  const double* z = nullptr;
  const double* nrm_x = nullptr;
  const double* nrm_z = nullptr;
  const double* vel_top = nullptr;
  const double* vel_bot = nullptr;
  const int* izc = nullptr;
};

struct Seed64 {
  int dst;                          // index of the destination field in the batch
  const double* src_T = nullptr;    // parent field time
  const double2* src_G = nullptr;   // parent field final gradient
  int src_row = 0, src_pitch = 0;   // interface row of the parent field
  Ifc64 ifc;
  const int* r0 = nullptr;          // per column first/last row of the target region
  const int* r1 = nullptr;
  int dst_side = 0, reflect = 0, target_side = 0;
};

// Solver counters summed over a batch: evaluations, committed writes that
// changed a node, waiting nodes released by the window, steps (summed over
// fields), largest step count of one field.
// Also: SM cycles of the solve's phases summed over fields (evaluate,
// arbitrate and commit, the evaluate phases of steps that evaluated a node
// next to an interface, spread, window release), evaluations of nodes next
// to an interface (cut-cell updates) and the steps that had one.
enum {
  kCtrEval = 0, kCtrWrite, kCtrPass, kCtrSteps, kCtrMaxSteps,
  kCtrCycEval, kCtrCycArb, kCtrCycEvalCut, kCtrCycSpread, kCtrCycRelease, kCtrCut, kCtrStepsCut,
  kCtrN
};

void e64_fill(Fld64* f, int nf, size_t max_slots, cudaStream_t st);
void e64_init_source(Fld64* f, const double* sx, const double* sz, int nf, cudaStream_t st);
void e64_seed_iface(Fld64* f, const Seed64* d, int nd, int nx, cudaStream_t st);
// List every seeded node and its neighbours in list_in; set the windows.
void e64_start(Fld64* f, int nf, size_t max_slots, const double* step, cudaStream_t st);
// Solve every field of the batch from its list_in (one thread block per
// field, all steps in one launch; max_tiles: the most tiles of a field,
// e64_tiles).  max_steps bounds the steps of a field;
// a field that reaches it sets cnt[2] = 1.
// threads: the solve block's size, one of e64_solve_sizes (others: the
// default); the result does not depend on it.
void e64_solve(Fld64* f, int nf, size_t max_slots, int max_tiles, long long max_steps,
               unsigned long long* ctr, int threads, cudaStream_t st);
const int* e64_solve_sizes(int* n);
// Tiles of a field's waiting-node index, and the most a field may have.
int e64_tiles(const Fld64& f);
int e64_tiles_max();
// Fixed-point check of every node: a node whose evaluation would change it
// is listed in list_in and counted in cnt[1].
void e64_verify(Fld64* f, int nf, size_t max_slots, cudaStream_t st);
void e64_finish(Fld64* f, int nf, size_t max_slots, const int* water_up, cudaStream_t st);
// PmP head-wave sweep of the selected fields; pre (device array of nsel
// pointers, may be null, entries may be null) receives each field's solved
// times at the nx sweep nodes before the sweep lowers them.
void e64_headwave(Fld64* f, const int* hw_slot, const double* hw_v, double dx_if, int nx,
                  double* scratch, const int* which, int nsel, double* const* pre,
                  cudaStream_t st);
void e64_export(const double* T, const double2* G, const int* slot_of_node, int nnode, double* oT,
                double* ogx, double* ogz, cudaStream_t st);

}  // namespace fmt2d
