// FP64 tiled eikonal solver: device data of the fields being solved and the
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

// One time field being solved (static region data plus state).
struct Fld64 {
  const uint32_t* code = nullptr;   // per slot (model.h bits)
  const double* vel = nullptr;      // per slot, FP64
  const int* izc = nullptr;         // 2*pitch: cut-cell top row (absolute) of the interface nodes
  const double* ifx = nullptr;      // pitch: interface node x
  const double* ifz = nullptr;      // 2*pitch: interface node z (top, bottom)
  int H = 0, pitch = 0, z_lo = 0, nx = 0, nz = 0;
  double x0 = 0, dx = 0, tol = 0;
  double* T = nullptr;              // per slot
  double2* G = nullptr;             // per slot: gradient of the winning candidate
  double2* Gout = nullptr;          // per slot: final gradient (suspect nodes refitted)
  uint8_t* fl = nullptr;            // per slot: kFlSeed | kFlCopy | kFlSusp
  double4* seed = nullptr;          // per slot: seeded (T, gx, gz, -)
  double* clock = nullptr;          // [0] window end, [1] window step, [2] changed this step
  int frozen_slot = -1;             // node fixed at the source (never a trigger)
  unsigned gbase = 0;               // global id of slot 0 (ids of a batch are contiguous)
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

void e64_fill(Fld64* f, int nf, size_t max_slots, cudaStream_t st);
void e64_init_source(Fld64* f, const double* sx, const double* sz, int nf, cudaStream_t st);
void e64_seed_iface(Fld64* f, const Seed64* d, int nd, int nx, cudaStream_t st);
// List every seeded node and its neighbours (list/cnt), set the windows.
void e64_start(Fld64* f, int nf, size_t max_slots, const double* step, unsigned* list,
               unsigned* cnt, unsigned* inq, cudaStream_t st);
// One step over the list `in` (see k_step); ver / pend: per node input
// version and deferred-time record, zeroed at the start of a batch.
void e64_step(Fld64* f, int nf, const unsigned* in, const unsigned* in_cnt, unsigned* out,
              unsigned* out_cnt, unsigned* zero_cnt, unsigned* inq, unsigned* done, unsigned* ver,
              unsigned long long* pend, int grid, unsigned long long* ctr, cudaStream_t st);
void e64_verify(Fld64* f, int nf, size_t max_slots, unsigned* list, unsigned* cnt, unsigned* inq,
                unsigned* bad, cudaStream_t st);
void e64_finish(Fld64* f, int nf, size_t max_slots, const int* water_up, cudaStream_t st);
void e64_headwave(Fld64* f, const int* hw_slot, const double* hw_v, double dx_if, int nx,
                  double* scratch, const int* which, int nsel, cudaStream_t st);
void e64_export(const double* T, const double2* G, const int* slot_of_node, int nnode, double* oT,
                double* ogx, double* ogz, cudaStream_t st);
int e64_step_grid(int device);

}  // namespace fmt2d
