// Device ray backtrace and Frechet rows (one thread per pick, FP64).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fmt2d {

// A region as the ray tracer reads it (slot layout of model.h).
struct TrRegion {
  const uint32_t* code = nullptr;
  const int* slot_of_node = nullptr;   // region node id - 1 -> slot (the reference's node order)
  const int* r0 = nullptr;             // per column: first / last grid row of the region
  const int* r1 = nullptr;             // (absolute, 0-based; r1 < r0: none)
  int z_lo = 0, H = 0, pitch = 0, itop = 0, ibot = 0, id = 0, nnode = 0;
};

// Model data shared by every pick.
struct TrModel {
  int nx = 0, nz = 0;
  double x0 = 0, dx = 0, tol = 0, vwater = 1.5;
  const double* vel = nullptr;        // propagation-grid velocity, ix fastest
  const double* xpos = nullptr;       // interface node x (= velocity-grid x)
  const double* ifz[6] = {};          // interface node depths, interfaces 1..5
  const int* inv_idx = nullptr;       // inversion numbering, 1-based, 0 inactive
  int iface_inv = 0, iface_start = 0, n_inv = 0;
  TrRegion reg[7];
};

// One pick: source (OBS) index, phase 1..5, receiver (shot) position.
struct TrPick {
  int src, phase;
  double rx, rz;
};

// Per pick: the fields of its source (indexed src*13 + tf) give T and the
// final gradient.
struct TrField {
  const double* T = nullptr;
  const double2* G = nullptr;
  const double* sft = nullptr;    // the field's time at every seafloor node (the entry
                                  // search's scan), for the terminal fields of phases 1-3
};

// One field whose seafloor-node times the entry search needs.
struct SfJob {
  const double* T = nullptr;
  int reg = 0;
  double* out = nullptr;          // nx values
};

// out[i] = the field's interpolated time at seafloor node i, for every job
// (the same interpolation the entry search applies, done once per field
// instead of once per pick).
void tr_sf_times(const TrModel* m, const SfJob* jobs, int njobs, int nx, cudaStream_t st);

// Trace every pick.  Pass 1 (rows == nullptr): t_calc, valid and the number
// of Frechet contributions of each pick (cnt).  Pass 2: the contributions
// themselves at off[pick] (keys = pick << 32 | parameter id, 1-based).
// entry (pass 1, may be null): per pick the receiver end of the ray (the
// seafloor entry point of an in-water pick of phases 1-3, else the receiver)
// and the water leg's time, 3 doubles.
void tr_launch(const TrModel* m, const TrField* fields, const double* src_x, const double* src_z,
               const TrPick* picks, int npick, double* t_calc, int* valid, unsigned* cnt,
               const unsigned long long* off, unsigned long long* keys, double* vals,
               double* entry, cudaStream_t st);

// Direct adjoint terms of the picks (the misfit's derivative with respect to
// the node times of each pick's terminal field): for target field k
// (tgt[k] = src*13 + tf) and each of its picks p = tpk[tp[k] .. tp[k+1]) in
// order, d[k][slot] += coef[p] * w for the nodes and bilinear weights through
// which its receiver-end time is read at the entry point recorded by the
// trace (entry, 3 doubles per pick).
void tr_adj_picks(const TrModel* m, const TrField* fields, const TrPick* picks,
                  const double* entry, const double* coef, const int* tgt, const int* tp,
                  const int* tpk, double* const* d, int ntgt, cudaStream_t st);

}  // namespace fmt2d
