// Discrete adjoint of the eikonal fields: device data.
//
// At the solver's fixed point every reached node holds the value of one
// winning update (a regular quadrant, a cut-cell time_from_1/2 event, a copy
// from a coincident node, or a seed).  That update is a smooth function of a
// few node times, slot velocities and, for a stage hand-off, one node time of
// the parent field.  Its partial derivatives are the node's link; the links
// form a graph without cycles (every update reads earlier times), and the
// adjoint of a node's time is its direct term plus the sum over the nodes
// that read it of (their adjoint) x (their link weight), taken in reverse
// order of that graph.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "eik64.cuh"

namespace fmt2d {

enum AdjKind : int {
  kAdjNone = 0,     // unreached (no link)
  kAdjRegular,      // regular_update2d quadrant
  kAdjRay,          // time_from_1_node2d straight ray
  kAdjCopy,         // a coincident member's time handed over
  kAdjPlane,        // time_from_2_nodes2d plane front
  kAdjSource,       // point-source corner seed
  kAdjHandOff,      // stage hand-off seed (interface node or grid node next to it)
  kAdjFixed,        // constant (the source node itself)
  kAdjMismatch      // the re-derived value differs from the stored one (counted)
};

// The winning update of one node, linearised.
struct AdjLink {
  int t[4];         // same-field slots whose times the value reads (-1: none)
  int v[4];         // slots whose velocities it reads (-1: none)
  double wt[4], wv[4];
  int xref;         // parent-field slot whose time a hand-off seed reads (-1: none)
  int kind;         // AdjKind
  double xw;        // its weight
  int z[3];         // interface nodes whose depths it reads: interface id * 65536 + column
  double wz[3];
};

// One field's adjoint state.
struct AdjField {
  Fld64 F;               // the solved field (frozen_slot set as the solve had it)
  AdjLink* link = nullptr;
  unsigned* cnt = nullptr;   // per slot: links reading its time that are not yet processed
  double* lam = nullptr;     // per slot: adjoint of the node's time
  double* d = nullptr;       // per slot: direct terms (picks, a child stage's hand-off)
  double* gv = nullptr;      // per slot: misfit gradient w.r.t. the slot velocity
  unsigned* fa = nullptr;    // work lists (nslots each)
  unsigned* fb = nullptr;
  unsigned* ctr = nullptr;   // kAdjCtr* counters
  double sx = 0, sz = 0;     // source position (level-0 fields)
  Seed64 seed;               // hand-off from the parent field (level > 0; seed.src_T set)
  int level = 0;
  int itop = 0, ibot = 0;    // the region's top / bottom interface ids
  int seed_iface = 0;        // the interface a hand-off seeds from (level > 0)
  double* gzf = nullptr;     // 3*nx: depth gradient of the top, bottom and seed interfaces' nodes
  // the region's slots whose velocity is sampled off an interface, by column
  // (slot_velocity_map): slot, side, d velocity / d depth
  const int* zrp = nullptr;
  const int* zslot = nullptr;
  const int* zside = nullptr;
  const double* zdv = nullptr;
  // each node's readers (links reading its time) as lists, built once per
  // level: count and offset into the level's reader arrays
  unsigned* rcnt = nullptr;
  unsigned* roff = nullptr;
};

enum {
  kAdjCtrFront = 0,   // nodes without readers (the reverse sweep's first list)
  kAdjCtrDone,        // nodes the reverse sweep processed
  kAdjCtrMismatch,    // re-derived values that differ from the stored times
  kAdjCtrRounds,      // rounds of the reverse sweep
  kAdjCtrReached,     // reached nodes (links)
  kAdjCtrUnlisted,    // a link read a node whose reader list lacks the linking node
  kAdjCtrN = 8
};

// Links of every slot of every field; counts each slot's readers.
void adj_links(AdjField* f, int nf, size_t max_slots, cudaStream_t st);
// Each node's readers (reader slot, link weight) at roff, in the fixed order
// the sweep sums them (spread targets in order, then link entries in order).
void adj_readers(AdjField* f, int nf, size_t max_slots, int* rk, double* rw, cudaStream_t st);
// The reverse sweep (one block per field) over the reader lists and the
// velocity gradient per slot.
void adj_sweep(AdjField* f, int nf, size_t max_slots, const int* rk, const double* rw,
               cudaStream_t st);
// Hand-off terms: child field c's adjoint at its hand-off seeds is added to
// its parent's direct terms (pairs child[k] -> parent[k], parent interface row
// src_row of the child's seed descriptor).
void adj_handoff(AdjField* f, const int* child, const int* parent, int npair, int nx,
                 cudaStream_t st);
// PmP head-wave sweep, reversed: a field's direct terms on the swept (final)
// times become terms on the solved times (pre) and on the sweep velocities
// hw_v, whose gradient is added to the slot velocity each came from.
void adj_headwave(AdjField* f, const int* which, int nsel, const int* hw_slot,
                  const double* hw_v, const int* hw_vslot, double* const* pre, double dx_if,
                  int nx, double* scratch, cudaStream_t st);
// Exchange the stored (swept) and the solved (pre) times at the sweep nodes.
void adj_swap_pre(AdjField* f, const int* which, int nsel, const int* hw_slot,
                  double* const* pre, int nx, cudaStream_t st);
// Interface-depth gradient per field (gzf: the region's top and bottom
// interfaces and the hand-off interface, per column), then summed over the
// fields in order into giface[(iface - 1) * nx + col] (interfaces 1..5).
void adj_depth(AdjField* f, int nf, int nx, double* giface, cudaStream_t st);
// gvel[node] += sum over fields k, in order, of sum over the region map
// entries of the node of w * gv_k[slot] (map k: node-major CSR).
void adj_to_grid(const AdjField* f, int nf, const int* const* map_rp, const int* const* map_slot,
                 const double* const* map_w, size_t nnode, double* gvel, cudaStream_t st);

}  // namespace fmt2d
