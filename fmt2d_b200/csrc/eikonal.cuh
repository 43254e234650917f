// Device-side data of the tiled eikonal solver.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fmt2d {

constexpr int kTW = 32;            // tile width
constexpr int kTH = 32;            // tile height
constexpr int kHalo = 2;           // second-order stencil reach
constexpr int kSP = kTW + 2 * kHalo + 1;  // smem pitch (odd: conflict-free columns)
constexpr int kSR = kTH + 2 * kHalo;      // smem rows
constexpr int kSI = kTW + 2 * kHalo;      // interface entries per side
constexpr float kHugeF = 1.0e20f;
constexpr float kReachedF = 1.0e19f;     // T_hi below this: node reached

// Static geometry of one region on the device (slot layout of model.h).
struct DevRegion {
  const uint32_t* code = nullptr;
  const float* vel = nullptr;
  const float* iface_dz = nullptr;   // 2*pitch: z - z(cut-cell top row)
  const int* izc = nullptr;          // 2*pitch: cut-cell top row (absolute), -1 none
  int H = 0, pitch = 0, tiles_x = 0, tiles_y = 0, z_lo = 0, nx = 0;
  double dx = 0, x0 = 0, tol = 0;
};

// One time field being solved.
struct DevField {
  DevRegion R;
  float* Th = nullptr;               // time, high part (slot-indexed)
  float* Tl = nullptr;               // time, low part (T = Th + Tl)
  float* gx = nullptr;               // gradient during the solve
  float* gz = nullptr;
  unsigned* act = nullptr;           // per tile kTileWords words: active-node masks
                                     // (32 rows, then top and bottom interface rows)
  unsigned* tkey = nullptr;          // per tile: smallest pending time (float bits)
  unsigned* tvis = nullptr;          // per tile: visits so far in this solve
  float* front = nullptr;            // this field's current front time (device scalar)
  float band = 1.0f;                 // width of the processing band, seconds
  float4* seed = nullptr;            // per slot: seeded (time hi, lo, gradient) or huge
  uint8_t* sflag = nullptr;          // per slot: bit 0 seeded, bit 1 value copied from a
                                     // coincident node
  int frozen_slot = -1;              // node fixed at initialisation (never a trigger)
  int tile_base = 0;                 // first block of this field in the launch
};

// A time change above this many seconds is propagated to neighbouring tiles;
// smaller changes are kept locally (the parity tolerance is 0.5 ms).
constexpr float kSigDT = 1.0e-6f;
// Changes above this re-activate the stencil neighbours inside a tile (an
// order above the FP32 rounding of a re-evaluated time offset).
constexpr double kLocalDT = 1.0e-7;

// A tile visited more often than this in one solve only takes decreases from
// then on.  The replacement iteration can cycle where the second-order switch
// of two nodes depends on each other's gradients; taking decreases only ends
// such a cycle at its lower values.
constexpr unsigned kMonoVisits = 64;

constexpr int kTileWords = kTH + 2;      // active masks stored per tile
constexpr unsigned kKeyNone = 0x7f800000u; // +inf: no pending node
constexpr uint8_t kFlagSeed = 1, kFlagCopy = 2;

__device__ __forceinline__ unsigned key_of(float t) {
  return t >= kReachedF ? kKeyNone : __float_as_uint(fmaxf(t, 0.0f));
}

}  // namespace fmt2d
