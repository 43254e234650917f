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
  unsigned* act = nullptr;           // 2 * ntiles round flags
  float4* seed = nullptr;            // per slot: seeded (time hi, lo, gradient) or huge
  uint8_t* sflag = nullptr;          // per slot: bit 0 seeded, bit 1 value copied from a
                                     // coincident node
  int frozen_slot = -1;              // node fixed at initialisation (never a trigger)
  int tile_base = 0;                 // first block of this field in the launch
};

// A time change above this many seconds is propagated to neighbouring tiles;
// smaller changes are kept locally (the parity tolerance is 0.5 ms).
constexpr float kSigDT = 1.0e-6f;
// Changes above this re-activate the stencil neighbours inside a tile.
constexpr double kLocalDT = 1.0e-8;

// Tile activation bits: why a tile must be visited.
enum : unsigned {
  kActAll = 1u,            // seeded, unconverged or flagged by the final pass
  kActTop = 2u, kActBot = 4u, kActLeft = 8u, kActRight = 16u,
  kActTL = 32u, kActTR = 64u, kActBL = 128u, kActBR = 256u,
};
constexpr uint8_t kFlagSeed = 1, kFlagCopy = 2;

}  // namespace fmt2d
