// Device data for stage coupling and field post-processing.
#pragma once
#include "eikonal.cuh"

namespace fmt2d {

// FP64 interface data (one per interface, nx nodes).
struct DevIface {
  const double* z = nullptr;
  const double* nrm_x = nullptr;
  const double* nrm_z = nullptr;
  const double* vel_top = nullptr;
  const double* vel_bot = nullptr;
  const int* izc = nullptr;       // cut-cell top row, -1 none
};

// Extra per-region data used outside the sweeps.
struct DevRegionX {
  const double* vel64 = nullptr;  // FP64 region velocity per slot
  const double* iface_x = nullptr;// node x of the interface rows (pitch)
  const double* iface_z = nullptr;// 2*pitch node depths of the top/bottom rows
  const int* r0 = nullptr;        // per column first/last region row
  const int* r1 = nullptr;
  int itop = 0, ibot = 0, id = 0, nz = 0;
};

// Stage seeding from an interface: where the previous field is read and how.
struct SeedDesc {
  DevField dst;
  DevRegionX dstx;
  const float* src_t = nullptr;   // previous field T (float2 per slot)
  const float* src_g = nullptr;   // previous field final gradient (float2 per slot)
  int src_row = 0;                // interface row of the previous field (slot base / pitch)
  int src_pitch = 0;
  DevIface ifc;                   // interface the stage starts from
  int dst_side = 0;               // 0: starts from the target's top interface, 1: bottom
  int reflect = 0;                // apply reflect_gradient_at_interface first
  int target_side = 0;            // +1 target region below the interface, -1 above
};

}  // namespace fmt2d
