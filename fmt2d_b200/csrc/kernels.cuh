// Kernel declarations shared between translation units.
#pragma once
#include "fields.cuh"

namespace fmt2d {

__global__ void eik_front(const DevField* fields, int nf, unsigned* n_pending);
__global__ void eik_select(const DevField* fields, int nf, int total_tiles, unsigned* queue,
                           unsigned* qlen);
__global__ void eik_visit(const DevField* fields, int nf, const unsigned* queue,
                          const unsigned* qlen, unsigned* qhead, int max_passes,
                          unsigned long long* counters);
__global__ void eik_final(const DevField* fields, int nf, float* const* gout,
                          uint8_t* const* susp, unsigned* n_bad);
size_t eik_round_smem();
__global__ void k_seed_masks(DevField* fields, int nf);

__global__ void k_fill(DevField* fields, int nf, size_t max_slots);
__global__ void k_init_source(DevField* fields, const DevRegionX* xs, const double* sx,
                              const double* sz, int nf, int nz);
__global__ void k_seed_iface(const SeedDesc* descs, int nd, int nz);
__global__ void k_fit_suspect(const DevField* fields, const DevRegionX* xs, float* const* gout,
                              uint8_t* const* susp, int nf);
__global__ void k_water_fix(const DevField* fields, float* const* gout, const int* upward, int nf);
__global__ void k_headwave(const DevField* fields, const DevRegionX* xs, float* const* gout,
                           const int* hw_slot, const double* hw_v, double dx_if, int nx,
                           double* scratch, const int* which, int nsel);
__global__ void k_export(const float* t2, const float* g2, const int* slot_of_node, int nnode,
                         double* T, double* gx, double* gz);

}  // namespace fmt2d
