// FMT2D CPU oracle: an FP64 C++ restatement of the reference's forward-and-
// sensitivity path (eikonal FMM, stage coupling, ray backtrace, Frechet rows,
// LSQR products).  TEST INFRASTRUCTURE ONLY: the product library never links
// or calls this code; tests, the smoke check and the CPU-baseline leg of the
// benchmark use it as the checker.
//
// Parity unpinned: the reference cannot be built here (no Fortran compiler)
// and has no golden vectors; analytic known answers and SciPy's LSQR pin it.
//
// Indexing mirrors the reference on purpose, because node and parameter
// numbering is a bit-exact contract: grid indices ix, iz and region node ids
// are 1-based, 0 means "no node".  Every routine names the reference routine
// (file:line) whose algorithm it restates.
#pragma once
#include <cstdint>
#include <vector>
#include <array>
#include <cmath>

namespace orc {

constexpr double kHugeTime = 1.0e20;              // mod_fmt2d.f90:616
constexpr double kTiny = 2.2250738585072014e-308; // Fortran tiny(1.0_dp)

// Propagation grid (type Tpropagation_grid2d, mod_fmt2d.f90:24-51).
struct Grid {
  int nx = 0, nz = 0;
  double dx = 0, dz = 0, x0 = 0, z0 = 0, tolerance = 0;
  std::vector<double> x, z;        // 1-based: x[1..nx], z[1..nz]
  std::vector<double> vel;         // P velocity, vel[g(ix,iz)]
  std::vector<int> node_region;    // last region that claimed the node
  std::vector<int> rnode_id;       // that region's node id
  std::vector<uint8_t> fully_regular;
  // ccind_from_2dc: per cell (ix,iz) an optional array indexed by interface
  // id (1..5).  cc_assoc marks "associated"; cc_idx holds the entries.
  std::vector<uint8_t> cc_assoc;
  std::vector<int> cc_idx;         // 6 ints per cell, [1..5] used
  int g(int ix, int iz) const { return (ix - 1) + (iz - 1) * nx; }
};

// Intersection of an interface with the grid (Tintersection2d, :193-220).
struct Isec {
  int id = 0, nnode = 0, n_ccells = 0;
  std::vector<double> x, z, nx_, nz_;          // 1-based node arrays, normal
  std::vector<double> vel_top, vel_bot;        // P velocity above / below
  std::vector<double> T, gx, gz;               // interface time + gradient
  bool has_T = false;
  std::vector<int> cc_ix, cc_iz, n_inodes;     // 1-based cut-cell arrays
  std::vector<int> inodes;                     // 4 per cut cell
  std::vector<int> ccell_from_inode;           // 4 per interface node
  std::vector<int> rright, rleft;              // region node ids (last define)
  bool has_rright = false, has_rleft = false;
  int regleft = 0, regright = 0;
  int inode(int k, int icell) const { return inodes[(icell - 1) * 4 + (k - 1)]; }
  int ccfi(int k, int n) const { return ccell_from_inode[(n - 1) * 4 + (k - 1)]; }
};

// Region (Tregion2d, :223-258).
struct Region {
  int id = 0, itop = 0, ibot = 0;
  int ngnode = 0, nnode = 0;
  std::vector<int> i1, i2, i3;       // 1-based per node
  std::vector<double> x, z, vel;     // 1-based per node
  std::vector<int> rid;              // region_rnode_id over the grid
  std::vector<int> itop_rid, ibot_rid;
  std::vector<int> status;
  std::vector<double> T, gx, gz;
};

// Time field (Ttime_field2d, :262-279).
struct TField {
  int reg = 0;
  int istart = 0;                   // intersection id the stage starts from
  std::vector<double> T, gx, gz;    // 1-based, size nnode+1
  bool solved = false;
};

// One ray section (Tray_section2d, :283-300).
struct RaySection {
  int reg = 0, tf = 0, istart = 0, iend = 0, place = 0;
  std::vector<double> px, pz;       // 0-based point list
  bool diffracted = false, headwave = false;
};

struct Ray {
  int raypath_id = 0, nsections = 0;
  std::vector<RaySection> sec;      // 1-based: sec[1..nsections]
  double receiver_time = 0, rgx = 0, rgz = 0;
  bool valid = true, headwave = false, diffracted = false;
  std::vector<int> pdev_indx;       // 1-based parameter indices
  std::vector<double> pdev;
};

// Phase (Tpath2d) restricted to what the hot path reads.
struct Path {
  int n_tf = 0;
  std::vector<int> sequence;        // 1-based
  std::vector<int> tf_sequence;     // 1-based
};

struct Model {
  Grid grid;
  Isec isec[6];                      // 1..5
  Region reg[7];                     // 1..6
  double vwater = 1.5;
  int nsurf_x = 0;                   // seafloor interface node count
  // inversion parameterisation (frechet2d.f90:28-100)
  std::vector<int> inv_idx;          // per grid node, 0 = inactive
  std::vector<uint8_t> active;
  int n_vel_parms = 0, n_inv_parms = 0;
  int iface_inv = 0;                 // interface inverted (0 = none)
  int iface_start = 0;               // its start_index
  Path path[6];                      // 1..5
  std::vector<double> vgx;           // velocity-grid x (smesh x), 1-based
};

// Per-source state: 12 time fields plus the coordinates.
struct Source {
  double x = 0, z = 0;
  TField tf[13];                     // 1..12
};

// Model build ---------------------------------------------------------------
void build_model(Model& m, int nx, int nz, double dx, const double* xpos,
                 const double* vel_pgrid, const double* iface_z /*5*nx*/,
                 double vwater, int iface_inv);
void resample_smesh(int nx, int nzs, const double* xpos, const double* topo,
                    const double* zrel, const double* vel /*nx*nzs, ix fastest*/,
                    double vwater, int* nz_out, std::vector<double>& vel_out,
                    double* zmax_out);

// FMM ------------------------------------------------------------------------
void propagate2d(Model& m, Region& r);
void fit_gradient_at_node2d(const Model& m, const Region& r, int cn,
                            double& dtdx, double& dtdz);

// Stage coupling ---------------------------------------------------------------
void initialize_region_from_source2d(Model& m, Region& r, double sx, double sz, double t0);
void transfer_times_to_intersection(Model& m, Isec& is, const TField& tf);
void reflect_gradient_at_interface(Model& m, Isec& is, const Region& target);
void sweep_region_from_interface2d(Model& m, Region& r, const Isec& is);
void run_forward_source(Model& m, Source& s, int phase_mask);

// Rays / Frechet -------------------------------------------------------------
double interpolate_interface2d(const Model& m, double px, const Isec& is);
void interface_normal2d(const Model& m, double px, const Isec& is, double& nx, double& nz, double& h);
void interpolate_time_gradient2d(const Model& m, const Region& r, const double* gx,
                                 const double* gz, double px, double pz, double& dtdx, double& dtdz);
double interpolate_arrivaltime2d(const Model& m, const Region& r, const double* T,
                                 double px, double pz);
void trace_ray_from_receiver2d(Model& m, Source& s, double rx, double rz, Ray& ray);
void find_optimal_entry(Model& m, Source& s, int itf, double rx, double rz,
                        double& ex, double& ez, double& wt);
void compute_frechet_for_ray2d(Model& m, Source& s, Ray& ray);

}  // namespace orc
