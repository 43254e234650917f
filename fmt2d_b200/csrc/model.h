// Host-side model geometry for the device solver.
//
// The propagation grid, the five interfaces and the six regions follow the
// reference's model build (propagate2d.f90:1335-1979, invert2d_main.f90:139-
// 500) so that region node numbering, cut cells and the fully-regular mask
// are bit-exact.  The device layout is this library's own: every region is a
// dense row band of the grid ("bbox") padded to a pitch, followed by two rows
// holding the region's top and bottom interface nodes.  A "slot" indexes that
// layout; all per-node device arrays of a region are slot-indexed.
#pragma once
#include <cstdint>
#include <vector>
#include <string>

namespace fmt2d {

constexpr double kHugeTime = 1.0e20;
constexpr int kTileW = 32;   // tile width (columns) of the eikonal sweeps
constexpr int kTileH = 32;   // tile height (rows)

// Per-slot static code (uint32):
//   bit 0      node belongs to the region
//   bit 1      updatable (interface nodes in an unregistered cut cell are not)
//   bit 2      fully regular (4 regular quadrants)
//   bit 3      interface node (slot in one of the two interface rows)
//   bits 4-7   cell exists, cells c=0..3 = (ix,iz),(ix,iz-1),(ix-1,iz),(ix-1,iz-1)
//   bits 8-11  cell is cut by the region's own top/bottom interface
//   bits 12-15 that cut cell carries a top-interface inode
//   bits 16-19 that cut cell carries a bottom-interface inode
//   bits 20-23 cell is cut by any interface (used by the gradient fit)
// Interface slots: bits 8 (own cut cell irregular), 12/16 (top/bottom inodes
// present in that cell), 20 (cell registered); the cell's top row is in
// Region::izc_top/izc_bot.
enum : uint32_t {
  kInRegion = 1u << 0,
  kUpdatable = 1u << 1,
  kFullyRegular = 1u << 2,
  kIfaceNode = 1u << 3,
};
inline uint32_t cell_exists_bit(int c) { return 1u << (4 + c); }
inline uint32_t cell_irr_bit(int c) { return 1u << (8 + c); }
inline uint32_t cell_top_bit(int c) { return 1u << (12 + c); }
inline uint32_t cell_bot_bit(int c) { return 1u << (16 + c); }
inline uint32_t cell_any_bit(int c) { return 1u << (20 + c); }

struct Interface {
  std::vector<double> z;          // node depth (node ix sits on grid column ix)
  std::vector<double> nrm_x, nrm_z;
  std::vector<double> vel_top, vel_bot;
  std::vector<int> izc;           // cut cell row (0-based), -1 if none
  std::vector<uint8_t> inode_ok;  // node lies inside its cut cell's rows
};

struct Region {
  int id = 0, itop = 0, ibot = 0;           // 1-based interface ids
  int ngnode = 0, nnode = 0;
  int z_lo = 0, z_hi = -1, H = 0, pitch = 0; // bbox rows (0-based), slot pitch
  int tiles_x = 0, tiles_y = 0;
  std::vector<int> r0, r1;                   // per column first/last row (r1<r0 empty)
  std::vector<int> col_base;                 // node id of the column's first node - 1
  std::vector<uint32_t> code;                // per slot
  std::vector<float> vel;                    // per slot
  std::vector<double> vel64;                 // per slot, FP64 (coupling arithmetic)
  std::vector<float> iface_dz;               // per interface slot (2*pitch): z - z(izc)
  std::vector<int> izc_top, izc_bot;         // cut-cell rows of the two interfaces
  std::vector<int> slot_of_node;             // region node id (0-based) -> slot
  size_t nslots() const { return (size_t)(H + 2) * pitch; }
  int slot_grid(int ix, int iz) const { return (iz - z_lo) * pitch + ix; }
  int slot_top(int ix) const { return H * pitch + ix; }
  int slot_bot(int ix) const { return (H + 1) * pitch + ix; }
};

struct Model {
  int nx = 0, nz = 0;
  double dx = 0, x0 = 0, tolerance = 0, vwater = 1.5;
  std::vector<double> xpos;                 // smesh node x (for the velocity grid)
  std::vector<double> vel;                  // pgrid velocity, ix fastest
  std::vector<uint8_t> cell_cut;            // per cell: bit k = interface k cuts it
  std::vector<int> node_region, rnode_id;   // last region claiming a grid node
  std::vector<uint8_t> fully_regular;
  Interface ifc[6];                         // 1..5
  Region reg[7];                            // 1..6
  // interface node id tables as left by the reference's region definitions
  std::vector<int> rright[6], rleft[6];
  // inversion numbering (iz outer, ix inner over nodes at or below the seafloor)
  std::vector<int> inv_idx;
  int n_vel_parms = 0, n_inv_parms = 0, iface_inv = 0;
  double zbot = 0;                          // depth of the bottom interface (5)
  size_t g(int ix, int iz) const { return (size_t)iz * nx + ix; }
};

// Builds the model from smesh-level inputs (read_smesh outputs plus the two
// interface files), resampling like invert2d_main.f90:279-340.
// Returns an empty string on success or an error message.
std::string build_model(Model& m, int nx, int nzs, const double* xpos, const double* topo,
                        const double* zrel, const double* vel, double vwater,
                        const double* sed_z, const double* moho_z, int iface_inv);

// The geometry (interfaces, regions, codes, inversion numbering) from m.vel
// and the seafloor, sediment-base and Moho depths.
void build_geometry(Model& m, const double* topo, const double* sed_z, const double* moho_z);

// A model step (apply_model_step, src/inversion2d.f90:7173-7237, then
// rebuild_geometry2d, :3661-3816): the propagation-grid velocity (nz x nx,
// ix fastest; NULL keeps it) and the depths of the inverted interface's nodes
// (NULL keeps them); the geometry is rebuilt.  Returns an error message or "".
std::string update_model(Model& m, const double* vel, const double* iface_z);

// Region `reg`'s slot velocities as a linear map of the propagation-grid
// velocity m.vel: interior grid slots take their node's value, slots next to
// the region's interfaces and the interface slots take the bilinear samples
// one grid step off the interface (vel_top / vel_bot).  Node-major CSR over
// the nx*nz grid nodes (rp), entries (slot, weight) in ascending slot order.
// Checks that the map reproduces every slot's velocity bit for bit; returns
// an error message or "".  With zrp set, also the slots whose velocity is a
// sample off one of the region's interfaces, column-major CSR over the nx
// interface nodes (zrp): slot, side (0 top, 1 bottom interface) and the
// sample's derivative with respect to that interface node's depth.
std::string slot_velocity_map(const Model& m, int reg, std::vector<int>& rp,
                              std::vector<int>& slot, std::vector<double>& w,
                              std::vector<int>* zrp = nullptr, std::vector<int>* zslot = nullptr,
                              std::vector<int>* zside = nullptr,
                              std::vector<double>* zdv = nullptr);

// Gaussian smoothing matrix of the smooth_type 2/3 LSQR layouts as 1-based
// CSR over all n_inv_parms rows (rows it does not cover stay empty), mvscale
// folded into the values: which 0 = R_h, 1 = R_v over the velocity
// parameters (build_gauss_smooth_matrix, src/inversion2d.f90:1252-1402),
// 2 = R_h over the inverted interface (build_iface_gauss_smooth_matrix,
// :1524-1616).  Returns an error message or "".
// Projection P from a coarse inversion grid onto the model's parameters
// (fine velocity parameters = bilinear interpolation of coarse nodes every kx
// columns and kz rows; fine interface parameters = linear interpolation of
// coarse interface nodes every ki nodes).  P is a 1-based CSR with one row per
// fine parameter; coarse velocity parameters are the coarse nodes some fine
// parameter uses, numbered iz outer / ix inner (coarse_idx over nzc x nxc,
// 0 unused), coarse interface parameters follow.  kx = kz = ki = 1 gives
// P = I.
std::string projection(const Model& m, int kx, int kz, int ki, std::vector<int>& coarse_idx,
                       int& nxc, int& nzc, int& nvp_c, int& npar_c, std::vector<int>& rp,
                       std::vector<int>& col, std::vector<double>& val);
// Rows of G P: each row's fine entries mapped through P, coarse columns
// ascending (1-based CSR in and out; columns outside 1..nfine ignored).
void project_rows(int ndata, const int* row_ptr, const int* gindx, const double* gval,
                  int nfine, const int* prp, const int* pcol, const double* pval,
                  std::vector<int>& rp, std::vector<int>& col, std::vector<double>& val);

// read_frechet_data2d's selection with lsqr_inversion2d's weighting
// (src/inversion2d.f90:3965-4052, :334-379); see fmt2d_select_data.
// phase_wt = {PsedP, PmP, Pg_ss and Pg_ss2}.  Returns ndata.
int select_data(int npick, const int* phase, const double* obs, const double* t_calc,
                const int* valid, const int* row_ptr, const int* gindx, const double* gval,
                int nparm, const double* mvscale, double crit_chi, const double* phase_wt,
                int* row_ptr_out, int* gindx_out, double* gval_out, double* residual,
                double* data_wt, int* pick_of_row);

std::string gauss_smooth_csr(const Model& m, int which, double corr_x, double corr_z,
                             double corr_x_iface, const double* mvscale, std::vector<int>& rp,
                             std::vector<int>& col, std::vector<double>& val);

}  // namespace fmt2d
