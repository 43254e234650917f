/* C interface of the FMT2D CPU oracle (an FP64 restatement of the reference
 * algorithm).  TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and
 * the CPU-baseline leg of bench.py as the checker; the product library never
 * links it.  All arrays are caller-owned.  Grid arrays are nx*nz with ix
 * fastest; region node arrays are 0-based copies of the reference's 1-based
 * node numbering (entry k holds node id k+1).
 *
 * Parity unpinned: the reference is Fortran and cannot be compiled here (no
 * Fortran compiler), and it ships no tests or golden vectors.  The restatement
 * is checked against closed-form traveltimes and against SciPy's LSQR instead
 * (tests/test_oracle_kat.py, tests/test_lsqr_oracle.py). */
#ifndef FMT2D_ORACLE_H
#define FMT2D_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Build the model like invert2d_main.f90:139-500: resample the smesh onto the
 * dz = dx propagation grid, build the 5 interfaces (sea surface, seafloor,
 * sediment base, Moho, bottom), their cut cells and the 6 regions.
 * vel is nx*nzs (ix fastest), sed_z and moho_z have nx entries on xpos.
 * iface_inv selects the inverted interface (4 = Moho, 0 = none). */
void* orc_create(int nx, int nzs, const double* xpos, const double* topo, const double* zrel,
                 const double* vel, double vwater, const double* sed_z, const double* moho_z,
                 int iface_inv);
void orc_destroy(void* h);
void orc_grid_info(void* h, int* nx, int* nz, double* dx, double* x0);
void orc_pgrid_velocity(void* h, double* out);
void orc_iface_z(void* h, int iface, double* out);
void orc_iface_vel(void* h, int iface, double* vel_top, double* vel_bot);
int orc_region_nnode(void* h, int reg, int* ngnode);
void orc_region_tables(void* h, int reg, int* i1, int* i2, int* i3, double* x, double* z,
                       double* vel, int* rid);
void orc_fully_regular(void* h, uint8_t* out);
void orc_cut_cells(void* h, int iface, int* ncc, int* cc_ix, int* cc_iz);
int orc_inv_idx(void* h, int* out, int* n_vel_parms);

/* Run the phase recipe of inversion2d.f90:4214-4476 for one source (placed on
 * the seafloor at sx) into source slot `slot`.  phase_mask bit p-1 enables
 * phase p (1 Pg, 2 PsedP, 3 PmP, 4 Pg_ss, 5 Pg_ss2). */
int orc_forward(void* h, int slot, double sx, int phase_mask);
double orc_source_z(void* h, int slot);
int orc_field(void* h, int slot, int tf, double* T, double* gx, double* gz);
/* Load a time field into a slot (e.g. a device field copied back) so rays can
 * be traced on it. */
int orc_set_field(void* h, int slot, int tf, const double* T, const double* gx, const double* gz);

/* One heap-FMM solve of region `reg` from the given status/T/gradient state
 * (status: -1 far, 0 accepted, 1 trial).  Arrays are updated in place. */
int orc_propagate(void* h, int reg, int* status, double* T, double* gx, double* gz);

/* One pick: receiver handling of invert2d_main.f90:517-537 and
 * inversion2d.f90:4488-4535 (entry search, backtrace, water time, Frechet).
 * Outputs: receiver time incl. water leg, valid flag, the row (1-based
 * parameter ids, ascending) and the ray points of all sections (x,z pairs). */
int orc_trace(void* h, int slot, int phase, double rx, double rz, double* t_out, int* valid,
              int* nnz, int* idx_out, double* val_out, int cap, int* npts, double* pts,
              int pts_cap, int* nsec);

/* LSQR (smooth_type 1) of inversion2d.f90:6578-7167 over a 1-based CSR. */
int orc_lsqr(void* h, int ndata, int nparm, const int* gindx, const double* gval,
             const int* row_ptr, const double* residual, const double* gtg_diag,
             const double* dm_sum, double eps_min, double wdv, double wdv_iface,
             double w_smooth, double w_smooth_iface, int max_iter, double* dm, int* iters,
             double* rnorm, double* test2);
void orc_spmv(int ndata, int nparm, const int* gindx, const double* gval, const int* row_ptr,
              int transpose, const double* x, double* y);
void orc_laplacian(void* h, int nparm, const double* vin, double* vout);
/* run_lsqr for smooth_type 1 (Laplacian), 2 (Gaussian R_h, R_v) or 3 (Laplacian
 * for velocity, Gaussian R_h for the interface), inversion2d.f90:6578-7167. */
int orc_lsqr_smooth(void* h, int smooth_type, int ndata, int nparm, const int* gindx,
                    const double* gval, const int* row_ptr, const double* residual,
                    const double* gtg_diag, const double* dm_sum, const double* mvscale,
                    double corr_x, double corr_z, double corr_x_iface, double eps_min,
                    double wdv, double wdv_iface, double w_smooth, double w_smooth_iface,
                    int max_iter, double* dm, int* iters, double* rnorm, double* test2);
/* run_lsqr (smooth_type 1) with the Laplacian on an explicit parameter grid
 * (inv_idx over gnz x gnx, ix fastest; iface_nx interface parameters after
 * the n_vel_parms velocity parameters). */
int orc_lsqr_geom(int gnx, int gnz, const int* inv_idx, int n_vel_parms, int iface_nx,
                  int ndata, int nparm, const int* gindx, const double* gval,
                  const int* row_ptr, const double* residual, const double* gtg_diag,
                  const double* dm_sum, double eps_min, double wdv, double wdv_iface,
                  double w_smooth, double w_smooth_iface, int max_iter, double* dm, int* iters,
                  double* rnorm, double* test2);
/* Gaussian smoothing matrices of build_gauss_smooth_matrix (which 0: R_h,
 * 1: R_v) and build_iface_gauss_smooth_matrix (which 2), inversion2d.f90:
 * 1252-1616, as 1-based CSR over the model's parameters; returns nnz. */
int orc_gauss_smooth(void* h, double corr_x, double corr_z, double corr_x_iface,
                     const double* mvscale, int which, int* rp, int* col, double* val, int cap);

#ifdef __cplusplus
}
#endif
#endif
