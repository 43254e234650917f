/* fmt2d_gpu.h — C ABI of the B200 implementation of FMT2D's forward-and-
 * sensitivity path.
 *
 * The reference keeps this path behind Fortran subroutine calls on derived
 * types with pointer components (not C-interoperable).  Each entry point below
 * replaces one of them for a caller that passes plain contiguous arrays (a
 * Fortran bind(C) interface module or Python ctypes):
 *
 *   fmt2d_upload_model   <- the model build of invert2d_main.f90:139-500
 *                           (read_smesh outputs + the two interface files);
 *                           builds find_intersection2d / define_region2d /
 *                           tag_regular_nodes2d / velocities_to_*2d state
 *                           (src/propagate2d.f90:1335-1979) on the device
 *   fmt2d_forward        <- the per-source stage loop of run_forward2d
 *                           (src/inversion2d.f90:4184-4476): initialize_region_
 *                           from_source2d, transfer_times_to_intersection,
 *                           reflect_gradient_at_interface, sweep_region_from_
 *                           interface2d and propagate2d (interface block
 *                           src/mod_fmt2d.f90:706-712) for every source
 *   fmt2d_get_field      <- reading tf%arrivaltime / tf%time_gradient
 *                           (src/mod_fmt2d.f90:262-279) in region node order
 *   fmt2d_set_frechet    <- the CSR that read_frechet_data2d builds
 *                           (src/inversion2d.f90:3965-4052) after the column
 *                           and row scaling of src/inversion2d.f90:371-379
 *   fmt2d_spmv           <- sparse_Ax / sparse_ATx (src/inversion2d.f90:2997-3042)
 *   fmt2d_gtg_diag       <- the gtg_diag loop of src/inversion2d.f90:466-475
 *   fmt2d_lsqr           <- run_lsqr (src/inversion2d.f90:6578-7167)
 *
 * Conventions: every function returns 0 on success and a negative FMT2D_ERR_*
 * code on failure (never exits the process); fmt2d_last_error() returns the
 * message of the last failure on that context.  Region node ids, phase ids
 * (1 Pg, 2 PsedP, 3 PmP, 4 Pg_ss, 5 Pg_ss2) and time-field ids (1..12) follow
 * the reference's numbering.  One context per host thread; calls on a context
 * are ordered on its CUDA stream.  All arrays are caller-owned host memory.
 */
#ifndef FMT2D_GPU_H
#define FMT2D_GPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FMT2D_API __attribute__((visibility("default")))
#else
#define FMT2D_API
#endif

#define FMT2D_OK 0
#define FMT2D_ERR_ARG (-1)      /* invalid argument */
#define FMT2D_ERR_CUDA (-2)     /* CUDA runtime failure or no device */
#define FMT2D_ERR_STATE (-3)    /* call out of order (e.g. no model uploaded) */
#define FMT2D_ERR_MODEL (-4)    /* model rejected by the geometry build */
#define FMT2D_ERR_CONVERGE (-5) /* eikonal solve did not reach its fixed point */

typedef struct fmt2d_ctx fmt2d_ctx;

/* Smesh-level model description (what read_smesh and read_refl return).
 * vel is nzs rows of nx values (row iz holds depth zrel[iz] below the
 * seafloor); sed_z and moho_z are interface depths at xpos.  Interface nodes
 * must sit on the propagation-grid columns (the reference's find_intersection2d
 * uses the interface index as the grid column). */
typedef struct fmt2d_model_desc {
  int nx;                 /* smesh / grid columns */
  int nzs;                /* smesh depth samples */
  const double* xpos;     /* [nx] km, uniform spacing = propagation dx = dz */
  const double* topo;     /* [nx] seafloor depth, km */
  const double* zrel;     /* [nzs] depth below the seafloor, km */
  const double* vel;      /* [nzs*nx] P velocity, km/s */
  double vwater;          /* water velocity, km/s */
  const double* sed_z;    /* [nx] sediment base depth (interface 3) */
  const double* moho_z;   /* [nx] Moho depth (interface 4) */
  int iface_inv;          /* inverted interface for Frechet rows (4 = Moho, 0 none) */
} fmt2d_model_desc;

/* Context on CUDA device `device` (owns device buffers and one stream).
 * device = -1 makes a host-only context: the model build and its tables work,
 * every call that needs the GPU returns FMT2D_ERR_STATE. */
FMT2D_API int fmt2d_ctx_create(fmt2d_ctx** out, int device);
FMT2D_API int fmt2d_ctx_destroy(fmt2d_ctx* ctx);
/* Message of the last failure on ctx (empty if none); writes at most len bytes. */
FMT2D_API int fmt2d_last_error(fmt2d_ctx* ctx, char* buf, int len);

FMT2D_API int fmt2d_upload_model(fmt2d_ctx* ctx, const fmt2d_model_desc* desc);
/* Grid size after the dz = dx resampling (invert2d_main.f90:242-246). */
FMT2D_API int fmt2d_model_info(fmt2d_ctx* ctx, int* nx, int* nz, double* dx, double* x0);
/* The propagation-grid velocity vel[nz*nx] (ix fastest) of the current model:
 * the velocity grid the inversion updates (vgrid%velocity, inverted on the
 * propagation grid itself). */
FMT2D_API int fmt2d_model_velocity(fmt2d_ctx* ctx, double* vel);
/* Depths z[nx] of interface k (1 sea surface, 2 seafloor, 3 sediment base,
 * 4 Moho, 5 model bottom), node ix on grid column ix (intrface(k)%z_nodes). */
FMT2D_API int fmt2d_model_interface(fmt2d_ctx* ctx, int k, double* z);
/* A model step of the inversion: what apply_model_step leaves
 * (src/inversion2d.f90:7173-7237) followed by rebuild_geometry2d
 * (:3661-3816).  vel[nz*nx] is the new propagation-grid velocity (NULL keeps
 * it), iface_z[nx] the new depths of the inverted interface (NULL keeps
 * them).  The geometry is rebuilt on the host and uploaded; field stores stay
 * allocated, every field is unsolved until the next forward.  The inversion
 * numbering must not change (FMT2D_ERR_MODEL otherwise, the model unchanged). */
FMT2D_API int fmt2d_update_model(fmt2d_ctx* ctx, const double* vel, const double* iface_z);
/* Region r (1..6): node count and, when arrays are given, the reference's node
 * table (i1 = grid column 1-based or 0 for interface nodes, i2 = grid row
 * 1-based or interface id, i3 = interface node index 1-based or 0). */
FMT2D_API int fmt2d_region_nodes(fmt2d_ctx* ctx, int region, int* nnode, int* i1, int* i2, int* i3);
/* Region r (1..6): node positions and P velocity in the reference's node order
 * (Tregion2d%x, %z, %velocity of propagate2d.f90:1564-1647, FP64); any array
 * may be NULL.  These are the exact doubles the device stencil computes with. */
FMT2D_API int fmt2d_region_geometry(fmt2d_ctx* ctx, int region, double* x, double* z, double* vel);
/* Inversion parameter numbering (frechet2d.f90:55-63): inv_idx[nx*nz] with ix
 * fastest, 1-based ids, 0 inactive; returns counts. */
FMT2D_API int fmt2d_inv_index(fmt2d_ctx* ctx, int* inv_idx, int* n_vel_parms, int* n_inv_parms);

/* A coarse inversion grid over the model's parameters (no reference
 * counterpart: the reference inverts on the propagation grid itself, which
 * is kx = kz = ki = 1 and gives P = I).  Coarse velocity nodes every kx grid
 * columns and kz grid rows, coarse interface nodes every ki interface nodes;
 * each fine velocity parameter is the bilinear interpolation of its coarse
 * cell's corners, each fine interface parameter the linear interpolation of
 * its two coarse interface nodes.  Returns the coarse grid size (*nxc, *nzc),
 * *nvp_c coarse velocity parameters (the coarse nodes some fine parameter
 * uses, numbered iz outer / ix inner in coarse_idx[nzc*nxc], 0 unused),
 * *npar_c with the coarse interface parameters after them, and P as 1-based
 * CSR: p_row_ptr[n_inv_parms + 1], p_col / p_val[*p_nnz].  Any array may be
 * NULL (sizes first).  Host-side: works on a host-only context. */
FMT2D_API int fmt2d_projection(fmt2d_ctx* ctx, int kx, int kz, int ki, int* nxc, int* nzc,
                               int* nvp_c, int* npar_c, int* coarse_idx, int* p_row_ptr,
                               int* p_col, double* p_val, long long* p_nnz);
/* Rows of G P for a 1-based CSR G over nfine fine parameters and P from
 * fmt2d_projection: coarse columns ascending, equal columns summed in the
 * order of the fine entries.  Outputs may be NULL to get *nnz first.  Host
 * only, no context. */
FMT2D_API int fmt2d_project_rows(int ndata, const int* row_ptr, const int* gindx,
                                 const double* gval, int nfine, const int* p_row_ptr,
                                 const int* p_col, const double* p_val, int* row_ptr_out,
                                 int* gindx_out, double* gval_out, long long* nnz);

/* The data of one LSQR solve from a batch of traced picks: the selection of
 * read_frechet_data2d (src/inversion2d.f90:3965-4052) with the weighting of
 * lsqr_inversion2d (:334-379).  Keeps, in pick order, the picks that are
 * valid, have obs >= 0 and |obs - t_calc| <= crit_chi; data_wt is wt_psed for
 * phase 2, wt_pmp for 3, wt_pgss for 4 and 5, else 1; residual = (obs -
 * t_calc) * data_wt; the kept rows' values become gval * mvscale[j-1] *
 * data_wt (columns 1..nparm; mvscale[nparm]).  Input rows: 1-based CSR over
 * all npick picks, as fmt2d_frechet_rows returns them.  Outputs (sized for
 * every pick kept): *ndata, row_ptr_out[ndata+1] (1-based), gindx_out and
 * gval_out[nnz], residual, data_wt and pick_of_row (0-based) [ndata].  Host
 * only, no context: it replaces Fortran array work, not a device routine. */
FMT2D_API int fmt2d_select_data(int npick, const int* phase, const double* obs,
                                const double* t_calc, const int* valid, const int* row_ptr,
                                const int* gindx, const double* gval, int nparm,
                                const double* mvscale, double crit_chi, double wt_psed,
                                double wt_pmp, double wt_pgss, int* ndata, int* row_ptr_out,
                                int* gindx_out, double* gval_out, double* residual,
                                double* data_wt, int* pick_of_row);

/* Readers of the reference's input files (read_tomo2d.f90), with Fortran
 * list-directed input rules (each READ starts a new line and may continue
 * over lines; blanks or commas between values; D exponents; r*v repeats).
 * Host only, no context; on error the message is in fmt2d_io_last_error.
 * Call with NULL arrays first to get the sizes.
 *
 * read_smesh (:8-81): header nx nz vwater vair, then xpos[nx], topo[nx],
 * zpos_rel[nz], then one record of nz velocities per ix; vel is returned
 * ix fastest (vel[iz*nx + ix]), the layout of fmt2d_model_desc. */
FMT2D_API int fmt2d_read_smesh(const char* path, int* nx, int* nz, double* vwater, double* vair,
                               double* xpos, double* topo, double* zrel, double* vel);
/* read_refl (:83-139): one "x z" pair per line, blank and malformed lines
 * skipped. */
FMT2D_API int fmt2d_read_refl(const char* path, int* n, double* x, double* z);
/* read_geom (:141-248): nobs, then per OBS "tag x z nrec" and nrec lines
 * "tag x z phase t_obs uncertainty"; obs_id is 1-based. */
FMT2D_API int fmt2d_read_geom(const char* path, int* nobs, int* nrec, double* obs_x,
                              double* obs_z, double* rec_x, double* rec_z, int* obs_id,
                              int* phase, double* t_obs, double* unc);
FMT2D_API int fmt2d_io_last_error(char* buf, int len);

/* Gaussian smoothing matrix of run_lsqr's smooth_type 2/3 layouts, built on
 * the host (works on a host-only context): which 0 = R_h and 1 = R_v over the
 * velocity parameters (build_gauss_smooth_matrix, src/inversion2d.f90:
 * 1252-1402), 2 = R_h over the inverted interface's parameters
 * (build_iface_gauss_smooth_matrix, :1524-1616); correlation lengths in km,
 * mvscale[n_inv_parms] folded into the values as the reference does.  1-based
 * CSR over all n_inv_parms rows, rows the matrix does not cover empty:
 * row_ptr[n_inv_parms + 1], col[nnz], val[nnz]; call with col = val = NULL
 * to get *nnz first. */
FMT2D_API int fmt2d_gauss_smooth(fmt2d_ctx* ctx, int which, double corr_x, double corr_z,
                                 double corr_x_iface, const double* mvscale, int* row_ptr,
                                 int* col, double* val, long long* nnz);

/* Solve every time field of the enabled phases (bit p-1 of phase_mask enables
 * phase p) for nsrc OBS sources placed on the seafloor below src_x[s]. */
FMT2D_API int fmt2d_forward(fmt2d_ctx* ctx, const double* src_x, int nsrc, int phase_mask);
/* fmt2d_forward of n contexts at once (one model each, of any grid size):
 * context i solves nsrc[i] sources at src_x[i] for phase_mask[i].  The
 * contexts' stage chains run concurrently on their own streams, so the
 * fields of many small or uneven models fill the device together instead of
 * one model after another (the reference runs run_forward2d once per model,
 * src/inversion2d.f90:4145-4545).  The contexts must be distinct and on one
 * device or several; status[i] (may be NULL) receives each forward's code,
 * the return value is the first failure (its context holds the message). */
FMT2D_API int fmt2d_forward_batch(fmt2d_ctx* const* ctxs, int n, const double* const* src_x,
                                  const int* nsrc, const int* phase_mask, int* status);
/* Time field tf (1..12) of source s in its region's node order, FP64; any of
 * T, dtdx, dtdz may be NULL.  Unreached nodes hold 1e20. */
FMT2D_API int fmt2d_get_field(fmt2d_ctx* ctx, int src, int tf, double* T, double* dtdx, double* dtdz);
/* fmt2d_get_field into DEVICE memory of the caller (T, dtdx, dtdz: nnode
 * doubles each on the context's device, any may be NULL); complete when the
 * call returns.  No reference counterpart (the reference's fields are host
 * arrays); the PyTorch operators use it to return CUDA tensors. */
FMT2D_API int fmt2d_get_field_device(fmt2d_ctx* ctx, int src, int tf, double* T, double* dtdx,
                                     double* dtdz);
/* Counters of the last fmt2d_forward (and of the exports since), in this
 * order: [0] steps of the longest field solve, summed over stage levels,
 * [1] stage levels, [2] solve passes (each ends in a fixed-point check of
 * every node), [3] deferred nodes passed over without evaluation, [4] device
 * milliseconds of the solves and checks, [5] kernel launches, [6] region nodes
 * of the solved time fields, [7] node evaluations, [8] steps summed over all
 * fields, [9] fields that reached the step cap, [10] node writes that changed
 * a node, [11] nodes the last fixed-point check found still moving (nonzero
 * only when fmt2d_forward returned FMT2D_ERR_CONVERGE), [12..16] SM cycles of
 * the solve's phases summed over fields (evaluate, arbitrate and commit, the
 * evaluate phases of steps with a node next to an interface, spread, window
 * release), [17] evaluations of nodes next to an interface, [18] steps that
 * evaluated one.
 * Writes min(n, FMT2D_N_STATS) values.  No reference counterpart (diagnostics). */
#define FMT2D_N_STATS 19
FMT2D_API int fmt2d_stats(fmt2d_ctx* ctx, double* values, int n);

/* Ray backtrace and Frechet rows of npick picks on the fields of the last
 * fmt2d_forward: per pick the source index src[i] (0-based, into that call's
 * sources), the phase (1..5) and the receiver (shot) position rx, rz.  This
 * is the per-pick work of run_forward2d (src/inversion2d.f90:4488-4535): the
 * in-water receiver handling of invert2d_main.f90:517-537 with
 * find_optimal_entry_inv (src/inversion2d.f90:6344-6438) and the water-leg
 * time, trace_ray_from_receiver2d (src/rays2d.f90:7-153) and
 * compute_frechet_for_ray2d (src/inversion2d.f90:4548-4787).  Outputs:
 * t_calc[npick] (receiver time incl. the water leg), valid[npick] (1 valid
 * ray), and *nnz, the number of Frechet entries of all valid picks, which
 * stay on the device for fmt2d_frechet_rows. */
FMT2D_API int fmt2d_trace(fmt2d_ctx* ctx, const int* src, const int* phase, const double* rx,
                          const double* rz, int npick, double* t_calc, int* valid,
                          long long* nnz);

/* fmt2d_trace without the Frechet rows: t_calc and valid only (the line
 * search's compute_rms_after_forward, src/inversion2d.f90:3298-3339, needs no
 * sensitivities).  fmt2d_frechet_rows then reports FMT2D_ERR_STATE. */
FMT2D_API int fmt2d_trace_times(fmt2d_ctx* ctx, const int* src, const int* phase,
                                const double* rx, const double* rz, int npick, double* t_calc,
                                int* valid);

/* Misfit and its gradient by the discrete adjoint of the time fields (no
 * counterpart in the reference, whose inversion uses the ray-based Frechet
 * rows G of fmt2d_trace; the gradient is the exact derivative of the
 * reference's discrete forward, where G^T r is the ray-theory one).  On the
 * fields of the last fmt2d_forward, for npick picks as in fmt2d_trace
 * (phases 1-5) with observed times t_obs (< 0: no pick) and sigma > 0:
 *   *misfit = 0.5 * sum over valid picks of ((t_calc - t_obs) / sigma)^2
 * and, when grad_slow / grad_vel are not NULL, its derivative with respect to
 * the propagation-grid slowness / velocity (nz*nx, ix fastest, the layout of
 * fmt2d_model_velocity); when grad_iface is not NULL, with respect to the
 * node depths of interfaces 1..5 (5*nx, interface i's node ix at
 * (i-1)*nx + ix; the depth moves the interface nodes of the cut cells, the
 * velocities sampled off the interface and the stage hand-off distances,
 * while region membership and cut cells are held).  t_calc and valid are
 * filled as fmt2d_trace fills them (the call traces the picks for their
 * times, without Frechet rows).  info (may be NULL) receives FMT2D_ADJ_N_INFO values: node values the
 * adjoint could not re-derive, links outside their node's reader list, nodes
 * its reverse sweep did not reach (all three 0 on success), the sweep's most
 * rounds, fields, reached nodes, ms. */
#define FMT2D_ADJ_N_INFO 8
FMT2D_API int fmt2d_misfit_gradient(fmt2d_ctx* ctx, const int* src, const int* phase,
                                    const double* rx, const double* rz, const double* t_obs,
                                    const double* sigma, int npick, double* misfit,
                                    double* t_calc, int* valid, double* grad_slow,
                                    double* grad_vel, double* grad_iface, double* info);
/* Per pick of the last fmt2d_trace (npick values each, any may be NULL): the
 * water leg's time (ray%water_time, 0 for a receiver below the seafloor or a
 * Pg_ss / Pg_ss2 pick) and the ray's receiver end (the seafloor entry point
 * find_optimal_entry_inv chose, src/inversion2d.f90:6344-6438, else the
 * receiver): what write_arrivals2d and entry_points.dat report
 * (fmt2d_main.f90:1655-1719). */
FMT2D_API int fmt2d_trace_entries(fmt2d_ctx* ctx, double* water_time, double* entry_x,
                                  double* entry_z);
/* The Frechet rows of the last fmt2d_trace as CSR over all its picks (an
 * invalid pick's row is empty): row_ptr[npick+1], gindx[nnz] parameter ids in
 * ascending order (the inversion numbering of fmt2d_inv_index, interface
 * parameters after the velocity ones), gval[nnz] = dt/d(slowness) for
 * velocity parameters and the interface-depth derivative otherwise.
 * index_base 1 gives the reference's 1-based row_ptr and gindx. */
FMT2D_API int fmt2d_frechet_rows(fmt2d_ctx* ctx, int* row_ptr, int* gindx, double* gval,
                                 int index_base);

/* Sensitivity matrix G (ndata picks x nparm parameters) as CSR host arrays,
 * index_base 1 for the reference's 1-based gindx / row_ptr (row_ptr has
 * ndata+1 entries).  Columns outside 1..nparm are kept but skipped by every
 * product, like sparse_Ax / sparse_ATx.  The context keeps G on the device as
 * CSR and as CSC (columns in ascending row order) until the next call. */
FMT2D_API int fmt2d_set_frechet(fmt2d_ctx* ctx, int ndata, int nparm, const int* row_ptr,
                                const int* gindx, const double* gval, int index_base);
/* y = G x (transpose 0: x[nparm] -> y[ndata]) or y = G^T x (transpose 1). */
FMT2D_API int fmt2d_spmv(fmt2d_ctx* ctx, int transpose, const double* x, double* y);
/* gtg[j] = sum over rows of G(i,j)^2, j = 1..nparm. */
FMT2D_API int fmt2d_gtg_diag(fmt2d_ctx* ctx, double* gtg);

/* run_lsqr's arguments that are not arrays (src/inversion2d.f90:6578-6598).
 * smooth_type selects the augmented system (:507-511): 1 [G; w_s L; w_d I]
 * with the Laplacian over the model's inversion numbering; 2 [G; w_s R_h;
 * w_s R_v; w_d I] with the interface Gaussian w_si R_i in the R_h block's
 * interface rows; 3 [G; w_s L (velocity rows) + w_si R_i (interface rows);
 * w_d I].  2 and 3 need fmt2d_set_smoothing first.  max_iter is the
 * reference's min(lsqr_max_iter, 2000), >= 1. */
typedef struct fmt2d_lsqr_params {
  int smooth_type;
  int max_iter;
  double wdv, wdv_iface;            /* damping weights (velocity, interface) */
  double w_smooth, w_smooth_iface;  /* smoothing weights */
  double eps_min;                   /* velocity columns with gtg < 0.01 eps_min are masked */
} fmt2d_lsqr_params;

/* The Gaussian smoothing operators of smooth_type 2 and 3:
 * build_gauss_smooth_matrix (R_h along grid rows within 3 corr_x, R_v along
 * grid columns within 3 corr_z) and build_iface_gauss_smooth_matrix (R_i along
 * the inverted interface within 3 corr_x_iface), src/inversion2d.f90:1252-1616,
 * with the column scaling mvscale[nparm] folded in as the reference does.
 * Built on the host, kept on the device (R_h and R_v also transposed) for the
 * following fmt2d_lsqr calls until the next model upload.  R_h is built when
 * corr_x > 0, R_v when corr_z > 0, R_i when corr_x_iface > 0 and an interface
 * is inverted.  R_i is applied as its own adjoint, as the reference does
 * (:6826-6833), which is its transpose when the interface columns share one
 * scaling. */
FMT2D_API int fmt2d_set_smoothing(fmt2d_ctx* ctx, double corr_x, double corr_z,
                                  double corr_x_iface, const double* mvscale);

/* The parameter grid the LSQR's Laplacian smooths over, for inverting on a
 * coarse grid (no reference counterpart: the reference inverts on the
 * propagation grid): coarse_idx[nzc*nxc] (ix fastest) holds 1-based velocity
 * parameter ids (0: none), n_vel_parms of them, followed by iface_nodes
 * interface parameters, as fmt2d_projection returns them; G is then G P
 * (fmt2d_project_rows) with n_vel_parms + iface_nodes columns.  coarse_idx
 * NULL returns to the model's own numbering (also the state after every model
 * upload or update).  smooth_type 1 only. */
FMT2D_API int fmt2d_set_param_grid(fmt2d_ctx* ctx, int nxc, int nzc, const int* coarse_idx,
                                   int n_vel_parms, int iface_nodes);

/* LSQR on the current G: residual[ndata], gtg_diag[nparm] (NULL: computed
 * from G), dm_sum[nparm] (NULL: zeros) -> dm[nparm] and the reference's
 * lsqr_iter_out, rnorm_out, bnorm_out, test2_out (any may be NULL).  Needs an
 * uploaded model whose n_inv_parms equals nparm. */
FMT2D_API int fmt2d_lsqr(fmt2d_ctx* ctx, const fmt2d_lsqr_params* params, const double* residual,
                         const double* gtg_diag, const double* dm_sum, double* dm, int* iters,
                         double* rnorm, double* bnorm, double* test2);
/* fmt2d_lsqr without any device allocation.  No counterpart in the reference
 * (which allocates its LSQR work arrays per call).  For callers that cannot
 * call cudaMalloc while they solve: a driver that overlaps this solve with
 * work on other streams (cudaMalloc / cudaFree can synchronise the whole
 * device), or a program whose device memory is reserved up front by its own
 * pool allocator, where a new cudaMalloc fails or fragments that reserve.
 * residual[ndata], gtg_diag[nparm] (NULL: computed), dm_sum[nparm] (NULL:
 * zeros) and dm[nparm] are DEVICE pointers owned by the caller; G is the one
 * set by fmt2d_set_frechet.  The work vectors live in one fixed 32 MiB device
 * array that every GPU loading the library holds until exit; problems that
 * need more (about ndata + 6.125 nparm doubles) are rejected with
 * FMT2D_ERR_ARG.  The first call in a device's CUDA context looks up that
 * array's address, so make it before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race.
 * Ordering: the call runs on the context's own stream (fmt2d_stream), which
 * is not ordered after the streams the caller wrote residual, gtg_diag and
 * dm_sum on; make those writes complete first (synchronise, or make the
 * stream fmt2d_stream returns wait on an event recorded after them).  dm and
 * the scalars are final when the call returns. */
FMT2D_API int fmt2d_lsqr_noalloc(fmt2d_ctx* ctx, const fmt2d_lsqr_params* params,
                                 const double* residual, const double* gtg_diag,
                                 const double* dm_sum, double* dm, int* iters, double* rnorm,
                                 double* bnorm, double* test2);
/* Device milliseconds and kernel launches of the last fmt2d_lsqr (diagnostics,
 * no reference counterpart). */
FMT2D_API int fmt2d_lsqr_stats(fmt2d_ctx* ctx, double* ms, int* launches);

/* Schedule of the eikonal solve (no reference counterpart; the reference's
 * heap has no schedule): the time window's step in cells at the region's
 * largest velocity for every stage (0 < window_cells <= 1e6), or 0, the
 * default: no window for a stage that starts from the point source and 32
 * cells for a stage seeded along an interface (whose seeds span the whole
 * line at once), the number of solve passes, each followed by a fixed-point check
 * of every node (1..64, default 6), and the most steps one field's solve may
 * take (0: the default, 4,000,000).  A forward whose last check still finds
 * nodes that move, or in which a field reached the step cap, returns
 * FMT2D_ERR_CONVERGE.  A window holds back every new time beyond it until
 * the times below it have settled (nodes settle in time slices); without one
 * a step commits, among nodes that read each other, the smallest new time
 * first, which already orders dependent nodes as the heap does.  Both
 * schedules reproduce the heap's times in the parity tests; the window
 * takes more steps. */
FMT2D_API int fmt2d_set_schedule(fmt2d_ctx* ctx, double window_cells, int max_passes,
                                 long long max_steps);
/* The window of stages seeded along an interface when fmt2d_set_schedule's
 * window_cells is 0 (default 32 cells at the region's largest velocity; 0: no
 * window).  The results do not depend on it in the parity tests; the number
 * of solver steps does. */
FMT2D_API int fmt2d_set_iface_window(fmt2d_ctx* ctx, double cells);

/* Threads of each field's solve block: 256, 384 or 512 (0: the default,
 * 384).  Results are the same bit for bit for every size (no evaluation of a
 * solve step sees a value written in that step); only the time differs: larger
 * blocks suit longer fronts (larger grids).  No reference counterpart. */
FMT2D_API int fmt2d_set_solve_threads(fmt2d_ctx* ctx, int threads);
/* Autotuner of the solve block size for a workload: one forward of nsrc
 * sources for phase_mask, then one forward timed per block size; the fastest
 * is kept for the context's later forwards and returned in *threads (may be
 * NULL), the times in ms[0..2] (256, 384, 512; may be NULL).  The fields of
 * the last forward stay valid.  No reference counterpart. */
FMT2D_API int fmt2d_autotune(fmt2d_ctx* ctx, const double* src_x, int nsrc, int phase_mask,
                             int* threads, double* ms);

/* The CUDA stream (cudaStream_t) all work of the context is issued on, for
 * callers that record events around fmt2d_forward.  No reference counterpart. */
FMT2D_API int fmt2d_stream(fmt2d_ctx* ctx, void** stream);

#ifdef __cplusplus
}
#endif
#endif /* FMT2D_GPU_H */
