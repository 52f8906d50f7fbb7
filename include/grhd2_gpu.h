/*
 * grhd2_gpu.h -- C-ABI of the B200 replacement for GRHD2's per-stage RHS and update path.
 *
 * The Fortran driver (grhd2.f90) keeps its .par parser, I/O and diagnostics and calls
 * these entry points through ISO_C_BINDING in place of the module procedures named in
 * each comment (file:line in RuelasF/GRHD).  All arguments are plain C types; every array
 * is in the reference's own Fortran layout (column-major, neq=5 fastest), so the Fortran
 * side passes c_loc() of its module arrays unchanged.
 *
 * Ownership: the caller owns host arrays; the library copies in and out.  The library owns
 * all device memory and one CUDA stream per handle.  State stays resident on the device
 * between calls; download() is only needed before output, checkpoints and diagnostics.
 *
 * Errors: every int-returning entry point returns 0 on success and a negative code on
 * failure; grhd2_gpu_last_error() gives the message.  The Fortran shim turns a nonzero
 * status into "write(*,*) msg; error stop 1", the reference's own convention
 * (evolution.f90:214-215, parameters.f90:1085-1096).
 *
 * Threading: one handle is used by one host thread at a time; handles are independent.
 */
#ifndef GRHD2_GPU_H
#define GRHD2_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRHD2_GPU_ABI_VERSION 1

/* error codes */
#define GRHD2_OK 0
#define GRHD2_ERR_ARG -1      /* invalid argument or configuration */
#define GRHD2_ERR_CUDA -2     /* CUDA runtime error (no device, launch failure, ...) */
#define GRHD2_ERR_NOMEM -3    /* device allocation failed */
#define GRHD2_ERR_STATE -4    /* call out of order (e.g. step before set_metric) */
#define GRHD2_ERR_CFL -5      /* non-finite metric or spacing in the CFL (evolution.f90:257-272) */
#define GRHD2_ERR_BOUNDARY -6 /* boundary precondition (e.g. nz odd for the 3D torus, conditions.f90:999) */

/* identifiers: variables.f90:224-243 */
enum { GRHD2_REC_GODUNOV = 1, GRHD2_REC_TVD = 2, GRHD2_REC_WENO3 = 3, GRHD2_REC_MP5 = 4,
       GRHD2_REC_WENO5 = 5 };
enum { GRHD2_RS_HLLE = 1, GRHD2_RS_HLLC = 2 };
enum { GRHD2_LIM_MINMOD = 1, GRHD2_LIM_SUPERBEE = 2, GRHD2_LIM_MC = 3 };
/* metric_type / geom_type strings of variables.f90:129-133 as integers */
enum { GRHD2_METRIC_MINKOWSKI = 0, GRHD2_METRIC_EF = 1, GRHD2_METRIC_KS = 2 };
enum { GRHD2_GEOM_CARTESIAN = 0, GRHD2_GEOM_CYLINDRICAL = 1, GRHD2_GEOM_SPHERICAL = 2,
       GRHD2_GEOM_SPHEROIDAL = 3 };
/* precision policies */
/* Precision policies.  FP64: every operation in FP64 (the parity path).  MIXED: the
 * reconstruction, Riemann fluxes and the metric contraction of the sources in FP32, their
 * lapse and sqrt(gamma) factors, con2prim and the RK state u, up in FP64.  MIXED_COMP64 and
 * MIXED_COMP32: MIXED with the RK3 accumulation compensated -- up and u carry the rounding
 * error of every stage combination in a second array (a double-double state: up + carry),
 * the carry stored in FP64 or in FP32. */
enum { GRHD2_PREC_FP64 = 0, GRHD2_PREC_MIXED = 1, GRHD2_PREC_MIXED_COMP64 = 2, GRHD2_PREC_MIXED_COMP32 = 3 };

/* Filled by the Fortran side from the globals of variables.f90.  case_id selects the
 * boundary routine of conditions.f90:773 (1 Sod, 2 strong shock, 3 Shu-Osher, 4 KHI,
 * 5 jet, 6 convergence, 7 Michel, 8 dust, 9 off-axis, 10 FM equatorial, 11 FM sagittal,
 * 12 FM 3D). */
typedef struct {
  int32_t nx, ny, nz, nghost, neq;                         /* neq must be 5 */
  int32_t rec_method, tvd_limiter, riemann, shock_sensor;  /* REC_*, LIM_*, RS_*, 0/1 */
  int32_t metric_kind, geom_kind, use_log_r, case_id;
  int32_t precision_policy;                                /* GRHD2_PREC_* */
  int32_t reserved;
  double dx, dy, dz, adb_idx, g1, cfl;
  double rho_floor, p_floor, v_max;                        /* 1e-10, 1e-13, 1-1e-5 */
} grhd2_gpu_config;

/* The k = 1 slices (the cache is k-invariant: initialization.f90:283,331,351,379) of the
 * reference's metric cache, variables.f90:70-99, Fortran order. */
typedef struct {
  const double *alpha_c;      /* (nx,ny)            */
  const double *beta_c;       /* (3,nx,ny)          */
  const double *gamma_c;      /* (3,3,nx,ny)        */
  const double *gamma_inv_c;  /* (3,3,nx,ny)        */
  const double *gmunu_c;      /* (0:3,0:3,nx,ny)    */
  const double *sqrt_gamma_c; /* (nx,ny)            */
  const double *chris_c;      /* (0:3,0:3,0:3,nx,ny)*/
  const double *dg_c;         /* (0:3,0:3,1:3,nx,ny)*/
  const double *dlna_c;       /* (0:3,nx,ny)        */
  const double *alpha_f_x, *beta_f_x, *gamma_f_x, *sqrt_gamma_f_x; /* (..,nx+1,ny), may be NULL if nx==1 */
  const double *alpha_f_y, *beta_f_y, *gamma_f_y, *sqrt_gamma_f_y; /* (..,nx,ny+1), NULL if ny==1 */
  const double *alpha_f_z, *beta_f_z, *gamma_f_z, *sqrt_gamma_f_z; /* (..,nx,ny),   NULL if nz==1 */
  const double *x_face;       /* (0:nx)  cylindrical axis test, evolution.f90:69 */
  const double *y_face;       /* (0:ny)  polar-face test, evolution.f90:122      */
} grhd2_gpu_metric_view;

/* Per-case boundary data (conditions.f90:229-246, :249-278, :820-870). */
typedef struct {
  const double *michel_injector; /* (5,nghost,ny,nz), case 7, else NULL */
  const double *dust_outer;      /* (5,nghost): evaluate_dust_accretion_state(x(nx+g)), case 8 */
  const double *x_c;             /* x(-g:nx+g) cell centres, case 5 nozzle test */
  double jet[7];                 /* ambient rho, p, vz; nozzle radius; jet rho, p, vz */
} grhd2_gpu_bc_view;

/* Failure and floor counters.  The reference keeps none; these count the branches of
 * cons_to_prim (equations.f90:116-204), the reconstruction floors
 * (reconstruction.f90:647-654) and HLLC exits to HLLE (fluxes.f90:195-396). */
typedef struct {
  int64_t c2p_floor_pre, c2p_causal_rescale, c2p_brent_used, c2p_root_fail, c2p_bad_V,
          c2p_final_sanitise, recon_floor_clamps, hllc_fallbacks;
} grhd2_gpu_counters;

typedef struct grhd2_gpu grhd2_gpu;

/* Create a handle on the current CUDA device (allocates device state).  Replaces the
 * allocation half of allocate_and_grid (initialization.f90:84) for the hot-path arrays.
 * Device buffers come from the device's stream-ordered memory pool (cudaMallocAsync on
 * the handle's stream); grhd2_gpu_destroy returns them in stream order, and the pool keeps
 * up to 8 GiB of released memory for later handles instead of handing it back to the
 * driver, so creating and destroying handles never synchronises the device. */
int grhd2_gpu_create(const grhd2_gpu_config *cfg, grhd2_gpu **out);
/* Upload the metric cache tables (precalculate_metric_cache, initialization.f90:265). */
int grhd2_gpu_set_metric(grhd2_gpu *h, const grhd2_gpu_metric_view *m);

/* What the analytic metric-cache build needs beyond the handle's configuration (which
 * supplies metric_kind, geom_kind, use_log_r, nx, ny, dx and dy). */
typedef struct {
  double bh_mass; /* M of the Eddington-Finkelstein and Kerr-Schild metrics (bh_mass key) */
  double a_spin;  /* Kerr-Schild spin a (spin key)                                        */
  double x_min;   /* first x face: r_min, or ln(r_min) on a logarithmic radial grid      */
  double y_min;   /* first y face (theta_min on polar grids)                              */
} grhd2_gpu_metric_params;
/* Build the metric tables on the device instead of uploading them: the same quantities
 * as precalculate_metric_cache (initialization.f90:265-391) from the analytic metrics
 * (metrics.f90:94-1242) at the cell centres x_min + (i - 1/2) dx, y_min + (j - 1/2) dy and
 * the faces x_min + i dx, y_min + j dy, k-invariant, one thread per (i, j) entry.  Drop-in
 * for grhd2_gpu_set_metric where the caller has no host cache to hand over (the host then
 * builds none).  The device's sin, cos and exp differ from the C library's by a few ulps, so
 * the tables agree with a host-built cache to ~1e-15 relative (bit for bit for Minkowski
 * Cartesian and cylindrical).  Asynchronous on the handle's stream except for a final
 * check of the tables' symmetry; GRHD2_ERR_ARG for an unknown metric or geometry kind. */
int grhd2_gpu_set_metric_analytic(grhd2_gpu *h, const grhd2_gpu_metric_params *mp);
/* Copy a device metric table to the host: which = 0 the centre table (74 fields x nx*ny:
 * lapse, shift, gamma_ij and gamma^ij upper triangles, sqrt(gamma), g^{mu nu},
 * Gamma^0_{mu nu} and d_d g_{mu nu} upper triangles, d_mu ln(alpha), beta^i/alpha), which
 * = 1, 2, 3 the x, y, z face table (21 fields x faces: lapse, normal shift, gamma_ij upper
 * triangle, sqrt(gamma), gamma^dd, the face frame's 9 cofactors, frame flag, axis/pole
 * flag).  n is the capacity of out in doubles; *n_out (may be NULL) receives the table's
 * size, 0 for a direction without faces.  Synchronises the handle's stream. */
int grhd2_gpu_metric_table(grhd2_gpu *h, int32_t which, double *out, size_t n, size_t *n_out);
/* Upload per-case boundary data (cache_michel_injector, conditions.f90:229). */
int grhd2_gpu_set_bc_data(grhd2_gpu *h, const grhd2_gpu_bc_view *b);
/* Copy state in: up(5,nx,ny,nz) and/or p(5,-g:nx+g,-g:ny+g,-g:nz+g); either may be NULL.
 * Used after initialisation, restart (grhd2.f90:95-116) and host-side perturbations. */
int grhd2_gpu_upload(grhd2_gpu *h, const double *up, const double *p);
/* up = prim_to_cons(p) over interior cells (grhd2.f90:126-134, equations.f90:30). */
int grhd2_gpu_prim_to_cons_all(grhd2_gpu *h);
/* dt = update_adaptive_dt() (evolution.f90:198). */
int grhd2_gpu_cfl(grhd2_gpu *h, double *dt_out);
/* One SSP-RK3 step of size dt: u = up; 3 x (rhs, combine, con2prim, boundary)
 * (grhd2.f90:232-265). */
int grhd2_gpu_step(grhd2_gpu *h, double dt);
/* The time loop body of grhd2.f90:179-265 without I/O: steps until t >= final_time or
 * max_steps steps (max_steps < 0: no limit), clamping the last dt (grhd2.f90:182-184). */
int grhd2_gpu_run(grhd2_gpu *h, double t0, double final_time, int64_t max_steps,
                  double *t_out, int64_t *steps_out);
/* rhs(5,nx,ny,nz) = calc_rhs(p) of the resident primitives (evolution.f90:30). */
int grhd2_gpu_calc_rhs(grhd2_gpu *h, double *rhs_host);
/* p = cons_to_prim(up) over interior cells, up modified in place (grhd2.f90:252-260). */
int grhd2_gpu_cons_to_prim_all(grhd2_gpu *h);
/* set_boundary_conditions(p) (conditions.f90:773).  The device state holds no ghost
 * cells (they are evaluated on load), so this only checks the case preconditions. */
int grhd2_gpu_set_boundary(grhd2_gpu *h);
/* Copy state out; either pointer may be NULL.  p receives interior cells and every ghost
 * cell that lies outside the domain in exactly one direction, filled as
 * set_boundary_conditions fills it; ghost cells outside in two or more directions
 * (never read by calc_rhs) are left untouched in the caller's array. */
int grhd2_gpu_download(grhd2_gpu *h, double *up, double *p);
/* ---- diagnostics of the resident state (device reductions; no download needed) ------
 * Per-cell terms follow the reference's arithmetic; sums run in a fixed parallel order,
 * reproducible run to run, equal to the reference's serial loops up to summation order. */
typedef struct {
  double mass_total, disk_mass, angular_momentum;         /* sums of up(D), up(S_3) x cell volume */
  double rho_min, p_min, rho_max, p_max, max_v_sq;       /* over finite values */
  int64_t atmosphere_cells, invalid_cells;
} grhd2_gpu_diagnostics;
/* calc_global_diagnostics (output.f90:1052-1125) without its file output. */
int grhd2_gpu_global_diagnostics(grhd2_gpu *h, grhd2_gpu_diagnostics *out);
/* The mass monitor of the time loop (grhd2.f90:283-301): sum of u(D) dx dy dz, u being
 * the state at the start of the last step (GRHD2_ERR_STATE before the first step). */
int grhd2_gpu_total_mass(grhd2_gpu *h, double *out);
/* calc_m_dot (output.f90:951-992): accretion rate through the cells i = idx_probe
 * (1-based, the first cell centre outside the horizon, initialization.f90:146-161). */
int grhd2_gpu_mdot(grhd2_gpu *h, int idx_probe, double *out);
/* calc_ppi_modes (output.f90:995-1049) without the time column: values[0] = c0, then for
 * m = 1..4: c_real, c_imag, |c_m|/c0, phase at values[1 + 4 (m-1) ...]; z = z(1:nz) cell
 * centres.  All zero when nz < 2. */
int grhd2_gpu_ppi_modes(grhd2_gpu *h, const double *z, double *values);
/* The cell data of a VTK frame (write_vtk_cell_data, output.f90:398-453) as the file holds
 * it: 7 blocks of nx*ny*nz big-endian doubles (i fastest) -- rho, p, v^1, v^2, v^3, alpha,
 * beta^1 -- with v^1 and beta^1 multiplied by r_scale[i-1] = exp(x(i)) when r_scale is not
 * NULL (the log-r grids; pass the host's exp values so the products equal a host writer's).
 * The caller writes the headers and these bytes between them.  out_host: 56*nx*ny*nz bytes. */
int grhd2_gpu_vtk_cell_data(grhd2_gpu *h, const double *r_scale, void *out_host);
/* Checkpoint snapshot (feeds save_checkpoint, output.f90:475-531, which writes up):
 * begin converts up to the reference layout in a device buffer on the handle's stream and
 * copies it to up_host on a separate copy stream, returning at once; steps enqueued
 * afterwards run while the copy proceeds.  wait blocks until up_host holds the snapshot;
 * write the checkpoint file after it.  up_host must stay valid and untouched until then;
 * page-locked memory lets the copy overlap the steps (pageable memory makes begin wait for
 * the copy).  A new begin waits on the device for the previous copy. */
int grhd2_gpu_snapshot_begin(grhd2_gpu *h, double *up_host);
int grhd2_gpu_snapshot_wait(grhd2_gpu *h);
/* calc_gw_strain (output.f90:852-948) without its file output: out = h_plus, h_cross and
 * the quadrupole sums Ixx_ddot, Iyy_ddot, Ixy_ddot.  x, y, z: cell-centre coordinates
 * (1:nx), (1:ny), (1:nz); spin: the Kerr-Schild spin (0 for Eddington-Finkelstein).  All
 * zero when the metric is Minkowski or bh_mass < 0.1 (the reference writes nothing then). */
int grhd2_gpu_gw_strain(grhd2_gpu *h, const double *x, const double *y, const double *z, int use_log_r,
                        double bh_mass, double spin, double *out);
/* Asynchronous upload / download (no reference counterpart): the same copies and layout
 * conversions, enqueued on the handle's stream without waiting.  The host arrays must stay
 * valid and unchanged until the stream has finished (grhd2_gpu_synchronize); page-locked
 * host memory lets the copies overlap kernels of other streams.  A caller that moves the
 * state every step pipelines its grids this way instead of waiting after each copy. */
int grhd2_gpu_upload_async(grhd2_gpu *h, const double *up, const double *p);
int grhd2_gpu_download_async(grhd2_gpu *h, double *up, double *p);
int grhd2_gpu_get_counters(grhd2_gpu *h, grhd2_gpu_counters *out);
int grhd2_gpu_reset_counters(grhd2_gpu *h);
/* Face fluxes for n independent faces (resolve_riemann_problem, fluxes.f90:56):
 * qL,qR,flux (5,n); alpha,sqg (n); beta (3,n); gamma (3,3,n); dir 1..3.  Uses the
 * handle's physics settings (riemann, adb_idx, metric/geometry kind). */
int grhd2_gpu_riemann_faces(grhd2_gpu *h, int n, int dir, const double *qL, const double *qR,
                            const double *alpha, const double *beta, const double *gamma,
                            const double *sqg, double *flux);
/* Allocation-free variant of grhd2_gpu_riemann_faces (no counterpart in the reference):
 * same arguments, same results, but it never allocates memory, on the device or the host.
 * grhd2_gpu_riemann_faces allocates device buffers on every call (from the device's
 * stream-ordered pool); a caller that runs under a fixed memory budget (the device memory
 * is already handed out to a caching allocator or to resident grids), or whose process
 * may not allocate device memory at all, can use this one instead.
 *  - Scratch is one fixed device array in the library, GRHD2_GPU_NOALLOC_MAX_FACES faces
 *    of 50 doubles each (6.6 MB).  n > GRHD2_GPU_NOALLOC_MAX_FACES returns GRHD2_ERR_ARG.
 *  - Nothing in the scratch has to start at zero: each call writes every element it
 *    later reads, and clears the one status word it checks (a face whose frame gamma^dd
 *    differs from its wavespeed gamma^dd returns GRHD2_ERR_ARG, as in
 *    grhd2_gpu_riemann_faces).
 *  - The first call on a device looks up the scratch address (cudaGetSymbolAddress) and
 *    caches it; make that first call before any stream capture.  The cached address
 *    belongs to the device's context at that time: after cudaDeviceReset (or a reset of
 *    the primary context by another library in the process) it is stale, and the process
 *    must not call this entry point on that device again.
 *  - The scratch is shared by every handle of a device: calls made at the same time from
 *    several host threads on the same device race on it.  Serialise them.
 * The call copies and launches on the handle's stream and returns after the flux is on
 * the host. */
#define GRHD2_GPU_NOALLOC_MAX_FACES 16384
int grhd2_gpu_riemann_faces_noalloc(grhd2_gpu *h, int n, int dir, const double *qL, const double *qR,
                                    const double *alpha, const double *beta, const double *gamma,
                                    const double *sqg, double *flux);
/* Physical flux F(q) for n states (calc_fluxes, equations.f90:434). */
int grhd2_gpu_physical_flux(grhd2_gpu *h, int n, int dir, const double *q, const double *alpha,
                            const double *beta, const double *gamma, const double *sqg,
                            double *flux);
/* Wait for all work of the handle; returns the first asynchronous error. */
int grhd2_gpu_synchronize(grhd2_gpu *h);

/* ---- batched grids (no reference counterpart) ---------------------------------------
 * The reference runs independent problems as separate processes
 * (inundaciones.sh:542-548).  Here independent grids -- any sizes, schemes, metrics and
 * boundary cases -- advance together: one launch per kernel kind covers every grid of the
 * batch that uses the same scheme, Riemann solver and precision, and a whole step can be
 * replayed as one CUDA graph.  Each grid keeps its own clock: it steps with its CFL dt,
 * clamped to its final time (grhd2.f90:182-184), and stops when it reaches it. */
typedef struct grhd2_gpu_batch grhd2_gpu_batch;
/* Like grhd2_gpu_create, but the handle works on the caller's CUDA stream (a cudaStream_t;
 * NULL creates a private stream).  Handles that will be batched must share one stream. */
int grhd2_gpu_create_on_stream(const grhd2_gpu_config *cfg, void *stream, grhd2_gpu **out);
/* Move a handle to another stream (NULL: a new private stream) after finishing its work
 * on the old one.  Lets a caller prepare a grid on its own stream, overlapping work that
 * runs on the batch stream, and then join it to a batch.  A batch that holds the handle
 * refuses to step until it is recreated. */
int grhd2_gpu_set_stream(grhd2_gpu *h, void *stream);
/* Device bytes a handle of this configuration allocates (for admission by free memory);
 * -1 for an invalid configuration. */
int64_t grhd2_gpu_device_bytes(const grhd2_gpu_config *cfg);
/* Group n handles (same device and stream, metric and state uploaded).  Grids of one
 * scheme (precision, reconstruction, Riemann solver) share each kernel launch; a scheme
 * group of 2e6 cells or more over several grids is run as two halves whose launches are
 * parallel branches of a step's graph. */
int grhd2_gpu_batch_create(grhd2_gpu **handles, int n, grhd2_gpu_batch **out);
/* Set grid k's clock: time t0, final time, and a step limit (< 0: none).  The CFL dt is
 * computed from the grid's metric (update_adaptive_dt). */
int grhd2_gpu_batch_set_clock(grhd2_gpu_batch *b, int k, double t0, double final_time, int64_t max_steps);
/* Advance every grid that has not reached its final time by up to nsteps steps (one CUDA
 * graph per step when use_graph != 0).  Asynchronous; grids that finish early stop. */
int grhd2_gpu_batch_step(grhd2_gpu_batch *b, int nsteps, int use_graph);
/* grhd2_gpu_cons_to_prim_all of every grid of the batch in one launch per scheme group
 * (or half group; same results and counters).  Asynchronous on the batch's stream: for a caller that
 * uploads the conserved state of many grids (grhd2_gpu_upload_async) and recovers their
 * primitives before stepping. */
int grhd2_gpu_batch_cons_to_prim(grhd2_gpu_batch *b);
/* Read grid k's clock (synchronises the stream). */
int grhd2_gpu_batch_get_clock(grhd2_gpu_batch *b, int k, double *t, int64_t *steps, int *active);
/* Per-launch timing of one batched step (names/ms as in grhd2_gpu_profile_step). */
int grhd2_gpu_batch_profile_step(grhd2_gpu_batch *b, float *ms, const char **names, int cap, int *n_out);
/* Clocks of every member in one call (arrays of n entries, any may be NULL); synchronises
 * the batch stream. */
int grhd2_gpu_batch_clocks(grhd2_gpu_batch *b, double *t, int64_t *steps, int *active);
/* Kernel variants of the face fluxes of one direction. */
#define GRHD2_FLUX_AUTO -1      /* the autotuned choice for this shape if one is cached, else SPLIT_VAR for
                                   launches under ~600k faces and SPLIT above */
#define GRHD2_FLUX_SPLIT 0      /* reconstruction kernel (thread per face) + Riemann kernel */
#define GRHD2_FLUX_FUSED 1      /* one kernel, thread per face, interface states kept on chip */
#define GRHD2_FLUX_SPLIT_VAR 2  /* reconstruction kernel (thread per face and variable) + Riemann kernel */
/* Use one variant for every scheme group and direction of the batch (or AUTO). */
int grhd2_gpu_batch_set_flux_variant(grhd2_gpu_batch *b, int variant);
/* The stage kernel: for grids with at most two active directions (1D, x-y and x-z grids),
 * one kernel per RK stage computes every face of a tile of cells and the tile's cell
 * update through shared memory (the primitives with their stencil halo are staged once;
 * interface states and face fluxes never reach global memory).  Same results and counters
 * as the face and cell kernels.  No reference counterpart (calc_rhs, the RK combination
 * and cons_to_prim of grhd2.f90:232-265 in one pass). */
#define GRHD2_STAGE_AUTO -1  /* the library's choice: the stage kernel for 1D grids (faster there), the
                                face and cell kernels for 2D grids */
#define GRHD2_STAGE_OFF 0    /* face kernels (per the flux variant) and the cell kernel */
#define GRHD2_STAGE_ON 1     /* the stage kernel where it applies (3D grids keep the face and cell kernels) */
int grhd2_gpu_batch_set_stage_kernel(grhd2_gpu_batch *b, int mode);
/* Number of scheme groups of the batch that step with the stage kernel, or a negative error. */
int grhd2_gpu_batch_stage_kernel(grhd2_gpu_batch *b);
/* How a batch runs its steps. */
#define GRHD2_STEP_AUTO -1       /* the library's choice (currently GRAPH, the faster on every size measured) */
#define GRHD2_STEP_GRAPH 0       /* the stage kernels (recon, Riemann, cell update per stage), one CUDA graph */
#define GRHD2_STEP_PERSISTENT 1  /* one cooperative launch per scheme group runs whole steps: fused
                                    face fluxes and cell updates separated by grid barriers */
int grhd2_gpu_batch_set_step_mode(grhd2_gpu_batch *b, int mode);
/* The mode in use (GRHD2_STEP_GRAPH or GRHD2_STEP_PERSISTENT), or a negative error. */
int grhd2_gpu_batch_step_mode(grhd2_gpu_batch *b);
/* Block tile of the face kernels: tx consecutive faces along i per block row, the rest of
 * the block along k (or j for grids without a k extent; the whole block along i for 1D
 * grids).  tx = 32, 64, 128 or 256; 0 restores the automatic choice. */
int grhd2_gpu_batch_set_tile(grhd2_gpu_batch *b, int tx);
/* Time every (variant, tile) pair -- SPLIT, SPLIT_VAR or FUSED, tx 32, 64 or 128 -- per scheme group
 * and active direction (reps launches after a warm-up, on the batch's current state) and
 * keep the fastest; the choice is also cached for later batches of the same precision,
 * scheme, solver, sensor, direction and size class.  The state and counters are left
 * unchanged.  variants[k], tiles[k] (k < cap; either may be NULL) receive the choices in
 * group order, x before y before z; *n_out their number.  Call after the state is set (a
 * grid whose clock is finished does no work and cannot be timed). */
int grhd2_gpu_batch_autotune(grhd2_gpu_batch *b, int reps, int *variants, int *tiles, int cap, int *n_out);
const char *grhd2_gpu_batch_last_error(const grhd2_gpu_batch *b);
void grhd2_gpu_batch_destroy(grhd2_gpu_batch *b);
/* The handle's CUDA stream (a cudaStream_t) so callers can order their own work and
 * record timing events on it.  No reference counterpart (the reference has no device). */
int grhd2_gpu_get_stream(grhd2_gpu *h, void **stream_out);
/* One SSP-RK3 step with a CUDA event around every kernel: ms[k] is the duration of the
 * k-th launch, names[k] its kernel ("face_flux_x", "cell_update", ...); *n_out launches
 * (at most cap are reported).  Observability for the per-stage timers the reference
 * lacks (its only timer is omp_get_wtime around the whole run, grhd2.f90:303-330). */
int grhd2_gpu_profile_step(grhd2_gpu *h, double dt, float *ms, const char **names, int cap, int *n_out);
const char *grhd2_gpu_last_error(const grhd2_gpu *h);
void grhd2_gpu_destroy(grhd2_gpu *h);
int grhd2_gpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
