/*
 * grhd2_oracle.h -- CPU restatement of GRHD2's per-stage RHS and update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle: a plain-C restatement of the
 * reference Fortran (RuelasF/GRHD) hot path, kept in the reference's own data layout
 * (Fortran column-major, array-of-structures, neq=5 fastest, ghosted primitives).
 * Only the test suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * The product library never links or calls it.
 *
 * Arithmetic follows the reference operation by operation (same evaluation order,
 * integer powers as repeated products, no FMA contraction: build with
 * -ffp-contract=off).  Two documented choices where Fortran is processor dependent:
 *   - MAX/MIN with a NaN argument: sequential "keep the first non-NaN" semantics
 *     (m = a; if (b > m || m != m) m = b), also used by the CUDA kernels;
 *   - transcendental functions: the host C library (the same glibc a gfortran build
 *     calls).
 *
 * Layouts (1-based Fortran indices as in variables.f90:60-99):
 *   p   (5, -g:nx+g, -g:ny+g, -g:nz+g)     primitives, ghosted
 *   u/up/rhs (5, nx, ny, nz)               conserved, interior only
 *   metric tables: the k = 1 slice of the reference's metric cache (it is k-invariant,
 *   initialization.f90:283,331,351,379), Fortran order with (i,j) trailing.
 */
#ifndef GRHD2_ORACLE_H
#define GRHD2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* identifiers mirror variables.f90:224-243 */
enum { ORC_REC_GODUNOV = 1, ORC_REC_TVD = 2, ORC_REC_WENO3 = 3, ORC_REC_MP5 = 4, ORC_REC_WENO5 = 5 };
enum { ORC_RS_HLLE = 1, ORC_RS_HLLC = 2 };
enum { ORC_LIM_MINMOD = 1, ORC_LIM_SUPERBEE = 2, ORC_LIM_MC = 3 };
enum { ORC_METRIC_MINKOWSKI = 0, ORC_METRIC_EF = 1, ORC_METRIC_KS = 2 };
enum { ORC_GEOM_CARTESIAN = 0, ORC_GEOM_CYLINDRICAL = 1, ORC_GEOM_SPHERICAL = 2,
       ORC_GEOM_SPHEROIDAL = 3 };

typedef struct {
  int32_t nx, ny, nz, nghost;
  int32_t rec_method, tvd_limiter, riemann, shock_sensor;
  int32_t metric_kind, geom_kind, case_id, pad0;
  double dx, dy, dz, adb_idx, g1, cfl;
  double rho_floor, p_floor, v_max;
} orc_config;

typedef struct {
  /* cell centres, (.., nx, ny) */
  const double *alpha_c, *beta_c, *gamma_c, *gamma_inv_c, *gmunu_c, *sqrt_gamma_c;
  const double *chris_c, *dg_c, *dlna_c;
  /* x faces (.., nx+1, ny), y faces (.., nx, ny+1), z faces (.., nx, ny) */
  const double *alpha_fx, *beta_fx, *gamma_fx, *sqg_fx;
  const double *alpha_fy, *beta_fy, *gamma_fy, *sqg_fy;
  const double *alpha_fz, *beta_fz, *gamma_fz, *sqg_fz;
  /* coordinates: x_face(0:nx), y_face(0:ny), x centres (-g:nx+g) */
  const double *x_face, *y_face, *x_c;
  /* boundary data: Michel injector (5,g,ny,nz), dust outer states (5,g) */
  const double *michel_injector, *dust_outer;
  /* jet parameters: ambient rho,p,vz ; nozzle radius ; jet rho,p,vz */
  double jet[7];
} orc_metric;

typedef struct {
  int64_t c2p_floor_pre, c2p_causal_rescale, c2p_brent_used, c2p_root_fail, c2p_bad_V,
          c2p_final_sanitise, recon_floor_clamps, hllc_fallbacks;
} orc_counters;

/* evolution.f90:30 calc_rhs */
void orc_calc_rhs(const orc_config *c, const orc_metric *m, const double *p, double *rhs,
                  orc_counters *cnt);
/* evolution.f90:198 update_adaptive_dt; returns 0 or a negative error code */
int orc_cfl(const orc_config *c, const orc_metric *m, double *dt_out);
/* equations.f90:94 cons_to_prim for one cell (i,j 1-based; metric is k-invariant) */
void orc_cons_to_prim(const orc_config *c, const orc_metric *m, double *cons, double *prim,
                      int i, int j, orc_counters *cnt);
/* grhd2.f90:252-260 sweep over all interior cells */
void orc_cons_to_prim_all(const orc_config *c, const orc_metric *m, double *up, double *p,
                          orc_counters *cnt);
/* equations.f90:30 prim_to_cons, one cell */
void orc_prim_to_cons(const orc_config *c, const orc_metric *m, const double *prim,
                      double *cons, int i, int j);
void orc_prim_to_cons_all(const orc_config *c, const orc_metric *m, const double *p,
                          double *up);
/* conditions.f90:773 set_boundary_conditions; returns 0 or a negative error code */
int orc_set_boundary(const orc_config *c, const orc_metric *m, double *p);
/* fluxes.f90:56 resolve_riemann_problem for one face; g is the Fortran (3,3) array */
void orc_riemann(const orc_config *c, const double *qL, const double *qR, int dir,
                 double alpha, const double *beta, const double *g, double sqg,
                 double *flux, orc_counters *cnt);
/* equations.f90:434 calc_fluxes */
void orc_physical_flux(const orc_config *c, const double *q, int dir, double alpha,
                       const double *beta, const double *g, double sqg, double *f);
/* reconstruction.f90:285 reconstruct_1d_core on one strip prim(5,-g:n+g) */
void orc_reconstruct(const orc_config *c, const double *prim, int nodes, int dir,
                     double *qL, double *qR, orc_counters *cnt);
/* grhd2.f90:232-265: one SSP-RK3 step (u = up; BC; 3 x (rhs, combine, c2p, BC)).
 * rhs is scratch of size 5*nx*ny*nz. Returns 0 or a negative error code. */
int orc_step(const orc_config *c, const orc_metric *m, double *u, double *up, double *p,
             double *rhs, double dt, orc_counters *cnt);
/* grhd2.f90:179-265 time loop without I/O: runs while t < final_time or until max_steps
 * steps; returns the number of steps taken (>= 0) or a negative error code. */
int64_t orc_run(const orc_config *c, const orc_metric *m, double *up, double *p,
                double t0, double final_time, int64_t max_steps, double *t_out,
                orc_counters *cnt);
/* Diagnostics (loops in the reference's order, serial).
 * grhd2.f90:283-301 mass monitor: sum of u(D) dx dy dz over interior cells */
double orc_total_mass(const orc_config *c, const double *u);
/* output.f90:951-992 calc_m_dot at cell i = idx_probe (1-based): -sum_j,k up(D) v_eff dy dz,
 * v_eff = alpha p(vx) - beta^1; returns 0 and writes *out, or -1 for an invalid index */
int orc_mdot(const orc_config *c, const orc_metric *m, const double *up, const double *p, int idx_probe,
             double *out);
/* output.f90:995-1049 calc_ppi_modes without the time column: values[0] = c0, then per
 * mode m = 1..4: c_real, c_imag, |c|/c0, phase (values[1 + 4 (m-1) ..]); z = z(1:nz) */
void orc_ppi_modes(const orc_config *c, const double *up, const double *p, const double *z, double *values);
/* output.f90:1052-1125 calc_global_diagnostics without the time column:
 * f = mass_total, disk_mass, angular_momentum, rho_min, p_min, rho_max, p_max, max_v_sq;
 * n = atmosphere_cells, invalid_cells */
void orc_global_diagnostics(const orc_config *c, const orc_metric *m, const double *up, const double *p,
                            double *f, int64_t *n);
/* output.f90:852-948 calc_gw_strain (Finn-Evans quadrupole proxy, observer at 1000 M,
 * cells inside the horizon and the numerical atmosphere excluded): out = h_plus, h_cross,
 * Ixx_ddot, Iyy_ddot, Ixy_ddot; xc, yc, zc the cell centres (1:n); spin the KS spin (0 for
 * EF).  Returns 0, 1 when the reference skips (Minkowski or bh_mass < 0.1), or -1 when
 * the horizon radius is undefined (metrics.f90:66-87). */
int orc_gw_strain(const orc_config *c, const orc_metric *m, const double *p, const double *xc, const double *yc,
                  const double *zc, int use_log_r, double bh_mass, double spin, double *out);
/* The pieces of calc_gw_strain, exposed for the reference's GW tests
 * (tests/test_gw_geometry.f90, tests/test_gw_stress.f90): event_horizon_radius
 * (metrics.f90:66-87; -1 where it is undefined), kerr_schild_spheroidal_position
 * (output.f90:743-768), gw_cartesian_kinematics (output.f90:797-834; v the Eulerian
 * velocity, beta the shift, both in grid components) and finn_evans_cell_stress
 * (output.f90:837-850). */
int orc_horizon_radius(double mass, double spin, double *r_plus);
void orc_ks_spheroidal_position(double r, double theta, double phi, double spin, double *pos);
void orc_gw_kinematics(double r, double theta, double phi, double spin, double alpha, const double *beta,
                       const double *v, int use_log_r, double *pos, double *vel, double *jac);
void orc_finn_evans_stress(double rho, double pres, double mr3, const double *pos, const double *vel, double dV,
                           double *ixx, double *iyy, double *ixy);
/* calc_sources (equations.f90:509-552) with calculate_stress_energy_tensor
 * (metrics.f90:1251-1310) for one cell (i,j 1-based) and primitive state prim(5) */
void orc_sources(const orc_config *c, const orc_metric *m, const double *prim, int i, int j, double *src);
/* root_brent (equations.f90:339-424) alone, for its restatement cross-check: cs(5) the
 * conserved state, ginv the inverse 3-metric (Fortran order) */
double orc_root_brent(const orc_config *c, const double *cs, const double *ginv);
/* number of OpenMP threads used by orc_run / orc_step (1 without OpenMP) */
int orc_num_threads(void);
/* the exp used by WENO3 (reconstruction.f90:169), exposed for its accuracy test */
double orc_exp(double x);

#ifdef __cplusplus
}
#endif
#endif
