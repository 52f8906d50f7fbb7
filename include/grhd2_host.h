/*
 * grhd2_host.h -- host-side problem setup that feeds the grhd2_gpu C-ABI.
 *
 * In a Fortran deployment this side is the unchanged reference driver: the .par reader
 * (parameters.f90), the presets and the metric cache (initialization.f90), the initial
 * conditions and perturbations (conditions.f90) and the analytic metrics (metrics.f90).
 * This library restates those init-time routines in C++ so the GPU path can be driven
 * without a Fortran compiler (benchmarks, the solve server, tests).  It performs no
 * hot-path arithmetic: every per-stage operation lives in grhd2_gpu.
 *
 * Parameters use the reference's .par keys (parameters.f90:147-349), one "key = value"
 * per line, '#' or '!' comments.  Angles theta_min/max and phi_min/max are in units of pi.
 */
#ifndef GRHD2_HOST_H
#define GRHD2_HOST_H

#include <stdint.h>
#include "grhd2_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct grhd2_problem grhd2_problem;

typedef struct {
  int32_t case_id, nx, ny, nz, nghost;
  int32_t perturbation_type; /* 0 none, 1 pressure noise, 2 density noise, 3 density mode */
  int64_t perturbation_seed;
  double final_time, cfl, perturbation_time, perturbation_amplitude, perturbation_mode;
  double x_min, x_max, y_min, y_max, z_min, z_max;
  double bh_mass, a_spin, fm_l, fm_w_in;
} grhd2_problem_info;

/* Build a problem from .par text (problem = sod | michel | fishbone_equatorial | ...). On
 * failure returns a negative code and writes a message into err (if errlen > 0). */
int grhd2_problem_create(const char *par_text, grhd2_problem **out, char *err, int errlen);
/* grhd2_problem_create with flags.  GRHD2_PROBLEM_NO_METRIC_CACHE: build no host metric
 * cache (the caller builds the tables on the device with grhd2_gpu_set_metric_analytic);
 * grhd2_problem_metric then fills only x_face and y_face and returns GRHD2_ERR_STATE. */
#define GRHD2_PROBLEM_NO_METRIC_CACHE 1u
int grhd2_problem_create_ex(const char *par_text, uint32_t flags, grhd2_problem **out, char *err, int errlen);
void grhd2_problem_destroy(grhd2_problem *pb);
int grhd2_problem_config(const grhd2_problem *pb, int32_t precision_policy, grhd2_gpu_config *cfg);
int grhd2_problem_metric(const grhd2_problem *pb, grhd2_gpu_metric_view *mv);
int grhd2_problem_bc(const grhd2_problem *pb, grhd2_gpu_bc_view *bv);
int grhd2_problem_info_get(const grhd2_problem *pb, grhd2_problem_info *info);
/* Initial primitives p(5,-g:nx+g,-g:ny+g,-g:nz+g) after set_initial_conditions
 * (conditions.f90:26); the array is owned by the problem. */
const double *grhd2_problem_prims(const grhd2_problem *pb);
/* Number of doubles in the ghosted primitive array and in an interior conserved array. */
int64_t grhd2_problem_prim_size(const grhd2_problem *pb);
int64_t grhd2_problem_cons_size(const grhd2_problem *pb);
/* Apply the configured perturbation (inject_pressure_noise / inject_density_noise /
 * inject_density_mode, conditions.f90:603-768) to a ghosted primitive array in place.
 * The noise generator is SplitMix64(seed) mapped to [0,1), not gfortran's
 * random_number; the selection rule and the arithmetic are the reference's. */
int grhd2_problem_perturb(const grhd2_problem *pb, double *p);
/* Cell-centre coordinates x(-g:nx+g), y(-g:ny+g), z(-g:nz+g). */
const double *grhd2_problem_x(const grhd2_problem *pb);
const double *grhd2_problem_y(const grhd2_problem *pb);
const double *grhd2_problem_z(const grhd2_problem *pb);

/* Analytic metric evaluation at (x, y) for the problem's metric and geometry
 * (metrics.f90 calculate_metric / christoffel / derivatives); any output may be NULL. */
int grhd2_problem_eval_metric(const grhd2_problem *pb, double x, double y, double *alpha,
                              double *beta, double *gamma, double *gmunu, double *det,
                              double *dlnalpha, double *chris, double *dg);

/* The same evaluation for any metric kind and geometry (GRHD2_METRIC_*, GRHD2_GEOM_*), with
 * the module globals metric_type, geom_type, use_log_r, bh_mass, a_spin and ny set directly
 * and no .par checks -- as the reference's set-up tests set them
 * (tests/test_minkowski_spherical.f90:19-87 evaluates Eddington-Finkelstein at M = 0).
 * Replaces set_metric_type + calculate_metric / calculate_christoffel_symbols /
 * calculate_metric_derivatives (metrics.f90:94-201, :209-1242). */
int grhd2_host_metric_at(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass,
                         double a_spin, int32_t ny, double x, double y, double *alpha, double *beta,
                         double *gamma, double *gmunu, double *det, double *dlnalpha, double *chris,
                         double *dg);
/* prepare_fishbone_moncrief (conditions.f90:470-510): the torus's constant specific angular
 * momentum l and the potential W_in at its inner edge; *ok = 0 where the reference reports
 * failure. */
int grhd2_host_fm_prepare(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass,
                          double a_spin, double r_in, double r_max, double *l_ang, double *w_in,
                          int32_t *ok);
/* evaluate_fishbone_moncrief_state (conditions.f90:516-572) at (radius, theta), the metric
 * evaluated there (radius is mapped to log(radius) on a logarithmic grid): state(5) and
 * whether the point belongs to the torus (*inside = 0: the floor atmosphere). */
int grhd2_host_fm_state(int32_t metric_kind, int32_t geom_kind, int32_t use_log_r, double bh_mass,
                        double a_spin, double adiabatic_index, double rho_floor, double p_floor,
                        double radius, double theta, double r_in, double K, double l_ang, double w_in,
                        double *state, int32_t *inside);
/* evaluate_dust_accretion_state (conditions.f90:249-278) at the radial coordinate x (r, or
 * log r on a logarithmic grid) with the module globals bh_mass, dust_accretion_constant and
 * p_floor set directly, as tests/test_case_corrections.f90:186-232 sets them: state(5).
 * GRHD2_ERR_ARG for the parameters the reference rejects (r <= 0, M <= 0, constant >= 0). */
int grhd2_host_dust_state(int32_t use_log_r, double bh_mass, double dust_accretion_constant, double p_floor,
                          double x, double *state);

#ifdef __cplusplus
}
#endif
#endif
