/*
 * grhd2_oracle.c -- CPU restatement of GRHD2's per-stage RHS and update path.
 *
 * TEST INFRASTRUCTURE ONLY (parity oracle and CPU baseline).  See grhd2_oracle.h for the
 * layout and the two documented processor-dependent choices.  Every function cites the
 * reference routine (file:line in RuelasF/GRHD) whose arithmetic it restates; the
 * evaluation order of each expression follows the Fortran source left to right, with
 * integer powers written as repeated products (x**2 -> x*x, x**3 -> (x*x)*x).
 *
 * Build: gcc -O2 -std=c99 -ffp-contract=off -fno-fast-math -fopenmp -fPIC -shared.
 */
#include "grhd2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NEQ 5
#define EQ_DE 0
#define EQ_PR 1
#define EQ_VX 2
#define EQ_VY 3
#define EQ_VZ 4
#define DIR_X 1
#define DIR_Y 2
#define DIR_Z 3

/* ---------------------------------------------------------------------------------- */
/* Fortran intrinsic semantics                                                          */
/* ---------------------------------------------------------------------------------- */
static inline double fmax_ref(double a, double b) { return (b > a || a != a) ? b : a; }
static inline double fmin_ref(double a, double b) { return (b < a || a != a) ? b : a; }
static inline double max3(double a, double b, double c) { return fmax_ref(fmax_ref(a, b), c); }
static inline double min3(double a, double b, double c) { return fmin_ref(fmin_ref(a, b), c); }
static inline double max4(double a, double b, double c, double d) {
  return fmax_ref(fmax_ref(fmax_ref(a, b), c), d);
}
static inline double min4(double a, double b, double c, double d) {
  return fmin_ref(fmin_ref(fmin_ref(a, b), c), d);
}
static inline double max5(double a, double b, double c, double d, double e) {
  return fmax_ref(max4(a, b, c, d), e);
}
static inline double min5(double a, double b, double c, double d, double e) {
  return fmin_ref(min4(a, b, c, d), e);
}
/* exp(x) for the WENO3 adaptive epsilon (reconstruction.f90:169).  The reference calls
 * the C library's exp, whose last-bit rounding the CUDA exp does not share; a one-ulp
 * difference there flips downstream branches (MP5's "< 1e-10" test, HLLC tolerances) and
 * breaks bit-level parity.  Both this oracle and the kernels therefore evaluate exp with
 * the same published method: Cody-Waite reduction x = k ln2 + r, k = rint(x/ln2), ln2
 * split into a 32-bit head and a tail; e^r by the Taylor series through r^13/13!
 * (|r| <= ln2/2, truncation below 5e-18 relative) in Horner form; exact scaling by 2^k.
 * It differs from a correctly rounded exp by at most about one ulp.  Build with
 * -DORC_LIBM_EXP to use the C library's exp instead. */
static double exp_cw(double x) {
#ifdef ORC_LIBM_EXP
  return exp(x);
#else
  if (x != x) return x;
  if (x > 709.78) return HUGE_VAL;
  if (x < -745.2) return 0.0;
  const double log2e = 0x1.71547652b82fep+0;
  const double ln2_hi = 0x1.62e42feep-1;         /* ln 2 to 32 significant bits */
  const double ln2_lo = 0x1.a39ef35793c76p-33;   /* ln 2 - ln2_hi */
  const double k = rint(x * log2e);
  const double r = (x - k * ln2_hi) - k * ln2_lo;
  double p = 1.0 / 6227020800.0;
  p = 1.0 / 479001600.0 + r * p;
  p = 1.0 / 39916800.0 + r * p;
  p = 1.0 / 3628800.0 + r * p;
  p = 1.0 / 362880.0 + r * p;
  p = 1.0 / 40320.0 + r * p;
  p = 1.0 / 5040.0 + r * p;
  p = 1.0 / 720.0 + r * p;
  p = 1.0 / 120.0 + r * p;
  p = 1.0 / 24.0 + r * p;
  p = 1.0 / 6.0 + r * p;
  p = 0.5 + r * p;
  p = 1.0 + r * p;
  return ldexp(1.0 + r * p, (int)k);
#endif
}

double orc_exp(double x) { return exp_cw(x); }

/* Fortran sign(1.0d0, x): honours the sign bit, including -0.0 */
static inline double sgn1(double x) { return copysign(1.0, x); }
static inline int isfin(double x) { return isfinite(x); }

/* ---------------------------------------------------------------------------------- */
/* layout helpers                                                                       */
/* ---------------------------------------------------------------------------------- */
typedef struct {
  int nx, ny, nz, g;
  size_t sx, sy, sz; /* element strides of p in i, j, k (in units of doubles) */
} lay_t;

static lay_t mklay(const orc_config *c) {
  lay_t L;
  L.nx = c->nx; L.ny = c->ny; L.nz = c->nz; L.g = c->nghost;
  L.sx = NEQ;
  L.sy = (size_t)NEQ * (size_t)(c->nx + 2 * c->nghost + 1);
  L.sz = L.sy * (size_t)(c->ny + 2 * c->nghost + 1);
  return L;
}
/* p(v, i, j, k), v 0-based, i,j,k Fortran 1-based (ghosts allowed) */
static inline size_t pidx(const lay_t *L, int v, int i, int j, int k) {
  return (size_t)v + L->sx * (size_t)(i + L->g) + L->sy * (size_t)(j + L->g) +
         L->sz * (size_t)(k + L->g);
}
static inline size_t uidx(const orc_config *c, int v, int i, int j, int k) {
  return (size_t)v + NEQ * ((size_t)(i - 1) + (size_t)c->nx * ((size_t)(j - 1) +
                                                              (size_t)c->ny * (size_t)(k - 1)));
}
static inline size_t cell(const orc_config *c, int i, int j) {
  return (size_t)(i - 1) + (size_t)c->nx * (size_t)(j - 1);
}
#define G3(g, a, b) ((g)[((a) - 1) + 3 * ((b) - 1)])

static void add_counters(orc_counters *dst, const orc_counters *src) {
  if (!dst) return;
  dst->c2p_floor_pre += src->c2p_floor_pre;
  dst->c2p_causal_rescale += src->c2p_causal_rescale;
  dst->c2p_brent_used += src->c2p_brent_used;
  dst->c2p_root_fail += src->c2p_root_fail;
  dst->c2p_bad_V += src->c2p_bad_V;
  dst->c2p_final_sanitise += src->c2p_final_sanitise;
  dst->recon_floor_clamps += src->recon_floor_clamps;
  dst->hllc_fallbacks += src->hllc_fallbacks;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---------------------------------------------------------------------------------- */
/* reconstruction.f90:28-278 limiters and interface formulas                            */
/* ---------------------------------------------------------------------------------- */
/* reconstruction.f90:28 */
static inline double minmod_2(double a, double b) {
  return 0.5 * (sgn1(a) + sgn1(b)) * fmin_ref(fabs(a), fabs(b));
}
/* reconstruction.f90:34 */
static inline double minmod_3(double a, double b, double c) {
  return sgn1(a) * fmax_ref(0.0, min3(fabs(a), sgn1(a) * b, sgn1(a) * c));
}
/* reconstruction.f90:40 */
static inline double minmod_4(double a, double b, double c, double d) {
  return 0.125 * (sgn1(a) + sgn1(b)) * fabs(sgn1(a) + sgn1(c)) * fabs(sgn1(a) + sgn1(d)) *
         min4(fabs(a), fabs(b), fabs(c), fabs(d));
}
/* reconstruction.f90:141-181 (adaptive-epsilon WENO3); q[0..2] = q(-1:1) */
static double weno3_interface(const double *q) {
  const double eps_min = 1.0e-14;
  const double d0 = 2.0 / 3.0, d1 = 1.0 / 3.0;
  double p0 = 0.5 * q[1] + 0.5 * q[2];
  double p1 = -0.5 * q[0] + 1.5 * q[1];
  double t0 = q[1] - q[2], t1 = q[0] - q[1];
  double beta_0 = t0 * t0;
  double beta_1 = t1 * t1;
  double shock_sensor = fabs(beta_0 - beta_1) / (fmax_ref(beta_0, beta_1) + eps_min);
  double eps_hybrid = eps_min + (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * exp_cw(-10.0 * shock_sensor);
  double e0 = eps_hybrid + beta_0, e1 = eps_hybrid + beta_1;
  double alpha_0 = d0 / (e0 * e0);
  double alpha_1 = d1 / (e1 * e1);
  double weight_0 = alpha_0 / (alpha_0 + alpha_1);
  double weight_1 = alpha_1 / (alpha_0 + alpha_1);
  return weight_0 * p0 + weight_1 * p1;
}
/* reconstruction.f90:187-215 (WENO5-Z); q[0..4] = q(-2:2) */
static double weno5_interface(const double *q) {
  const double eps = 1.0e-14;
  const double d0 = 0.3, d1 = 0.6, d2 = 0.1;
  double a, b;
  a = q[2] - 2.0 * q[3] + q[4]; b = 3.0 * q[2] - 4.0 * q[3] + q[4];
  double b0 = 13.0 / 12.0 * (a * a) + 0.25 * (b * b);
  a = q[1] - 2.0 * q[2] + q[3]; b = q[1] - q[3];
  double b1 = 13.0 / 12.0 * (a * a) + 0.25 * (b * b);
  a = q[0] - 2.0 * q[1] + q[2]; b = q[0] - 4.0 * q[1] + 3.0 * q[2];
  double b2 = 13.0 / 12.0 * (a * a) + 0.25 * (b * b);
  double tau5 = fabs(b0 - b2);
  double a0 = d0 * (1.0 + (tau5 / (eps + b0)));
  double a1 = d1 * (1.0 + (tau5 / (eps + b1)));
  double a2 = d2 * (1.0 + (tau5 / (eps + b2)));
  double w0 = a0 / (a0 + a1 + a2);
  double w1 = a1 / (a0 + a1 + a2);
  double w2 = a2 / (a0 + a1 + a2);
  double p0 = (1.0 / 3.0) * q[2] + (5.0 / 6.0) * q[3] - (1.0 / 6.0) * q[4];
  double p1 = -((1.0 / 6.0) * q[1]) + (5.0 / 6.0) * q[2] + (1.0 / 3.0) * q[3];
  double p2 = (1.0 / 3.0) * q[0] - (7.0 / 6.0) * q[1] + (11.0 / 6.0) * q[2];
  return w0 * p0 + w1 * p1 + w2 * p2;
}
/* reconstruction.f90:222-254 (MP5); q[0..4] = q(-2:2) */
static double mp5_interface(const double *q) {
  const double alpha_mp5 = 4.0, eps = 1.0e-10;
  double val_L = (2.0 * q[0] - 13.0 * q[1] + 47.0 * q[2] + 27.0 * q[3] - 3.0 * q[4]) / 60.0;
  double val_mp = q[2] + minmod_2(q[3] - q[2], alpha_mp5 * (q[2] - q[1]));
  if ((val_L - q[2]) * (val_L - val_mp) < eps) return val_L;
  double d_jm1 = q[0] - 2.0 * q[1] + q[2];
  double d_j = q[1] - 2.0 * q[2] + q[3];
  double d_jp1 = q[2] - 2.0 * q[3] + q[4];
  double dm4_jph = minmod_4(4.0 * d_j - d_jp1, 4.0 * d_jp1 - d_j, d_j, d_jp1);
  double dm4_jmh = minmod_4(4.0 * d_j - d_jm1, 4.0 * d_jm1 - d_j, d_j, d_jm1);
  double val_ul = q[2] + alpha_mp5 * (q[2] - q[1]);
  double val_av = 0.5 * (q[2] + q[3]);
  double val_md = val_av - 0.5 * dm4_jph;
  double val_lc = q[2] + 0.5 * (q[2] - q[1]) + 4.0 * dm4_jmh / 3.0;
  double val_min = fmax_ref(min3(q[2], q[3], val_md), min3(q[2], val_ul, val_lc));
  double val_max = fmin_ref(max3(q[2], q[3], val_md), max3(q[2], val_ul, val_lc));
  return val_L + minmod_2(val_min - val_L, val_max - val_L);
}
/* reconstruction.f90:259-278 */
static double tvd_slope(double a, double b, int limiter_id) {
  switch (limiter_id) {
  case ORC_LIM_MINMOD: return minmod_2(a, b);
  case ORC_LIM_SUPERBEE:
    if (a * b <= 0.0) return 0.0;
    return sgn1(a) * fmax_ref(fmin_ref(2.0 * fabs(a), fabs(b)), fmin_ref(fabs(a), 2.0 * fabs(b)));
  case ORC_LIM_MC: return minmod_3(2.0 * b, 0.5 * (a + b), 2.0 * a);
  default: return minmod_2(a, b);
  }
}

/* ---------------------------------------------------------------------------------- */
/* reconstruction.f90:285-657 reconstruct_1d_core                                        */
/* prim(v,i) = prim[v + 5*(i+g)], i = -g..nodes+g ; qL/qR(v,i) = q[v + 5*i], i=0..nodes  */
/* ---------------------------------------------------------------------------------- */
void orc_reconstruct(const orc_config *c, const double *prim, int nodes, int dir,
                     double *qL, double *qR, orc_counters *cnt) {
  const int g = c->nghost;
#define P1(v, i) prim[(v) + NEQ * ((i) + g)]
  const double atm_factor = 1.0e2;
  const double p_tol_tvd = 0.80, rho_tol_tvd = 0.50, p_tol_weno = 0.40, rho_tol_weno = 0.15;
  const double p_tol_godunov = 10.0, rho_tol_godunov = 10.0;
  const int nonmink = c->metric_kind != ORC_METRIC_MINKOWSKI;
  const double rho_floor = c->rho_floor, p_floor = c->p_floor;
  double st[6];
  int i, k;

  for (i = 0; i <= nodes; ++i) {
    double p_jump = 0.0, rho_jump = 0.0;
    if (c->rec_method != ORC_REC_GODUNOV && c->shock_sensor) {
      double p_max = max5(P1(EQ_PR, i - 2), P1(EQ_PR, i - 1), P1(EQ_PR, i), P1(EQ_PR, i + 1), P1(EQ_PR, i + 2));
      double p_min = min5(P1(EQ_PR, i - 2), P1(EQ_PR, i - 1), P1(EQ_PR, i), P1(EQ_PR, i + 1), P1(EQ_PR, i + 2));
      double rho_max = max5(P1(EQ_DE, i - 2), P1(EQ_DE, i - 1), P1(EQ_DE, i), P1(EQ_DE, i + 1), P1(EQ_DE, i + 2));
      double rho_min = min5(P1(EQ_DE, i - 2), P1(EQ_DE, i - 1), P1(EQ_DE, i), P1(EQ_DE, i + 1), P1(EQ_DE, i + 2));
      p_jump = (p_max > 1.0e3 * p_floor) ? (p_max - p_min) / fmax_ref(p_min, p_floor) : 0.0;
      rho_jump = (rho_max > 1.0e3 * rho_floor) ? (rho_max - rho_min) / fmax_ref(rho_min, rho_floor) : 0.0;
    }
    for (k = 0; k < NEQ; ++k) {
      double *l = &qL[k + NEQ * i], *r = &qR[k + NEQ * i];
      int godunov = 0, tvd_mc = 0, weno3 = 0;
      switch (c->rec_method) {
      case ORC_REC_GODUNOV:
        godunov = 1;
        break;
      case ORC_REC_TVD:
        if (c->shock_sensor) {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1;
          else if (P1(EQ_DE, i) <= atm_factor * rho_floor || P1(EQ_DE, i + 1) <= atm_factor * rho_floor) godunov = 1;
          else if (p_jump >= p_tol_godunov || rho_jump >= rho_tol_godunov) godunov = 1;
        }
        if (!godunov) {
          double sminL = P1(k, i) - P1(k, i - 1), smaxL = P1(k, i + 1) - P1(k, i);
          *l = P1(k, i) + 0.5 * tvd_slope(sminL, smaxL, c->tvd_limiter);
          double sminR = P1(k, i + 1) - P1(k, i), smaxR = P1(k, i + 2) - P1(k, i + 1);
          *r = P1(k, i + 1) - 0.5 * tvd_slope(sminR, smaxR, c->tvd_limiter);
          continue;
        }
        break;
      case ORC_REC_WENO3:
        if (c->shock_sensor) {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1;
          else if (P1(EQ_DE, i) <= atm_factor * rho_floor || P1(EQ_DE, i + 1) <= atm_factor * rho_floor) godunov = 1;
          else if (p_jump >= p_tol_godunov || rho_jump >= rho_tol_godunov) godunov = 1;
          else if (p_jump >= p_tol_tvd || rho_jump >= rho_tol_tvd) tvd_mc = 1;
          else weno3 = 1;
        } else {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1; else weno3 = 1;
        }
        break;
      case ORC_REC_MP5:
        if (c->shock_sensor) {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1;
          else if (P1(EQ_DE, i) <= atm_factor * rho_floor || P1(EQ_DE, i + 1) <= atm_factor * rho_floor) godunov = 1;
          else if (p_jump >= p_tol_godunov || rho_jump >= rho_tol_godunov) godunov = 1;
          else if (p_jump >= p_tol_tvd || rho_jump >= rho_tol_tvd) tvd_mc = 1;
          else if (p_jump >= p_tol_weno || rho_jump >= rho_tol_weno ||
                   (nonmink && dir == DIR_X && i <= 3) ||
                   (nonmink && dir == DIR_Y && (i <= 2 || i >= nodes - 2))) weno3 = 1;
          else {
            st[0] = P1(k, i - 2); st[1] = P1(k, i - 1); st[2] = P1(k, i); st[3] = P1(k, i + 1); st[4] = P1(k, i + 2);
            *l = mp5_interface(st);
            st[0] = P1(k, i + 3); st[1] = P1(k, i + 2); st[2] = P1(k, i + 1); st[3] = P1(k, i); st[4] = P1(k, i - 1);
            *r = mp5_interface(st);
            continue;
          }
        } else {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1;
          else {
            st[0] = P1(k, i - 2); st[1] = P1(k, i - 1); st[2] = P1(k, i); st[3] = P1(k, i + 1); st[4] = P1(k, i + 2);
            *l = mp5_interface(st);
            st[0] = P1(k, i + 3); st[1] = P1(k, i + 2); st[2] = P1(k, i + 1); st[3] = P1(k, i); st[4] = P1(k, i - 1);
            *r = mp5_interface(st);
            continue;
          }
        }
        break;
      case ORC_REC_WENO5:
      default:
        if (c->shock_sensor) {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1;
          else if (P1(EQ_DE, i) <= atm_factor * rho_floor || P1(EQ_DE, i + 1) <= atm_factor * rho_floor) godunov = 1;
          else if (p_jump >= p_tol_godunov || rho_jump >= rho_tol_godunov) godunov = 1;
          else if (p_jump >= p_tol_tvd || rho_jump >= rho_tol_tvd) tvd_mc = 1;
          else if (p_jump >= p_tol_weno || rho_jump >= rho_tol_weno) weno3 = 1;
        } else {
          if (nonmink && dir == DIR_X && i <= 0) godunov = 1;
        }
        if (!godunov && !tvd_mc && !weno3) {
          st[0] = P1(k, i - 2); st[1] = P1(k, i - 1); st[2] = P1(k, i); st[3] = P1(k, i + 1); st[4] = P1(k, i + 2);
          *l = weno5_interface(st);
          st[0] = P1(k, i + 3); st[1] = P1(k, i + 2); st[2] = P1(k, i + 1); st[3] = P1(k, i); st[4] = P1(k, i - 1);
          *r = weno5_interface(st);
          continue;
        }
        break;
      }
      if (godunov) {
        *l = P1(k, i);
        *r = P1(k, i + 1);
      } else if (tvd_mc) {
        double sminL = P1(k, i) - P1(k, i - 1), smaxL = P1(k, i + 1) - P1(k, i);
        *l = P1(k, i) + 0.5 * tvd_slope(sminL, smaxL, ORC_LIM_MC);
        double sminR = P1(k, i + 1) - P1(k, i), smaxR = P1(k, i + 2) - P1(k, i + 1);
        *r = P1(k, i + 1) - 0.5 * tvd_slope(sminR, smaxR, ORC_LIM_MC);
      } else if (weno3) {
        st[0] = P1(k, i - 1); st[1] = P1(k, i); st[2] = P1(k, i + 1);
        *l = weno3_interface(st);
        st[0] = P1(k, i + 2); st[1] = P1(k, i + 1); st[2] = P1(k, i);
        *r = weno3_interface(st);
      }
    }
  }
  /* reconstruction.f90:647-655 positivity floors */
  for (i = 0; i <= nodes; ++i) {
    double *v;
    v = &qL[EQ_DE + NEQ * i]; if (cnt && !(*v >= rho_floor)) cnt->recon_floor_clamps++; *v = fmax_ref(*v, rho_floor);
    v = &qR[EQ_DE + NEQ * i]; if (cnt && !(*v >= rho_floor)) cnt->recon_floor_clamps++; *v = fmax_ref(*v, rho_floor);
    v = &qL[EQ_PR + NEQ * i]; if (cnt && !(*v >= p_floor)) cnt->recon_floor_clamps++; *v = fmax_ref(*v, p_floor);
    v = &qR[EQ_PR + NEQ * i]; if (cnt && !(*v >= p_floor)) cnt->recon_floor_clamps++; *v = fmax_ref(*v, p_floor);
  }
#undef P1
}

/* ---------------------------------------------------------------------------------- */
/* equations.f90 / fluxes.f90 pointwise physics                                         */
/* ---------------------------------------------------------------------------------- */
/* the velocity cap shared by calc_fluxes (equations.f90:451-464), prim_to_cons_face
 * (fluxes.f90:87-100), the wavespeed routines and calculate_stress_energy_tensor */
static double capped_velocity(const double *g, double *v, double v_max) {
  double v_sq = 0.0;
  int ii, jj;
  for (ii = 1; ii <= 3; ++ii)
    for (jj = 1; jj <= 3; ++jj) v_sq = v_sq + G3(g, ii, jj) * v[ii - 1] * v[jj - 1];
  if (v_sq >= v_max) {
    v[0] = v[0] * sqrt(v_max / v_sq);
    v[1] = v[1] * sqrt(v_max / v_sq);
    v[2] = v[2] * sqrt(v_max / v_sq);
    v_sq = v_max;
  }
  return v_sq;
}
static void lower_index(const double *g, const double *v, double *v_cov) {
  int ii, jj;
  for (ii = 1; ii <= 3; ++ii) {
    v_cov[ii - 1] = 0.0;
    for (jj = 1; jj <= 3; ++jj) v_cov[ii - 1] = v_cov[ii - 1] + G3(g, ii, jj) * v[jj - 1];
  }
}

/* equations.f90:434-502 calc_fluxes */
void orc_physical_flux(const orc_config *c, const double *q, int dir, double alpha,
                       const double *beta, const double *g, double sqg, double *f) {
  double v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]}, v_cov[3];
  double v_sq = capped_velocity(g, v, c->v_max);
  lower_index(g, v, v_cov);
  double v_norm, beta_norm;
  if (dir == DIR_X) { v_norm = v[0]; beta_norm = beta[0]; }
  else if (dir == DIR_Y) { v_norm = v[1]; beta_norm = beta[1]; }
  else { v_norm = v[2]; beta_norm = beta[2]; }
  double h = 1.0 + c->g1 * q[EQ_PR] / q[EQ_DE];
  double W = 1.0 / sqrt(1.0 - v_sq);
  double v_eff = alpha * v_norm - beta_norm;
  f[EQ_DE] = q[EQ_DE] * W * v_eff;
  f[EQ_PR] = q[EQ_DE] * h * (W * W) * v_eff + q[EQ_PR] * beta_norm - f[EQ_DE];
  f[EQ_VX] = q[EQ_DE] * h * (W * W) * v_cov[0] * v_eff + (dir == DIR_X ? alpha * q[EQ_PR] : 0.0);
  f[EQ_VY] = q[EQ_DE] * h * (W * W) * v_cov[1] * v_eff + (dir == DIR_Y ? alpha * q[EQ_PR] : 0.0);
  f[EQ_VZ] = q[EQ_DE] * h * (W * W) * v_cov[2] * v_eff + (dir == DIR_Z ? alpha * q[EQ_PR] : 0.0);
  for (int n = 0; n < NEQ; ++n) f[n] = f[n] * sqg;
}

/* fluxes.f90:76-122 prim_to_cons_face */
static void prim_to_cons_face(const orc_config *c, const double *q, double *u, const double *g,
                              double sqg) {
  double v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]}, v_cov[3];
  double v_sq = capped_velocity(g, v, c->v_max);
  lower_index(g, v, v_cov);
  double h = 1.0 + c->g1 * q[EQ_PR] / q[EQ_DE];
  double W = 1.0 / sqrt(1.0 - v_sq);
  u[EQ_DE] = q[EQ_DE] * W;
  u[EQ_PR] = q[EQ_DE] * h * (W * W) - q[EQ_PR] - q[EQ_DE] * W;
  u[EQ_VX] = q[EQ_DE] * h * (W * W) * v_cov[0];
  u[EQ_VY] = q[EQ_DE] * h * (W * W) * v_cov[1];
  u[EQ_VZ] = q[EQ_DE] * h * (W * W) * v_cov[2];
  for (int n = 0; n < NEQ; ++n) u[n] = u[n] * sqg;
}

/* fluxes.f90:669-720 calc_wavespeeds_srhd */
static void wavespeeds_srhd(const orc_config *c, const double *q, int dir, const double *g,
                            double *wmin, double *wmax) {
  double v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]};
  double v_sq = capped_velocity(g, v, c->v_max);
  double enthalpy = 1.0 + c->g1 * q[EQ_PR] / q[EQ_DE];
  double cs_sq = c->adb_idx * q[EQ_PR] / (q[EQ_DE] * enthalpy);
  double cs = sqrt(cs_sq);
  double v_norm = (dir == DIR_X) ? v[0] : (dir == DIR_Y ? v[1] : v[2]);
  double term1 = 1.0 / (1.0 - v_sq * cs_sq);
  double term2 = cs * sqrt((1.0 - v_sq) * (1.0 / term1 - (v_norm * v_norm) * (1.0 - cs_sq)));
  double eig1 = v_norm;
  double eig2 = term1 * (v_norm * (1.0 - cs_sq) + term2);
  double eig3 = term1 * (v_norm * (1.0 - cs_sq) - term2);
  *wmax = max4(0.0, eig1, eig2, eig3);
  *wmin = min4(0.0, eig1, eig2, eig3);
}

/* fluxes.f90:724-803 calc_wavespeeds_grhd (the n_steps==0 probe at :791-802 is
 * unreachable during evolution because n_steps is incremented first, grhd2.f90:229) */
static void wavespeeds_grhd(const orc_config *c, const double *q, int dir, double alpha,
                            const double *beta, const double *g, double *wmin, double *wmax) {
  double v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]};
  double v_sq = capped_velocity(g, v, c->v_max);
  double enthalpy = 1.0 + c->g1 * q[EQ_PR] / q[EQ_DE];
  double cs_sq = c->adb_idx * q[EQ_PR] / (q[EQ_DE] * enthalpy);
  double cs = sqrt(cs_sq);
  double det_g = G3(g, 1, 1) * (G3(g, 2, 2) * G3(g, 3, 3) - G3(g, 2, 3) * G3(g, 3, 2))
               - G3(g, 1, 2) * (G3(g, 2, 1) * G3(g, 3, 3) - G3(g, 2, 3) * G3(g, 3, 1))
               + G3(g, 1, 3) * (G3(g, 2, 1) * G3(g, 3, 2) - G3(g, 2, 2) * G3(g, 3, 1));
  double v_norm, beta_norm, gamma_up_ii;
  if (dir == DIR_X) {
    v_norm = v[0]; beta_norm = beta[0];
    gamma_up_ii = (G3(g, 2, 2) * G3(g, 3, 3) - G3(g, 2, 3) * G3(g, 3, 2)) / det_g;
  } else if (dir == DIR_Y) {
    v_norm = v[1]; beta_norm = beta[1];
    gamma_up_ii = (G3(g, 1, 1) * G3(g, 3, 3) - G3(g, 1, 3) * G3(g, 3, 1)) / det_g;
  } else {
    v_norm = v[2]; beta_norm = beta[2];
    gamma_up_ii = (G3(g, 1, 1) * G3(g, 2, 2) - G3(g, 1, 2) * G3(g, 2, 1)) / det_g;
  }
  double term1 = alpha / (1.0 - v_sq * cs_sq);
  double term2 = cs * sqrt(fmax_ref(0.0, (1.0 - v_sq) * (gamma_up_ii * (1.0 - v_sq * cs_sq) -
                                                         (v_norm * v_norm) * (1.0 - cs_sq))));
  double eig1 = alpha * v_norm - beta_norm;
  double eig2 = term1 * (v_norm * (1.0 - cs_sq) + term2) - beta_norm;
  double eig3 = term1 * (v_norm * (1.0 - cs_sq) - term2) - beta_norm;
  *wmax = max4(0.0, eig1, eig2, eig3);
  *wmin = min4(0.0, eig1, eig2, eig3);
}

static void wavespeeds(const orc_config *c, const double *q, int dir, double alpha,
                       const double *beta, const double *g, double *wmin, double *wmax) {
  /* fluxes.f90:44-50 init_wavespeed_solver: SRHD iff Minkowski + Cartesian */
  if (c->metric_kind == ORC_METRIC_MINKOWSKI && c->geom_kind == ORC_GEOM_CARTESIAN)
    wavespeeds_srhd(c, q, dir, g, wmin, wmax);
  else
    wavespeeds_grhd(c, q, dir, alpha, beta, g, wmin, wmax);
}

/* fluxes.f90:125-156 calc_hlle_fluxes */
static void hlle(const orc_config *c, const double *qL, const double *qR, int dir, double alpha,
                 const double *beta, const double *g, double sqg, double *flux) {
  double uL[NEQ], uR[NEQ], fL[NEQ], fR[NEQ];
  double lLmin, lLmax, lRmin, lRmax;
  orc_physical_flux(c, qL, dir, alpha, beta, g, sqg, fL);
  orc_physical_flux(c, qR, dir, alpha, beta, g, sqg, fR);
  prim_to_cons_face(c, qL, uL, g, sqg);
  prim_to_cons_face(c, qR, uR, g, sqg);
  wavespeeds(c, qL, dir, alpha, beta, g, &lLmin, &lLmax);
  wavespeeds(c, qR, dir, alpha, beta, g, &lRmin, &lRmax);
  double a_plus = max3(0.0, lLmax, lRmax);
  double a_minus = min3(0.0, lLmin, lRmin);
  if (fabs(a_plus - a_minus) < 1.0e-14) {
    for (int n = 0; n < NEQ; ++n) flux[n] = 0.0;
  } else {
    for (int n = 0; n < NEQ; ++n)
      flux[n] = (a_plus * fL[n] - a_minus * fR[n] + a_plus * a_minus * (uR[n] - uL[n])) / (a_plus - a_minus);
  }
}

/* fluxes.f90:476-487 metric_dot */
static double metric_dot(const double *a, const double *b, const double *g) {
  double s = 0.0;
  for (int i = 1; i <= 3; ++i)
    for (int j = 1; j <= 3; ++j) s = s + G3(g, i, j) * a[i - 1] * b[j - 1];
  return s;
}

/* fluxes.f90:402-473 build_face_orthonormal_frame. frame(:,a) = frame[3*a + i],
 * coframe(a,i) = cof[a + 3*i] (0-based a, i). */
static int face_frame(const double *g, int dir, double *frame, double *cof, double *gup) {
  int i, j, a;
  for (i = 0; i < 9; ++i) { frame[i] = 0.0; cof[i] = 0.0; }
  *gup = 0.0;
  for (i = 0; i < 9; ++i) if (!isfin(g[i])) return 0;
  double det_g = G3(g, 1, 1) * (G3(g, 2, 2) * G3(g, 3, 3) - G3(g, 2, 3) * G3(g, 3, 2))
               - G3(g, 1, 2) * (G3(g, 2, 1) * G3(g, 3, 3) - G3(g, 2, 3) * G3(g, 3, 1))
               + G3(g, 1, 3) * (G3(g, 2, 1) * G3(g, 3, 2) - G3(g, 2, 2) * G3(g, 3, 1));
  if (!isfin(det_g) || det_g <= 1.0e-30) return 0;
  double ginv[9];
#define GI(a, b) ginv[((a) - 1) + 3 * ((b) - 1)]
  GI(1, 1) = (G3(g, 2, 2) * G3(g, 3, 3) - G3(g, 2, 3) * G3(g, 3, 2)) / det_g;
  GI(1, 2) = (G3(g, 1, 3) * G3(g, 3, 2) - G3(g, 1, 2) * G3(g, 3, 3)) / det_g;
  GI(1, 3) = (G3(g, 1, 2) * G3(g, 2, 3) - G3(g, 1, 3) * G3(g, 2, 2)) / det_g;
  GI(2, 1) = (G3(g, 2, 3) * G3(g, 3, 1) - G3(g, 2, 1) * G3(g, 3, 3)) / det_g;
  GI(2, 2) = (G3(g, 1, 1) * G3(g, 3, 3) - G3(g, 1, 3) * G3(g, 3, 1)) / det_g;
  GI(2, 3) = (G3(g, 1, 3) * G3(g, 2, 1) - G3(g, 1, 1) * G3(g, 2, 3)) / det_g;
  GI(3, 1) = (G3(g, 2, 1) * G3(g, 3, 2) - G3(g, 2, 2) * G3(g, 3, 1)) / det_g;
  GI(3, 2) = (G3(g, 1, 2) * G3(g, 3, 1) - G3(g, 1, 1) * G3(g, 3, 2)) / det_g;
  GI(3, 3) = (G3(g, 1, 1) * G3(g, 2, 2) - G3(g, 1, 2) * G3(g, 2, 1)) / det_g;
  for (i = 0; i < 9; ++i) if (!isfin(ginv[i])) return 0;
  *gup = GI(dir, dir);
  if (*gup <= 1.0e-30 || !isfin(*gup)) return 0;
  for (i = 1; i <= 3; ++i) frame[0 * 3 + (i - 1)] = GI(i, dir) / sqrt(*gup);
#undef GI
  int tangent[2];
  if (dir == DIR_X) { tangent[0] = DIR_Y; tangent[1] = DIR_Z; }
  else if (dir == DIR_Y) { tangent[0] = DIR_Z; tangent[1] = DIR_X; }
  else if (dir == DIR_Z) { tangent[0] = DIR_X; tangent[1] = DIR_Y; }
  else return 0;
  for (int b = 2; b <= 3; ++b) {
    double seed[3] = {0.0, 0.0, 0.0};
    seed[tangent[b - 2] - 1] = 1.0;
    for (a = 1; a <= b - 1; ++a) {
      double projection = metric_dot(seed, &frame[3 * (a - 1)], g);
      for (i = 0; i < 3; ++i) seed[i] = seed[i] - projection * frame[3 * (a - 1) + i];
    }
    double norm_sq = metric_dot(seed, seed, g);
    if (!isfin(norm_sq) || norm_sq <= 1.0e-28) return 0;
    for (i = 0; i < 3; ++i) frame[3 * (b - 1) + i] = seed[i] / sqrt(norm_sq);
  }
  for (a = 1; a <= 3; ++a)
    for (i = 1; i <= 3; ++i)
      for (j = 1; j <= 3; ++j)
        cof[(a - 1) + 3 * (i - 1)] = cof[(a - 1) + 3 * (i - 1)] + G3(g, i, j) * frame[3 * (a - 1) + (j - 1)];
  for (i = 0; i < 9; ++i) if (!isfin(frame[i]) || !isfin(cof[i])) return 0;
  return 1;
}

/* fluxes.f90:490-504 primitives_to_local_frame */
static void to_local_frame(const double *q, const double *cof, double *ql) {
  for (int n = 0; n < NEQ; ++n) ql[n] = q[n];
  ql[EQ_VX] = 0.0; ql[EQ_VY] = 0.0; ql[EQ_VZ] = 0.0;
  for (int a = 1; a <= 3; ++a)
    for (int i = 1; i <= 3; ++i)
      ql[EQ_VX + a - 1] = ql[EQ_VX + a - 1] + cof[(a - 1) + 3 * (i - 1)] * q[EQ_VX + i - 1];
}

/* fluxes.f90:509-568 calc_srhd_local_state */
static int srhd_local_state(const orc_config *c, const double *ql, double *u, double *f,
                            double *wmin, double *wmax) {
  int n;
  for (n = 0; n < NEQ; ++n) { u[n] = 0.0; f[n] = 0.0; }
  *wmin = 0.0; *wmax = 0.0;
  double rho = ql[EQ_DE], pressure = ql[EQ_PR];
  double vel[3] = {ql[EQ_VX], ql[EQ_VY], ql[EQ_VZ]};
  if (!isfin(rho) || !isfin(pressure) || !isfin(vel[0]) || !isfin(vel[1]) || !isfin(vel[2]) ||
      rho <= 0.0 || pressure < 0.0) return 0;
  double v_sq = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
  if (!isfin(v_sq) || v_sq < 0.0) return 0;
  if (v_sq >= c->v_max) return 0;
  double h = 1.0 + c->g1 * pressure / rho;
  if (!isfin(h) || h <= 0.0) return 0;
  double cs_sq = c->adb_idx * pressure / (rho * h);
  if (!isfin(cs_sq) || cs_sq < 0.0 || cs_sq >= 1.0) return 0;
  double W = 1.0 / sqrt(1.0 - v_sq);
  double D = rho * W;
  double tau = rho * h * (W * W) - pressure - D;
  double mom[3];
  for (n = 0; n < 3; ++n) mom[n] = rho * h * (W * W) * vel[n];
  u[EQ_DE] = D; u[EQ_PR] = tau; u[EQ_VX] = mom[0]; u[EQ_VY] = mom[1]; u[EQ_VZ] = mom[2];
  f[EQ_DE] = D * vel[0];
  f[EQ_PR] = mom[0] - D * vel[0];
  f[EQ_VX] = mom[0] * vel[0] + pressure;
  f[EQ_VY] = mom[1] * vel[0];
  f[EQ_VZ] = mom[2] * vel[0];
  double denom = 1.0 - v_sq * cs_sq;
  double radicand = (1.0 - v_sq) * (1.0 - v_sq * cs_sq - (vel[0] * vel[0]) * (1.0 - cs_sq));
  if (denom <= 1.0e-14 || radicand < -1.0e-12) return 0;
  double acoustic = sqrt(cs_sq) * sqrt(fmax_ref(0.0, radicand));
  *wmin = (vel[0] * (1.0 - cs_sq) - acoustic) / denom;
  *wmax = (vel[0] * (1.0 - cs_sq) + acoustic) / denom;
  for (n = 0; n < NEQ; ++n) if (!isfin(u[n]) || !isfin(f[n])) return 0;
  if (!isfin(*wmin) || !isfin(*wmax)) return 0;
  return 1;
}

/* fluxes.f90:571-591 conservative_state_is_admissible */
static int admissible(const double *u) {
  for (int n = 0; n < NEQ; ++n) if (!isfin(u[n])) return 0;
  if (u[EQ_DE] <= 0.0) return 0;
  double E = u[EQ_PR] + u[EQ_DE];
  double msq = u[EQ_VX] * u[EQ_VX] + u[EQ_VY] * u[EQ_VY] + u[EQ_VZ] * u[EQ_VZ];
  double scale = max3(DBL_MIN, E * E, u[EQ_DE] * u[EQ_DE] + msq);
  if (E <= 0.0) return 0;
  if (E * E - u[EQ_DE] * u[EQ_DE] - msq <= 1.0e-13 * scale) return 0;
  return 1;
}

/* fluxes.f90:596-624 local_flux_to_coordinate */
static int local_flux_to_coordinate(const double *ul, const double *fl, double w, double alpha,
                                    double sqg, double gup, const double *cof, double *flux) {
  double mf[NEQ];
  int n, i, a;
  for (n = 0; n < NEQ; ++n) flux[n] = 0.0;
  for (n = 0; n < NEQ; ++n) mf[n] = fl[n] - w * ul[n];
  double factor = sqg * alpha * sqrt(gup);
  if (!isfin(factor)) return 0;
  for (n = 0; n < NEQ; ++n) if (!isfin(mf[n])) return 0;
  flux[EQ_DE] = factor * mf[EQ_DE];
  flux[EQ_PR] = factor * mf[EQ_PR];
  for (i = 1; i <= 3; ++i)
    for (a = 1; a <= 3; ++a)
      flux[EQ_VX + i - 1] = flux[EQ_VX + i - 1] + factor * cof[(a - 1) + 3 * (i - 1)] * mf[EQ_VX + a - 1];
  for (n = 0; n < NEQ; ++n) if (!isfin(flux[n])) return 0;
  return 1;
}

/* fluxes.f90:174-397 calc_hllc_fluxes (every exit to HLLE is counted) */
static void hllc(const orc_config *c, const double *qL, const double *qR, int dir, double alpha,
                 const double *beta, const double *g, double sqg, double *flux, orc_counters *cnt) {
  double qLh[NEQ], qRh[NEQ], uL[NEQ], uR[NEQ], fL[NEQ], fR[NEQ], uhll[NEQ], fhll[NEQ], pv[NEQ];
  double usL[NEQ], usR[NEQ], fsL[NEQ], fsR[NEQ];
  double frame[9], cof[9], gup;
  double lLmin, lLmax, lRmin, lRmax;
  int n;
#define FALLBACK do { if (cnt) cnt->hllc_fallbacks++; hlle(c, qL, qR, dir, alpha, beta, g, sqg, flux); return; } while (0)
  if (dir < DIR_X || dir > DIR_Z || alpha <= 0.0 || sqg <= 0.0 || !isfin(alpha) || !isfin(sqg)) FALLBACK;
  if (!face_frame(g, dir, frame, cof, &gup)) FALLBACK;
  to_local_frame(qL, cof, qLh);
  to_local_frame(qR, cof, qRh);
  if (!srhd_local_state(c, qLh, uL, fL, &lLmin, &lLmax)) FALLBACK;
  if (!srhd_local_state(c, qRh, uR, fR, &lRmin, &lRmax)) FALLBACK;
  double lambda_left = fmin_ref(lLmin, lRmin);
  double lambda_right = fmax_ref(lLmax, lRmax);
  double face_speed = beta[dir - 1] / (alpha * sqrt(gup));
  if (!isfin(face_speed) || lambda_right - lambda_left <= 1.0e-13) FALLBACK;
  if (face_speed <= lambda_left) {
    if (!local_flux_to_coordinate(uL, fL, face_speed, alpha, sqg, gup, cof, flux)) FALLBACK;
    return;
  } else if (face_speed >= lambda_right) {
    if (!local_flux_to_coordinate(uR, fR, face_speed, alpha, sqg, gup, cof, flux)) FALLBACK;
    return;
  }
  double denom = lambda_right - lambda_left;
  for (n = 0; n < NEQ; ++n) {
    uhll[n] = (lambda_right * uR[n] - lambda_left * uL[n] + fL[n] - fR[n]) / denom;
    fhll[n] = (lambda_right * fL[n] - lambda_left * fR[n] + lambda_right * lambda_left * (uR[n] - uL[n])) / denom;
  }
  for (n = 0; n < NEQ; ++n) if (!isfin(uhll[n]) || !isfin(fhll[n])) FALLBACK;
  double E_hll = uhll[EQ_PR] + uhll[EQ_DE];
  double FE_hll = fhll[EQ_PR] + fhll[EQ_DE];
  double M_hll = uhll[EQ_VX];
  double FM_hll = fhll[EQ_VX];
  double A_quad = FE_hll;
  double B_quad = -(E_hll + FM_hll);
  double C_quad = M_hll;
  double discriminant = B_quad * B_quad - 4.0 * A_quad * C_quad;
  double disc_scale = max3(DBL_MIN, B_quad * B_quad, fabs(4.0 * A_quad * C_quad));
  if (!isfin(discriminant) || discriminant < -1.0e-12 * disc_scale) FALLBACK;
  discriminant = fmax_ref(0.0, discriminant);
  double coefficient_scale = max3(DBL_MIN, fabs(B_quad), fabs(C_quad));
  int quadratic_case = fabs(A_quad) > 1.0e-13 * coefficient_scale;
  double lambda_star;
  if (!quadratic_case) {
    if (fabs(B_quad) <= 1.0e-14 * fmax_ref(DBL_MIN, fabs(C_quad))) FALLBACK;
    lambda_star = -C_quad / B_quad;
  } else {
    denom = -B_quad - sqrt(discriminant);
    if (fabs(denom) > 1.0e-14 * max3(DBL_MIN, fabs(B_quad), sqrt(discriminant))) {
      lambda_star = denom / (2.0 * A_quad);
    } else {
      denom = -B_quad + sqrt(discriminant);
      if (fabs(denom) <= 1.0e-14 * max3(DBL_MIN, fabs(B_quad), sqrt(discriminant))) FALLBACK;
      lambda_star = (2.0 * C_quad) / denom;
    }
  }
  double root_tol = 1.0e-10 * max3(1.0, fabs(lambda_left), fabs(lambda_right));
  int root_is_valid = isfin(lambda_star) && lambda_star >= lambda_left - root_tol &&
                      lambda_star <= lambda_right + root_tol && fabs(lambda_star) <= 1.0 + root_tol;
  if (!root_is_valid && quadratic_case) {
    double root_alt = (-B_quad + sqrt(discriminant)) / (2.0 * A_quad);
    if (isfin(root_alt) && root_alt >= lambda_left - root_tol && root_alt <= lambda_right + root_tol &&
        fabs(root_alt) <= 1.0 + root_tol) {
      lambda_star = root_alt;
      root_is_valid = 1;
    }
  }
  if (!root_is_valid) FALLBACK;
  lambda_star = fmin_ref(lambda_right, fmax_ref(lambda_left, lambda_star));
  double A_left = lambda_left * (uL[EQ_PR] + uL[EQ_DE]) - uL[EQ_VX];
  double B_left = uL[EQ_VX] * (lambda_left - qLh[EQ_VX]) - qLh[EQ_PR];
  double A_right = lambda_right * (uR[EQ_PR] + uR[EQ_DE]) - uR[EQ_VX];
  double B_right = uR[EQ_VX] * (lambda_right - qRh[EQ_VX]) - qRh[EQ_PR];
  denom = 1.0 - lambda_left * lambda_star;
  if (fabs(denom) <= 1.0e-13) FALLBACK;
  double p_star_left = (A_left * lambda_star - B_left) / denom;
  denom = 1.0 - lambda_right * lambda_star;
  if (fabs(denom) <= 1.0e-13) FALLBACK;
  double p_star_right = (A_right * lambda_star - B_right) / denom;
  double state_scale = max5(DBL_MIN, fabs(uL[EQ_PR] + uL[EQ_DE]), fabs(uR[EQ_PR] + uR[EQ_DE]),
                            fabs(uL[EQ_VX]), fabs(uR[EQ_VX]));
  double pressure_tolerance = 1.0e-8 * max5(DBL_MIN, fabs(qLh[EQ_PR]), fabs(qRh[EQ_PR]),
                                            fabs(p_star_left), fabs(p_star_right)) +
                              1.0e2 * DBL_EPSILON * state_scale;
  if (!isfin(p_star_left) || !isfin(p_star_right) ||
      fabs(p_star_left - p_star_right) > pressure_tolerance) FALLBACK;
  double p_star = 0.5 * (p_star_left + p_star_right);
  if (!isfin(p_star) || fabs(lambda_left - lambda_star) <= 1.0e-13 ||
      fabs(lambda_right - lambda_star) <= 1.0e-13) FALLBACK;
  for (n = 0; n < NEQ; ++n) pv[n] = 0.0;
  pv[EQ_PR] = lambda_star;
  pv[EQ_VX] = 1.0;
  for (n = 0; n < NEQ; ++n) {
    usL[n] = (lambda_left * uL[n] - fL[n] + p_star * pv[n]) / (lambda_left - lambda_star);
    usR[n] = (lambda_right * uR[n] - fR[n] + p_star * pv[n]) / (lambda_right - lambda_star);
  }
  for (n = 0; n < NEQ; ++n) {
    fsL[n] = fL[n] + lambda_left * (usL[n] - uL[n]);
    fsR[n] = fR[n] + lambda_right * (usR[n] - uR[n]);
  }
  if (!admissible(usL) || !admissible(usR)) FALLBACK;
  for (n = 0; n < NEQ; ++n) if (!isfin(fsL[n]) || !isfin(fsR[n])) FALLBACK;
  const double *usel = (face_speed <= lambda_star) ? usL : usR;
  const double *fsel = (face_speed <= lambda_star) ? fsL : fsR;
  if (!local_flux_to_coordinate(usel, fsel, face_speed, alpha, sqg, gup, cof, flux)) FALLBACK;
#undef FALLBACK
}

/* fluxes.f90:56-72 resolve_riemann_problem (HLLD is a stub in the reference: not ported) */
void orc_riemann(const orc_config *c, const double *qL, const double *qR, int dir,
                 double alpha, const double *beta, const double *g, double sqg,
                 double *flux, orc_counters *cnt) {
  if (c->riemann == ORC_RS_HLLC)
    hllc(c, qL, qR, dir, alpha, beta, g, sqg, flux, cnt);
  else
    hlle(c, qL, qR, dir, alpha, beta, g, sqg, flux);
}

/* ---------------------------------------------------------------------------------- */
/* equations.f90:509-552 calc_sources + metrics.f90:1251-1310 stress-energy tensor        */
/* ---------------------------------------------------------------------------------- */
static void calc_sources(const orc_config *c, const orc_metric *m, const double *prim, int i,
                         int j, double *src) {
  int n, mu, nu, d;
  for (n = 0; n < NEQ; ++n) src[n] = 0.0;
  if (c->metric_kind == ORC_METRIC_MINKOWSKI && c->geom_kind == ORC_GEOM_CARTESIAN) return;
  size_t cc = cell(c, i, j);
  double alpha = m->alpha_c[cc];
  double sqg = m->sqrt_gamma_c[cc];
  const double *chris = &m->chris_c[64 * cc];
  const double *dg = &m->dg_c[48 * cc];
  const double *dlna = &m->dlna_c[4 * cc];
  /* calculate_stress_energy_tensor */
  const double *beta = &m->beta_c[3 * cc];
  const double *g = &m->gamma_c[9 * cc];
  const double *gmunu = &m->gmunu_c[16 * cc];
  double v[3] = {prim[EQ_VX], prim[EQ_VY], prim[EQ_VZ]};
  double v_sq = capped_velocity(g, v, c->v_max);
  double h = 1.0 + c->g1 * prim[EQ_PR] / prim[EQ_DE];
  double W = 1.0 / sqrt(1.0 - v_sq);
  double uf[4];
  uf[0] = W / alpha;
  uf[1] = W * (v[0] - beta[0] / alpha);
  uf[2] = W * (v[1] - beta[1] / alpha);
  uf[3] = W * (v[2] - beta[2] / alpha);
  double T[16];
  for (mu = 0; mu <= 3; ++mu)
    for (nu = mu; nu <= 3; ++nu) {
      T[mu + 4 * nu] = (prim[EQ_DE] * h * uf[mu] * uf[nu]) + (prim[EQ_PR] * gmunu[mu + 4 * nu]);
      if (mu != nu) T[nu + 4 * mu] = T[mu + 4 * nu];
    }
  for (d = 1; d <= 3; ++d)
    for (mu = 0; mu <= 3; ++mu)
      for (nu = 0; nu <= 3; ++nu)
        src[EQ_VX + d - 1] = src[EQ_VX + d - 1] + 0.5 * T[mu + 4 * nu] * dg[mu + 4 * nu + 16 * (d - 1)];
  for (mu = 0; mu <= 3; ++mu) {
    src[EQ_PR] = src[EQ_PR] + T[mu + 4 * 0] * dlna[mu];
    for (nu = 0; nu <= 3; ++nu) src[EQ_PR] = src[EQ_PR] - T[mu + 4 * nu] * chris[0 + 4 * mu + 16 * nu];
  }
  for (n = 0; n < NEQ; ++n) src[n] = src[n] * alpha * sqg;
  src[EQ_PR] = src[EQ_PR] * alpha;
}

void orc_sources(const orc_config *c, const orc_metric *m, const double *prim, int i, int j, double *src) {
  calc_sources(c, m, prim, i, j, src);
}

/* ---------------------------------------------------------------------------------- */
/* evolution.f90:30-191 calc_rhs                                                        */
/* ---------------------------------------------------------------------------------- */
static void face_metric(const orc_config *c, const orc_metric *m, int dir, int i, int j,
                        double *a, double *b, double *g, double *sqg) {
  size_t f;
  const double *A, *B, *Gm, *S;
  if (dir == DIR_X) { f = (size_t)i + (size_t)(c->nx + 1) * (size_t)(j - 1); A = m->alpha_fx; B = m->beta_fx; Gm = m->gamma_fx; S = m->sqg_fx; }
  else if (dir == DIR_Y) { f = (size_t)(i - 1) + (size_t)c->nx * (size_t)j; A = m->alpha_fy; B = m->beta_fy; Gm = m->gamma_fy; S = m->sqg_fy; }
  else { f = (size_t)(i - 1) + (size_t)c->nx * (size_t)(j - 1); A = m->alpha_fz; B = m->beta_fz; Gm = m->gamma_fz; S = m->sqg_fz; }
  *a = A[f];
  for (int n = 0; n < 3; ++n) b[n] = B[3 * f + n];
  for (int n = 0; n < 9; ++n) g[n] = Gm[9 * f + n];
  *sqg = S[f];
}

static int is_polar(const orc_config *c) {
  return c->geom_kind == ORC_GEOM_SPHERICAL || c->geom_kind == ORC_GEOM_SPHEROIDAL;
}

void orc_calc_rhs(const orc_config *c, const orc_metric *m, const double *p, double *rhs,
                  orc_counters *cnt) {
  const int nx = c->nx, ny = c->ny, nz = c->nz, g = c->nghost;
  const lay_t L = mklay(c);
  const double eps64 = 64.0 * DBL_EPSILON;
  size_t total = (size_t)NEQ * nx * ny * nz;
  memset(rhs, 0, total * sizeof(double));

  /* 1. X sweep with sources (evolution.f90:48-94) */
#pragma omp parallel
  {
    orc_counters lc; memset(&lc, 0, sizeof lc);
    double *prim = (double *)malloc(sizeof(double) * NEQ * (nx + 2 * g + 1));
    double *qL = (double *)malloc(sizeof(double) * NEQ * (nx + 1));
    double *qR = (double *)malloc(sizeof(double) * NEQ * (nx + 1));
    double *fs = (double *)malloc(sizeof(double) * NEQ * (nx + 1));
    long strip;
#pragma omp for schedule(static)
    for (strip = 0; strip < (long)ny * nz; ++strip) {
      int j = (int)(strip % ny) + 1, k = (int)(strip / ny) + 1;
      for (int i = -g; i <= nx + g; ++i)
        for (int v = 0; v < NEQ; ++v) prim[v + NEQ * (i + g)] = p[pidx(&L, v, i, j, k)];
      orc_reconstruct(c, prim, nx, DIR_X, qL, qR, &lc);
      for (int i = 0; i <= nx; ++i) {
        if (c->geom_kind == ORC_GEOM_CYLINDRICAL && fabs(m->x_face[i]) <= eps64) {
          for (int v = 0; v < NEQ; ++v) fs[v + NEQ * i] = 0.0;
        } else {
          double a, b[3], gm[9], sqg;
          face_metric(c, m, DIR_X, i, j, &a, b, gm, &sqg);
          orc_riemann(c, &qL[NEQ * i], &qR[NEQ * i], DIR_X, a, b, gm, sqg, &fs[NEQ * i], &lc);
        }
      }
      for (int i = 1; i <= nx; ++i) {
        double src[NEQ], pc[NEQ];
        for (int v = 0; v < NEQ; ++v) pc[v] = p[pidx(&L, v, i, j, k)];
        calc_sources(c, m, pc, i, j, src);
        for (int v = 0; v < NEQ; ++v)
          rhs[uidx(c, v, i, j, k)] = -(fs[v + NEQ * i] - fs[v + NEQ * (i - 1)]) / c->dx + src[v];
      }
    }
    free(prim); free(qL); free(qR); free(fs);
#pragma omp critical
    add_counters(cnt, &lc);
  }

  /* 2. Y sweep (evolution.f90:100-146) */
  if (ny > 1) {
#pragma omp parallel
    {
      orc_counters lc; memset(&lc, 0, sizeof lc);
      double *prim = (double *)malloc(sizeof(double) * NEQ * (ny + 2 * g + 1));
      double *qL = (double *)malloc(sizeof(double) * NEQ * (ny + 1));
      double *qR = (double *)malloc(sizeof(double) * NEQ * (ny + 1));
      double *fs = (double *)malloc(sizeof(double) * NEQ * (ny + 1));
      long strip;
#pragma omp for schedule(static)
      for (strip = 0; strip < (long)nx * nz; ++strip) {
        int i = (int)(strip % nx) + 1, k = (int)(strip / nx) + 1;
        for (int j = -g; j <= ny + g; ++j)
          for (int v = 0; v < NEQ; ++v) prim[v + NEQ * (j + g)] = p[pidx(&L, v, i, j, k)];
        orc_reconstruct(c, prim, ny, DIR_Y, qL, qR, &lc);
        for (int j = 0; j <= ny; ++j) {
          if (is_polar(c) && fabs(sin(m->y_face[j])) <= eps64) {
            for (int v = 0; v < NEQ; ++v) fs[v + NEQ * j] = 0.0;
          } else {
            double a, b[3], gm[9], sqg;
            face_metric(c, m, DIR_Y, i, j, &a, b, gm, &sqg);
            orc_riemann(c, &qL[NEQ * j], &qR[NEQ * j], DIR_Y, a, b, gm, sqg, &fs[NEQ * j], &lc);
          }
        }
        for (int j = 1; j <= ny; ++j)
          for (int v = 0; v < NEQ; ++v)
            rhs[uidx(c, v, i, j, k)] = rhs[uidx(c, v, i, j, k)] - (fs[v + NEQ * j] - fs[v + NEQ * (j - 1)]) / c->dy;
      }
      free(prim); free(qL); free(qR); free(fs);
#pragma omp critical
      add_counters(cnt, &lc);
    }
  }

  /* 3. Z sweep (evolution.f90:152-189) */
  if (nz > 1) {
#pragma omp parallel
    {
      orc_counters lc; memset(&lc, 0, sizeof lc);
      double *prim = (double *)malloc(sizeof(double) * NEQ * (nz + 2 * g + 1));
      double *qL = (double *)malloc(sizeof(double) * NEQ * (nz + 1));
      double *qR = (double *)malloc(sizeof(double) * NEQ * (nz + 1));
      double *fs = (double *)malloc(sizeof(double) * NEQ * (nz + 1));
      long strip;
#pragma omp for schedule(static)
      for (strip = 0; strip < (long)nx * ny; ++strip) {
        int i = (int)(strip % nx) + 1, j = (int)(strip / nx) + 1;
        for (int k = -g; k <= nz + g; ++k)
          for (int v = 0; v < NEQ; ++v) prim[v + NEQ * (k + g)] = p[pidx(&L, v, i, j, k)];
        orc_reconstruct(c, prim, nz, DIR_Z, qL, qR, &lc);
        double a, b[3], gm[9], sqg;
        face_metric(c, m, DIR_Z, i, j, &a, b, gm, &sqg);
        for (int k = 0; k <= nz; ++k)
          orc_riemann(c, &qL[NEQ * k], &qR[NEQ * k], DIR_Z, a, b, gm, sqg, &fs[NEQ * k], &lc);
        for (int k = 1; k <= nz; ++k)
          for (int v = 0; v < NEQ; ++v)
            rhs[uidx(c, v, i, j, k)] = rhs[uidx(c, v, i, j, k)] - (fs[v + NEQ * k] - fs[v + NEQ * (k - 1)]) / c->dz;
      }
      free(prim); free(qL); free(qR); free(fs);
#pragma omp critical
      add_counters(cnt, &lc);
    }
  }
}

/* ---------------------------------------------------------------------------------- */
/* evolution.f90:198-275 update_adaptive_dt                                             */
/* ---------------------------------------------------------------------------------- */
int orc_cfl(const orc_config *c, const orc_metric *m, double *dt_out) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  if (!isfin(c->dx) || c->dx <= 0.0 || (ny > 1 && (!isfin(c->dy) || c->dy <= 0.0)) ||
      (nz > 1 && (!isfin(c->dz) || c->dz <= 0.0)))
    return -1;
  double max_vx = 0.0, max_vy = 0.0, max_vz = 0.0;
  long invalid = 0;
  /* the metric is k-invariant: every k repeats the same (i,j) values, so the maxima
   * over (i,j) equal the maxima over (i,j,k) */
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      size_t cc = cell(c, i, j);
      double alpha = m->alpha_c[cc];
      const double *beta = &m->beta_c[3 * cc];
      const double *ginv = &m->gamma_inv_c[9 * cc];
      if (!isfin(alpha) || alpha <= 0.0 || !isfin(beta[0]) || !isfin(beta[1]) || !isfin(beta[2]) ||
          !isfin(G3(ginv, 1, 1)) || G3(ginv, 1, 1) <= 0.0 ||
          (ny > 1 && (!isfin(G3(ginv, 2, 2)) || G3(ginv, 2, 2) <= 0.0)) ||
          (nz > 1 && (!isfin(G3(ginv, 3, 3)) || G3(ginv, 3, 3) <= 0.0))) {
        invalid += nz;
        continue;
      }
      max_vx = fmax_ref(max_vx, alpha * sqrt(G3(ginv, 1, 1)) + fabs(beta[0]));
      if (ny > 1) max_vy = fmax_ref(max_vy, alpha * sqrt(G3(ginv, 2, 2)) + fabs(beta[1]));
      if (nz > 1) max_vz = fmax_ref(max_vz, alpha * sqrt(G3(ginv, 3, 3)) + fabs(beta[2]));
    }
  if (invalid > 0) return -2;
  double inverse_dt = max_vx / c->dx;
  if (ny > 1) inverse_dt = inverse_dt + max_vy / c->dy;
  if (nz > 1) inverse_dt = inverse_dt + max_vz / c->dz;
  if (!isfin(inverse_dt) || inverse_dt <= 0.0) return -3;
  *dt_out = c->cfl / inverse_dt;
  return 0;
}

/* ---------------------------------------------------------------------------------- */
/* equations.f90:94-424 cons_to_prim, root_safe_newton, root_brent                     */
/* ---------------------------------------------------------------------------------- */
/* equations.f90:212-220 */
static void eval_V_and_dV(double g1, double W, const double *cs, double *V, double *dV) {
  double denom = g1 * (W * W) - 1.0;
  *V = (g1 * (W * W) * (cs[EQ_PR] + cs[EQ_DE]) - cs[EQ_DE] * W) / denom;
  *dV = (g1 * W * (cs[EQ_DE] * W - 2.0 * (cs[EQ_PR] + cs[EQ_DE])) + cs[EQ_DE]) / (denom * denom);
}
static double qsq(const double *ginv, const double *cs) {
  double s = 0.0;
  for (int ii = 1; ii <= 3; ++ii)
    for (int jj = 1; jj <= 3; ++jj) s = s + G3(ginv, ii, jj) * cs[EQ_VX + ii - 1] * cs[EQ_VX + jj - 1];
  return s;
}
/* equations.f90:223-246 */
static void eval_residual(double g1, double W, const double *cs, const double *ginv, double *res,
                          double *dres) {
  double V, dV;
  eval_V_and_dV(g1, W, cs, &V, &dV);
  double Q_sq = qsq(ginv, cs);
  double W3 = W * W * W;
  *res = (V * V) * (1.0 - 1.0 / (W * W)) - Q_sq;
  *dres = 2.0 * V * (dV * (W3 - W) + V) / W3;
}
/* equations.f90:343-424 root_brent (the reference's SAVE'd d,e are always written in the
 * first iteration before being read, so per-call locals give the same results) */
static double root_brent(const orc_config *c, const double *cs, const double *ginv) {
  const double EPS = 3.0e-8, x_acc = 1.0e-8, x1 = 1.0;
  double W_max_guess = (sqrt(qsq(ginv, cs)) + cs[EQ_DE]) / fmax_ref(cs[EQ_DE], c->rho_floor);
  double x2 = fmax_ref(1.0e4, W_max_guess * 2.0);
  double a, b, cc, d = 0.0, e = 0.0, fa, fb, fc, o, q, r, y1, tol1, xm, df;
  eval_residual(c->g1, x1, cs, ginv, &fa, &df);
  eval_residual(c->g1, x2, cs, ginv, &fb, &df);
  if (sgn1(fa) * sgn1(fb) > 0.0) return -1.0;
  a = x1; b = x2; cc = b; fc = fb;
  for (int iter = 1; iter <= 100; ++iter) {
    if (sgn1(fb) * sgn1(fc) > 0.0) { cc = a; fc = fa; d = b - a; e = d; }
    if (fabs(fc) < fabs(fb)) { a = b; b = cc; cc = a; fa = fb; fb = fc; fc = fa; }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * x_acc;
    xm = 0.5 * (cc - b);
    if (fabs(xm) <= tol1 || fabs(fb) < 1.0e-14) return b;
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      y1 = fb / fa;
      if (fabs(a - cc) < 1.0e-14) {
        o = 2.0 * xm * y1; q = 1.0 - y1;
      } else {
        q = fa / fc; r = fb / fc;
        o = y1 * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (y1 - 1.0);
      }
      if (o > 0.0) q = -q;
      o = fabs(o);
      if (2.0 * o < fmin_ref(3.0 * xm * q - fabs(tol1 * q), fabs(e * q))) { e = d; d = o / q; }
      else { d = xm; e = d; }
    } else {
      d = xm; e = d;
    }
    a = b; fa = fb;
    if (fabs(d) > tol1) b = b + d;
    else b = b + copysign(tol1, xm);
    eval_residual(c->g1, b, cs, ginv, &fb, &df);
  }
  return -1.0;
}
/* root_brent on its own, for the restatement cross-check (the Newton-bisection hybrid
 * rarely falls back to it) */
double orc_root_brent(const orc_config *c, const double *cs, const double *ginv) { return root_brent(c, cs, ginv); }

/* equations.f90:249-340 root_safe_newton; *brent set when the Brent fallback ran */
static double root_safe_newton(const orc_config *c, const double *cs, const double *ginv, int *brent) {
  const double x_acc = 1.0e-10, x1 = 1.0;
  double W_max_guess = (sqrt(qsq(ginv, cs)) + cs[EQ_DE]) / fmax_ref(cs[EQ_DE], c->rho_floor);
  double x2 = fmax_ref(1.0e3, W_max_guess * 2.0);
  double x_low = x1, x_high = x2, f_low, f_high, df, f, root, diff_x, diff_x_old, temp;
  int converged = 0;
  *brent = 0;
  eval_residual(c->g1, x1, cs, ginv, &f_low, &df);
  eval_residual(c->g1, x2, cs, ginv, &f_high, &df);
  if (fabs(f_low) < 1.0e-14) return x_low;
  else if (fabs(f_high) < 1.0e-14) return x_high;
  else if (sgn1(f_low) * sgn1(f_high) > 0.0) return -1.0;
  if (f_low < 0.0) { x_low = x1; x_high = x2; }
  else { x_high = x1; x_low = x2; }
  root = 0.5 * (x1 + x2);
  diff_x_old = fabs(x2 - x1);
  diff_x = diff_x_old;
  eval_residual(c->g1, root, cs, ginv, &f, &df);
  for (int iter = 1; iter <= 100; ++iter) {
    if (((root - x_high) * df - f) * ((root - x_low) * df - f) > 0.0 ||
        fabs(2.0 * f) > fabs(diff_x_old * df)) {
      diff_x_old = diff_x;
      diff_x = 0.5 * (x_high - x_low);
      root = x_low + diff_x;
      if (fabs(x_low - root) < 1.0e-14) return root;
    } else {
      diff_x_old = diff_x;
      diff_x = f / df;
      temp = root;
      root = root - diff_x;
      if (fabs(temp - root) < 1.0e-14) return root;
    }
    if (fabs(diff_x) < x_acc) { converged = 1; return root; }
    eval_residual(c->g1, root, cs, ginv, &f, &df);
    if (f < 0.0) x_low = root; else x_high = root;
  }
  if (!converged || fabs(f) > 1.0e-6) { *brent = 1; root = root_brent(c, cs, ginv); }
  return root;
}

static void set_floor_state(double *prim, double *cons, double lDf, double lTf,
                            double rho_floor, double p_floor) {
  prim[EQ_DE] = rho_floor; prim[EQ_PR] = p_floor;
  prim[EQ_VX] = 0.0; prim[EQ_VY] = 0.0; prim[EQ_VZ] = 0.0;
  cons[EQ_DE] = lDf; cons[EQ_PR] = lTf;
  cons[EQ_VX] = 0.0; cons[EQ_VY] = 0.0; cons[EQ_VZ] = 0.0;
}

void orc_cons_to_prim(const orc_config *c, const orc_metric *m, double *cons, double *prim,
                      int i, int j, orc_counters *cnt) {
  size_t cc = cell(c, i, j);
  const double *g = &m->gamma_c[9 * cc];
  const double *ginv = &m->gamma_inv_c[9 * cc];
  double sqg = m->sqrt_gamma_c[cc];
  double lDf = c->rho_floor * sqg;
  double lTf = c->p_floor * (c->g1 - 1.0) * sqg;
  if (cons[EQ_DE] <= lDf) {
    if (cnt) cnt->c2p_floor_pre++;
    set_floor_state(prim, cons, lDf, lTf, c->rho_floor, c->p_floor);
    return;
  }
  double S1 = cons[EQ_VX], S2 = cons[EQ_VY], S3 = cons[EQ_VZ];
  double S_sq = S1 * (G3(ginv, 1, 1) * S1 + G3(ginv, 1, 2) * S2 + G3(ginv, 1, 3) * S3)
              + S2 * (G3(ginv, 2, 1) * S1 + G3(ginv, 2, 2) * S2 + G3(ginv, 2, 3) * S3)
              + S3 * (G3(ginv, 3, 1) * S1 + G3(ginv, 3, 2) * S2 + G3(ginv, 3, 3) * S3);
  double E_tot = cons[EQ_PR] + cons[EQ_DE];
  double S_sq_max = fmax_ref(0.0, E_tot * E_tot - cons[EQ_DE] * cons[EQ_DE]) * c->v_max;
  if (S_sq > S_sq_max && S_sq > 1.0e-20) {
    if (cnt) cnt->c2p_causal_rescale++;
    double sf = sqrt(S_sq_max / S_sq);
    cons[EQ_VX] = cons[EQ_VX] * sf;
    cons[EQ_VY] = cons[EQ_VY] * sf;
    cons[EQ_VZ] = cons[EQ_VZ] * sf;
  }
  int brent;
  double W = root_safe_newton(c, cons, ginv, &brent);
  if (brent && cnt) cnt->c2p_brent_used++;
  if (W < 1.0) {
    if (cnt) cnt->c2p_root_fail++;
    set_floor_state(prim, cons, lDf, lTf, c->rho_floor, c->p_floor);
    return;
  }
  double V, dV;
  eval_V_and_dV(c->g1, W, cons, &V, &dV);
  if (V <= 0.0 || isnan(V)) {
    if (cnt) cnt->c2p_bad_V++;
    set_floor_state(prim, cons, lDf, lTf, c->rho_floor, c->p_floor);
    return;
  }
  prim[EQ_DE] = cons[EQ_DE] / (W * sqg);
  prim[EQ_PR] = (V - cons[EQ_PR] - cons[EQ_DE]) / sqg;
  prim[EQ_VX] = (G3(ginv, 1, 1) * cons[EQ_VX] + G3(ginv, 1, 2) * cons[EQ_VY] + G3(ginv, 1, 3) * cons[EQ_VZ]) / V;
  prim[EQ_VY] = (G3(ginv, 2, 1) * cons[EQ_VX] + G3(ginv, 2, 2) * cons[EQ_VY] + G3(ginv, 2, 3) * cons[EQ_VZ]) / V;
  prim[EQ_VZ] = (G3(ginv, 3, 1) * cons[EQ_VX] + G3(ginv, 3, 2) * cons[EQ_VY] + G3(ginv, 3, 3) * cons[EQ_VZ]) / V;
  double vsf = 0.0;
  for (int ii = 1; ii <= 3; ++ii)
    for (int jj = 1; jj <= 3; ++jj) vsf = vsf + G3(g, ii, jj) * prim[EQ_VX + ii - 1] * prim[EQ_VX + jj - 1];
  if (prim[EQ_DE] < c->rho_floor || prim[EQ_PR] < c->p_floor || isnan(prim[EQ_DE]) ||
      isnan(prim[EQ_PR]) || isnan(prim[EQ_VX]) || isnan(prim[EQ_VY]) || isnan(prim[EQ_VZ]) ||
      isnan(vsf) || vsf >= c->v_max) {
    if (cnt) cnt->c2p_final_sanitise++;
    set_floor_state(prim, cons, lDf, lTf, c->rho_floor, c->p_floor);
  }
}

void orc_cons_to_prim_all(const orc_config *c, const orc_metric *m, double *up, double *p,
                          orc_counters *cnt) {
  const lay_t L = mklay(c);
  const long ncell = (long)c->nx * c->ny * c->nz;
#pragma omp parallel
  {
    orc_counters lc; memset(&lc, 0, sizeof lc);
    long n;
#pragma omp for schedule(static)
    for (n = 0; n < ncell; ++n) {
      int i = (int)(n % c->nx) + 1, j = (int)((n / c->nx) % c->ny) + 1, k = (int)(n / ((long)c->nx * c->ny)) + 1;
      double pr[NEQ];
      orc_cons_to_prim(c, m, &up[uidx(c, 0, i, j, k)], pr, i, j, &lc);
      for (int v = 0; v < NEQ; ++v) p[pidx(&L, v, i, j, k)] = pr[v];
    }
#pragma omp critical
    add_counters(cnt, &lc);
  }
}

/* equations.f90:30-88 prim_to_cons */
void orc_prim_to_cons(const orc_config *c, const orc_metric *m, const double *prim,
                      double *cons, int i, int j) {
  size_t cc = cell(c, i, j);
  const double *g = &m->gamma_c[9 * cc];
  double sqg = m->sqrt_gamma_c[cc];
  double v[3] = {prim[EQ_VX], prim[EQ_VY], prim[EQ_VZ]}, v_cov[3];
  double v_sq = capped_velocity(g, v, c->v_max);
  lower_index(g, v, v_cov);
  double h = 1.0 + c->g1 * prim[EQ_PR] / prim[EQ_DE];
  double W = 1.0 / sqrt(1.0 - v_sq);
  cons[EQ_DE] = prim[EQ_DE] * W;
  cons[EQ_PR] = prim[EQ_DE] * h * (W * W) - prim[EQ_PR] - prim[EQ_DE] * W;
  cons[EQ_VX] = prim[EQ_DE] * h * (W * W) * v_cov[0];
  cons[EQ_VY] = prim[EQ_DE] * h * (W * W) * v_cov[1];
  cons[EQ_VZ] = prim[EQ_DE] * h * (W * W) * v_cov[2];
  for (int n = 0; n < NEQ; ++n) cons[n] = cons[n] * sqg;
}

void orc_prim_to_cons_all(const orc_config *c, const orc_metric *m, const double *p,
                          double *up) {
  const lay_t L = mklay(c);
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i) {
        double pr[NEQ];
        for (int v = 0; v < NEQ; ++v) pr[v] = p[pidx(&L, v, i, j, k)];
        orc_prim_to_cons(c, m, pr, &up[uidx(c, 0, i, j, k)], i, j);
      }
}

/* ---------------------------------------------------------------------------------- */
/* conditions.f90:773-1066 set_boundary_conditions (whole-array semantics, corners      */
/* included, in the reference's statement order)                                        */
/* ---------------------------------------------------------------------------------- */
static void copy_cell(const lay_t *L, double *p, int i, int j, int k, int si, int sj, int sk) {
  for (int v = 0; v < NEQ; ++v) p[pidx(L, v, i, j, k)] = p[pidx(L, v, si, sj, sk)];
}
/* q(:,:,1-g,:) = q(:,:,ny+1-g,:); q(:,:,ny+g,:) = q(:,:,g,:) ; same for z, interleaved per g */
static void periodic_yz(const lay_t *L, double *p) {
  const int g0 = L->g;
  for (int g = 1; g <= g0; ++g) {
    for (int k = -g0; k <= L->nz + g0; ++k)
      for (int i = -g0; i <= L->nx + g0; ++i) copy_cell(L, p, i, 1 - g, k, i, L->ny + 1 - g, k);
    for (int k = -g0; k <= L->nz + g0; ++k)
      for (int i = -g0; i <= L->nx + g0; ++i) copy_cell(L, p, i, L->ny + g, k, i, g, k);
    for (int j = -g0; j <= L->ny + g0; ++j)
      for (int i = -g0; i <= L->nx + g0; ++i) copy_cell(L, p, i, j, 1 - g, i, j, L->nz + 1 - g);
    for (int j = -g0; j <= L->ny + g0; ++j)
      for (int i = -g0; i <= L->nx + g0; ++i) copy_cell(L, p, i, j, L->nz + g, i, j, g);
  }
}
static void periodic_z(const lay_t *L, double *p) {
  const int g0 = L->g;
  for (int g = 1; g <= g0; ++g) {
    for (int j = -g0; j <= L->ny + g0; ++j)
      for (int i = -g0; i <= L->nx + g0; ++i) copy_cell(L, p, i, j, 1 - g, i, j, L->nz + 1 - g);
    for (int j = -g0; j <= L->ny + g0; ++j)
      for (int i = -g0; i <= L->nx + g0; ++i) copy_cell(L, p, i, j, L->nz + g, i, j, g);
  }
}

int orc_set_boundary(const orc_config *c, const orc_metric *m, double *p) {
  const lay_t Ls = mklay(c), *L = &Ls;
  const int nx = c->nx, ny = c->ny, nz = c->nz, g0 = c->nghost;
  const double rf = c->rho_floor, pf = c->p_floor;
  int g, i, j, k;
#define Q(v, a, b, cc) p[pidx(L, v, a, b, cc)]
  switch (c->case_id) {
  case 1: case 2: case 3: /* conditions.f90:794-806 */
    for (g = 1; g <= g0; ++g)
      for (k = -g0; k <= nz + g0; ++k)
        for (j = -g0; j <= ny + g0; ++j) {
          copy_cell(L, p, 1 - g, j, k, 1, j, k);
          copy_cell(L, p, nx + g, j, k, nx, j, k);
        }
    periodic_yz(L, p);
    break;
  case 4: case 6: /* conditions.f90:808-818 */
    for (g = 1; g <= g0; ++g) {
      for (k = -g0; k <= nz + g0; ++k)
        for (j = -g0; j <= ny + g0; ++j) copy_cell(L, p, 1 - g, j, k, nx + 1 - g, j, k);
      for (k = -g0; k <= nz + g0; ++k)
        for (j = -g0; j <= ny + g0; ++j) copy_cell(L, p, nx + g, j, k, g, j, k);
      for (k = -g0; k <= nz + g0; ++k)
        for (i = -g0; i <= nx + g0; ++i) copy_cell(L, p, i, 1 - g, k, i, ny + 1 - g, k);
      for (k = -g0; k <= nz + g0; ++k)
        for (i = -g0; i <= nx + g0; ++i) copy_cell(L, p, i, ny + g, k, i, g, k);
      for (j = -g0; j <= ny + g0; ++j)
        for (i = -g0; i <= nx + g0; ++i) copy_cell(L, p, i, j, 1 - g, i, j, nz + 1 - g);
      for (j = -g0; j <= ny + g0; ++j)
        for (i = -g0; i <= nx + g0; ++i) copy_cell(L, p, i, j, nz + g, i, j, g);
    }
    break;
  case 5: { /* conditions.f90:820-870 */
    const double amb_rho = m->jet[0], amb_p = m->jet[1], amb_v = m->jet[2];
    const double noz_r = m->jet[3], jet_rho = m->jet[4], jet_p = m->jet[5], jet_v = m->jet[6];
    for (k = -g0; k <= nz + g0; ++k)
      for (j = -g0; j <= ny + g0; ++j)
        for (i = -g0; i <= nx + g0; ++i)
          if (i < 1 || i > nx || j < 1 || j > ny || k < 1 || k > nz) {
            Q(EQ_DE, i, j, k) = amb_rho; Q(EQ_PR, i, j, k) = amb_p;
            Q(EQ_VX, i, j, k) = 0.0; Q(EQ_VY, i, j, k) = 0.0; Q(EQ_VZ, i, j, k) = 0.0;
            Q(EQ_VZ, i, j, k) = amb_v;
          }
    for (k = -g0; k <= nz + g0; ++k)
      for (j = -g0; j <= ny + g0; ++j)
        for (g = 1; g <= g0; ++g) {
          copy_cell(L, p, 1 - g, j, k, g, j, k);
          Q(EQ_VX, 1 - g, j, k) = -Q(EQ_VX, g, j, k);
        }
    for (j = -g0; j <= ny + g0; ++j)
      for (i = -g0; i <= nx + g0; ++i)
        for (g = 1; g <= g0; ++g) {
          copy_cell(L, p, i, j, nz + g, i, j, nz);
          Q(EQ_VZ, i, j, nz + g) = fmax_ref(0.0, Q(EQ_VZ, i, j, nz));
          if (m->x_c[i + g0] <= noz_r) {
            Q(EQ_DE, i, j, 1 - g) = jet_rho; Q(EQ_PR, i, j, 1 - g) = jet_p;
            Q(EQ_VX, i, j, 1 - g) = 0.0; Q(EQ_VY, i, j, 1 - g) = 0.0;
            Q(EQ_VZ, i, j, 1 - g) = jet_v;
          } else {
            copy_cell(L, p, i, j, 1 - g, i, j, g);
            Q(EQ_VZ, i, j, 1 - g) = -Q(EQ_VZ, i, j, g);
          }
        }
    break;
  }
  case 7: /* conditions.f90:872-891 */
    for (k = 1; k <= nz; ++k)
      for (j = 1; j <= ny; ++j)
        for (g = 1; g <= g0; ++g) {
          copy_cell(L, p, 1 - g, j, k, 1, j, k);
          for (int v = 0; v < NEQ; ++v)
            Q(v, nx + g, j, k) = m->michel_injector[v + NEQ * ((g - 1) + (size_t)g0 * ((j - 1) + (size_t)ny * (k - 1)))];
        }
    periodic_yz(L, p);
    break;
  case 8: /* conditions.f90:893-914 */
    for (g = 1; g <= g0; ++g)
      for (k = 1; k <= nz; ++k)
        for (j = 1; j <= ny; ++j) {
          copy_cell(L, p, 1 - g, j, k, 1, j, k);
          Q(EQ_DE, 1 - g, j, k) = fmax_ref(Q(EQ_DE, 1, j, k), rf);
          Q(EQ_PR, 1 - g, j, k) = fmax_ref(Q(EQ_PR, 1, j, k), pf);
          Q(EQ_VX, 1 - g, j, k) = fmin_ref(0.0, Q(EQ_VX, 1, j, k));
          for (int v = 0; v < NEQ; ++v) Q(v, nx + g, j, k) = m->dust_outer[v + NEQ * (g - 1)];
        }
    periodic_yz(L, p);
    break;
  case 9: case 10: /* conditions.f90:916-947 */
    for (k = 1; k <= nz; ++k)
      for (j = 1; j <= ny; ++j) {
        size_t c1 = cell(c, 1, j), cn = cell(c, nx, j);
        for (g = 1; g <= g0; ++g) {
          copy_cell(L, p, 1 - g, j, k, 1, j, k);
          Q(EQ_DE, 1 - g, j, k) = fmax_ref(Q(EQ_DE, 1, j, k), rf);
          Q(EQ_PR, 1 - g, j, k) = fmax_ref(Q(EQ_PR, 1, j, k), pf);
          Q(EQ_VX, 1 - g, j, k) = fmin_ref(m->beta_c[3 * c1] / m->alpha_c[c1], Q(EQ_VX, 1, j, k));
          if (Q(EQ_DE, 1, j, k) < 1.0e-6) { Q(EQ_VY, 1 - g, j, k) = 0.0; Q(EQ_VZ, 1 - g, j, k) = 0.0; }
          Q(EQ_DE, nx + g, j, k) = fmax_ref(Q(EQ_DE, nx, j, k), rf);
          Q(EQ_PR, nx + g, j, k) = fmax_ref(Q(EQ_PR, nx, j, k), pf);
          Q(EQ_VX, nx + g, j, k) = fmax_ref(m->beta_c[3 * cn] / m->alpha_c[cn], Q(EQ_VX, nx, j, k));
          Q(EQ_VY, nx + g, j, k) = Q(EQ_VY, nx, j, k);
          Q(EQ_VZ, nx + g, j, k) = Q(EQ_VZ, nx, j, k);
        }
      }
    periodic_yz(L, p);
    break;
  case 11: case 12: { /* conditions.f90:949-1059 */
    if (c->case_id == 12 && (nz % 2) != 0) return -10;
    for (k = 1; k <= nz; ++k)
      for (j = 1; j <= ny; ++j) {
        size_t c1 = cell(c, 1, j), cn = cell(c, nx, j);
        for (g = 1; g <= g0; ++g) {
          copy_cell(L, p, 1 - g, j, k, 1, j, k);
          Q(EQ_DE, 1 - g, j, k) = fmax_ref(Q(EQ_DE, 1, j, k), rf);
          Q(EQ_PR, 1 - g, j, k) = fmax_ref(Q(EQ_PR, 1, j, k), pf);
          Q(EQ_VX, 1 - g, j, k) = fmin_ref(m->beta_c[3 * c1] / m->alpha_c[c1], Q(EQ_VX, 1, j, k));
          copy_cell(L, p, nx + g, j, k, nx, j, k);
          Q(EQ_DE, nx + g, j, k) = fmax_ref(Q(EQ_DE, nx, j, k), rf);
          Q(EQ_PR, nx + g, j, k) = fmax_ref(Q(EQ_PR, nx, j, k), pf);
          Q(EQ_VX, nx + g, j, k) = fmax_ref(m->beta_c[3 * cn] / m->alpha_c[cn], Q(EQ_VX, nx, j, k));
        }
      }
    for (k = 1; k <= nz; ++k) {
      int ks = k;
      if (c->case_id == 12) { ks = k + nz / 2; if (ks > nz) ks = ks - nz; }
      for (i = -g0; i <= nx + g0; ++i)
        for (g = 1; g <= g0; ++g) {
          copy_cell(L, p, i, 1 - g, k, i, g, ks);
          Q(EQ_VY, i, 1 - g, k) = -Q(EQ_VY, i, g, ks);
          if (c->case_id == 12) Q(EQ_VZ, i, 1 - g, k) = Q(EQ_VZ, i, g, ks);
          copy_cell(L, p, i, ny + g, k, i, ny + 1 - g, ks);
          Q(EQ_VY, i, ny + g, k) = -Q(EQ_VY, i, ny + 1 - g, ks);
          if (c->case_id == 12) Q(EQ_VZ, i, ny + g, k) = Q(EQ_VZ, i, ny + 1 - g, ks);
        }
    }
    periodic_z(L, p);
    break;
  }
  default:
    return -11;
  }
#undef Q
  return 0;
}

/* ---------------------------------------------------------------------------------- */
/* grhd2.f90:232-265 SSP-RK3 step, grhd2.f90:179-230 loop                               */
/* ---------------------------------------------------------------------------------- */
int orc_step(const orc_config *c, const orc_metric *m, double *u, double *up, double *p,
             double *rhs, double dt, orc_counters *cnt) {
  const long n = (long)NEQ * c->nx * c->ny * c->nz;
  long q;
  int rc;
  memcpy(u, up, sizeof(double) * (size_t)n);
  if ((rc = orc_set_boundary(c, m, p)) != 0) return rc;
  for (int rk = 1; rk <= 3; ++rk) {
    orc_calc_rhs(c, m, p, rhs, cnt);
    if (rk == 1) {
#pragma omp parallel for schedule(static)
      for (q = 0; q < n; ++q) up[q] = u[q] + rhs[q] * dt;
    } else if (rk == 2) {
#pragma omp parallel for schedule(static)
      for (q = 0; q < n; ++q) up[q] = 0.75 * u[q] + 0.25 * (up[q] + rhs[q] * dt);
    } else {
#pragma omp parallel for schedule(static)
      for (q = 0; q < n; ++q) up[q] = (u[q] + 2.0 * (up[q] + rhs[q] * dt)) / 3.0;
    }
    orc_cons_to_prim_all(c, m, up, p, cnt);
    if ((rc = orc_set_boundary(c, m, p)) != 0) return rc;
  }
  return 0;
}

int64_t orc_run(const orc_config *c, const orc_metric *m, double *up, double *p,
                double t0, double final_time, int64_t max_steps, double *t_out,
                orc_counters *cnt) {
  const size_t n = (size_t)NEQ * c->nx * c->ny * c->nz;
  double *u = (double *)malloc(sizeof(double) * n);
  double *rhs = (double *)malloc(sizeof(double) * n);
  double t = t0, dt;
  int64_t steps = 0;
  int rc = 0;
  if (!u || !rhs) { free(u); free(rhs); return -20; }
  while (t < final_time && (max_steps < 0 || steps < max_steps)) {
    if ((rc = orc_cfl(c, m, &dt)) != 0) break;
    if (t + dt > final_time) dt = final_time - t;
    steps++;
    t = t + dt;
    if ((rc = orc_step(c, m, u, up, p, rhs, dt, cnt)) != 0) break;
  }
  free(u); free(rhs);
  if (t_out) *t_out = t;
  return rc ? (int64_t)rc : steps;
}


/* ------------------------------------------------------------------------------------
 * Diagnostics: grhd2.f90:283-301 and output.f90:951-1125
 * ------------------------------------------------------------------------------------ */
double orc_total_mass(const orc_config *c, const double *u) {
  double total = 0.0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i) total = total + u[uidx(c, 0, i, j, k)] * c->dx * c->dy * c->dz;
  return total;
}

int orc_mdot(const orc_config *c, const orc_metric *m, const double *up, const double *p, int idx_probe,
             double *out) {
  if (idx_probe < 1 || idx_probe > c->nx) return -1; /* output.f90:959-962 */
  const lay_t L = mklay(c);
  double m_dot = 0.0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j) {
      const size_t q = cell(c, idx_probe, j);
      const double alpha = m->alpha_c[q];
      const double beta1 = m->beta_c[3 * q];
      const double v_eff = alpha * p[pidx(&L, 2, idx_probe, j, k)] - beta1;
      m_dot = m_dot + up[uidx(c, 0, idx_probe, j, k)] * v_eff * c->dy * c->dz;
    }
  *out = -m_dot;
  return 0;
}

void orc_ppi_modes(const orc_config *c, const double *up, const double *p, const double *z, double *values) {
  enum { MAXM = 4 };
  const lay_t L = mklay(c);
  for (int q = 0; q < 1 + 4 * MAXM; ++q) values[q] = 0.0;
  if (c->nz < 2) return; /* output.f90:1005 */
  const double cell_volume = c->dx * c->dy * c->dz;
  const double density_cut = 1.0e3 * c->rho_floor;
  double c0 = 0.0, cr[MAXM] = {0, 0, 0, 0}, ci[MAXM] = {0, 0, 0, 0};
  for (int k = 1; k <= c->nz; ++k) {
    double am = 0.0;
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i)
        if (p[pidx(&L, 0, i, j, k)] > density_cut) am = am + up[uidx(c, 0, i, j, k)] * cell_volume;
    c0 = c0 + am;
    for (int mm = 1; mm <= MAXM; ++mm) {
      cr[mm - 1] = cr[mm - 1] + am * cos((double)mm * z[k - 1]);
      ci[mm - 1] = ci[mm - 1] - am * sin((double)mm * z[k - 1]);
    }
  }
  values[0] = c0;
  for (int mm = 1; mm <= MAXM; ++mm) {
    double *v = values + 1 + 4 * (mm - 1);
    v[0] = cr[mm - 1];
    v[1] = ci[mm - 1];
    if (c0 > DBL_MIN) {
      v[2] = sqrt(cr[mm - 1] * cr[mm - 1] + ci[mm - 1] * ci[mm - 1]) / c0;
      v[3] = -atan2(ci[mm - 1], cr[mm - 1]) / (double)mm;
    }
  }
}

void orc_global_diagnostics(const orc_config *c, const orc_metric *m, const double *up, const double *p,
                            double *f, int64_t *n) {
  const lay_t L = mklay(c);
  const double cell_volume = c->dx * c->dy * c->dz;
  const double density_cut = 1.0e3 * c->rho_floor;
  double mass_total = 0.0, disk_mass = 0.0, angmom = 0.0;
  double rmin = DBL_MAX, pmin = DBL_MAX, rmax_ = -DBL_MAX, pmax = -DBL_MAX, vmax = 0.0;
  int64_t atmosphere = 0, invalid = 0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i) {
        const double rho = p[pidx(&L, 0, i, j, k)];
        const double pres = p[pidx(&L, 1, i, j, k)];
        const double *g = &m->gamma_c[9 * cell(c, i, j)];
        double v_sq = 0.0;
        for (int ii = 1; ii <= 3; ++ii)
          for (int jj = 1; jj <= 3; ++jj)
            v_sq = v_sq + G3(g, ii, jj) * p[pidx(&L, 1 + ii, i, j, k)] * p[pidx(&L, 1 + jj, i, j, k)];
        if (!isfinite(rho) || !isfinite(pres) || !isfinite(v_sq) || rho <= 0.0 || pres <= 0.0 || v_sq < 0.0 ||
            v_sq >= 1.0)
          invalid++;
        if (isfinite(rho)) {
          if (rho < rmin) rmin = rho;
          if (rho > rmax_) rmax_ = rho;
        }
        if (isfinite(pres)) {
          if (pres < pmin) pmin = pres;
          if (pres > pmax) pmax = pres;
        }
        if (isfinite(v_sq) && v_sq > vmax) vmax = v_sq;
        mass_total = mass_total + up[uidx(c, 0, i, j, k)] * cell_volume;
        angmom = angmom + up[uidx(c, 4, i, j, k)] * cell_volume;
        if (rho > density_cut) disk_mass = disk_mass + up[uidx(c, 0, i, j, k)] * cell_volume;
        else atmosphere++;
      }
  f[0] = mass_total; f[1] = disk_mass; f[2] = angmom;
  f[3] = rmin; f[4] = pmin; f[5] = rmax_; f[6] = pmax; f[7] = vmax;
  n[0] = atmosphere; n[1] = invalid;
}

/* metrics.f90:66-87 */
int orc_horizon_radius(double mass, double spin, double *r_plus) {
  if (mass < 0.0) return -1;
  double big = 1.0;
  if (mass * mass > big) big = mass * mass;
  if (spin * spin > big) big = spin * spin;
  const double tol = 64.0 * DBL_EPSILON * big;
  const double disc = mass * mass - spin * spin;
  if (disc < -tol) return -1;
  *r_plus = mass + sqrt(disc > 0.0 ? disc : 0.0);
  return 0;
}

/* output.f90:743-768 kerr_schild_spheroidal_position, with sin/cos of theta and phi given */
static void ks_position(double r, double st, double ct, double sp, double cp, double spin, double *pos) {
  if (fabs(st) <= 64.0 * DBL_EPSILON) {  /* both poles collapse exactly onto the axis */
    pos[0] = 0.0; pos[1] = 0.0; pos[2] = copysign(fabs(r), ct);
    return;
  }
  pos[0] = (r * cp - spin * sp) * st;
  pos[1] = (r * sp + spin * cp) * st;
  pos[2] = r * ct;
}

void orc_ks_spheroidal_position(double r, double theta, double phi, double spin, double *pos) {
  ks_position(r, sin(theta), cos(theta), sin(phi), cos(phi), spin, pos);
}

/* output.f90:797-834 gw_cartesian_kinematics: coordinate rates alpha v - beta (the radial
 * rate times r on a logarithmic grid), the Cartesian position and velocity of the
 * Kerr-Schild spheroidal chart, and the flat-space Jacobian sigma sin(theta) */
static void gw_kinematics(double r, double st, double ct, double sp, double cp, double spin, double alpha,
                          const double *beta, const double *v, int use_log_r, double *pos, double *vel, double *jac) {
  double rates[3];
  for (int d = 0; d < 3; ++d) rates[d] = alpha * v[d] - beta[d];
  if (use_log_r) rates[0] = r * rates[0];
  ks_position(r, st, ct, sp, cp, spin, pos);
  vel[0] = rates[0] * cp * st + rates[1] * (r * cp - spin * sp) * ct - rates[2] * (r * sp + spin * cp) * st;
  vel[1] = rates[0] * sp * st + rates[1] * (r * sp + spin * cp) * ct + rates[2] * (r * cp - spin * sp) * st;
  vel[2] = rates[0] * ct - r * rates[1] * st;
  const double sigma = r * r + spin * spin * (ct * ct);
  *jac = sigma * st;
}

void orc_gw_kinematics(double r, double theta, double phi, double spin, double alpha, const double *beta,
                       const double *v, int use_log_r, double *pos, double *vel, double *jac) {
  gw_kinematics(r, sin(theta), cos(theta), sin(phi), cos(phi), spin, alpha, beta, v, use_log_r, pos, vel, jac);
}

/* output.f90:837-850 finn_evans_cell_stress */
void orc_finn_evans_stress(double rho, double pres, double mr3, const double *pos, const double *vel, double dV,
                           double *ixx, double *iyy, double *ixy) {
  *ixx = (2.0 * rho * (vel[0] * vel[0]) + 2.0 * pres - 2.0 * rho * mr3 * (pos[0] * pos[0])) * dV;
  *iyy = (2.0 * rho * (vel[1] * vel[1]) + 2.0 * pres - 2.0 * rho * mr3 * (pos[1] * pos[1])) * dV;
  *ixy = (2.0 * rho * vel[0] * vel[1] - 2.0 * rho * mr3 * pos[0] * pos[1]) * dV;
}

/* output.f90:852-948 */
int orc_gw_strain(const orc_config *c, const orc_metric *m, const double *p, const double *xc, const double *yc,
                  const double *zc, int use_log_r, double bh_mass, double spin, double *out) {
  for (int q = 0; q < 5; ++q) out[q] = 0.0;
  if (c->metric_kind == ORC_METRIC_MINKOWSKI || bh_mass < 0.1) return 1;
  double r_h;
  if (orc_horizon_radius(bh_mass, spin, &r_h)) return -1;
  const lay_t L = mklay(c);
  double ixx = 0.0, iyy = 0.0, ixy = 0.0;
  for (int k = 1; k <= c->nz; ++k)
    for (int j = 1; j <= c->ny; ++j)
      for (int i = 1; i <= c->nx; ++i) {
        const double r = use_log_r ? exp(xc[i - 1]) : xc[i - 1];
        if (r <= r_h) continue;
        const double th = yc[j - 1], ph = zc[k - 1];
        double rho = p[pidx(&L, 0, i, j, k)], pres = p[pidx(&L, 1, i, j, k)];
        rho = rho - c->rho_floor; if (!(rho > 0.0)) rho = 0.0;  /* max(0, rho - rho_floor) */
        pres = pres - c->p_floor; if (!(pres > 0.0)) pres = 0.0;
        if (rho <= 0.0 && pres <= 0.0) continue;
        const size_t q = cell(c, i, j);
        const double v[3] = {p[pidx(&L, 2, i, j, k)], p[pidx(&L, 3, i, j, k)], p[pidx(&L, 4, i, j, k)]};
        double pos[3], vel[3], jac, cx, cy, cxy;
        gw_kinematics(r, sin(th), cos(th), sin(ph), cos(ph), spin, m->alpha_c[q], &m->beta_c[3 * q], v, use_log_r,
                      pos, vel, &jac);
        const double dV = jac * (use_log_r ? r : 1.0) * c->dx * c->dy * c->dz;
        const double r2 = pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2];
        const double mr3 = bh_mass / (r2 * sqrt(r2));
        orc_finn_evans_stress(rho, pres, mr3, pos, vel, dV, &cx, &cy, &cxy);
        ixx = ixx + cx;
        iyy = iyy + cy;
        ixy = ixy + cxy;
      }
  out[0] = (ixx - iyy) / 1000.0;
  out[1] = (2.0 * ixy) / 1000.0;
  out[2] = ixx; out[3] = iyy; out[4] = ixy;
  return 0;
}
