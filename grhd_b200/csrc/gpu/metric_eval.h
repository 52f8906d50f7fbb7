// metric_eval.h -- the reference's analytic 3+1 metrics (metrics.f90:209-1242) and the
// set_metric_type dispatch (metrics.f90:94-201), as one set of functions that the host
// set-up (grhd_b200/csrc/host/problem.cpp, built by g++) and the device metric-cache build
// (grhd2_gpu_set_metric_analytic, built by nvcc) both compile.  The arithmetic and its
// order are the reference's; unqualified math calls resolve to the C library on the host
// and to CUDA's double-precision functions on the device, so the two builds agree bit for
// bit wherever no sin, cos or exp is taken (Minkowski Cartesian and cylindrical) and to a
// few ulps elsewhere.
//
// Layouts (Fortran order): gamma(3,3) -> g[(a-1)+3(b-1)], gmunu(0:3,0:3) -> gm[mu+4nu],
// chris(0:3,0:3,0:3) -> ch[l+4m+16n], dg(0:3,0:3,1:3) -> dg[m+4n+16(d-1)], dlnalpha(0:3).
#pragma once

#include <cmath>

#ifndef GRHD_HD
#if defined(__CUDACC__)
#define GRHD_HD __host__ __device__
#else
#define GRHD_HD
#endif
#endif

namespace grhd2_metric {

enum Geom { CART = 0, CYL = 1, SPH = 2, SPHEROID = 3 };
enum Metric { MINK = 0, EF = 1, KS = 2 };

// what set_metric_type selects on (metrics.f90:94-201) and the derivative tables' ny == 1
// rule (the theta derivatives vanish on grids with one theta cell)
struct Kind {
  int metric, geom, log_r, ny;
  double bh_mass, a_spin;
};

struct MetricOut {
  double alpha, beta[3], gamma[9], gmunu[16], det, dlna[4];
};

GRHD_HD inline void clear(MetricOut &m) {
  m.alpha = 0.0;
  m.det = 0.0;
  for (int q = 0; q < 3; ++q) m.beta[q] = 0.0;
  for (int q = 0; q < 9; ++q) m.gamma[q] = 0.0;
  for (int q = 0; q < 16; ++q) m.gmunu[q] = 0.0;
  for (int q = 0; q < 4; ++q) m.dlna[q] = 0.0;
}

GRHD_HD inline double sq(double x) { return x * x; }

#define GG(a, b) m.gamma[((a) - 1) + 3 * ((b) - 1)]
#define GM(a, b) m.gmunu[(a) + 4 * (b)]
#define CH(l, a, b) ch[(l) + 4 * (a) + 16 * (b)]
#define DG(a, b, d) dg[(a) + 4 * (b) + 16 * ((d) - 1)]

// metrics.f90:209-239
GRHD_HD inline void metric_minkowski(MetricOut &m) {
  m.alpha = 1.0;
  GG(1, 1) = 1.0; GG(2, 2) = 1.0; GG(3, 3) = 1.0;
  m.det = 1.0;
  GM(0, 0) = -1.0; GM(1, 1) = 1.0; GM(2, 2) = 1.0; GM(3, 3) = 1.0;
}
// metrics.f90:419-450
GRHD_HD inline void metric_cylindrical(double x, MetricOut &m) {
  m.alpha = 1.0;
  GG(1, 1) = 1.0; GG(2, 2) = sq(x); GG(3, 3) = 1.0;
  m.det = sq(x);
  GM(0, 0) = -1.0; GM(1, 1) = 1.0; GM(2, 2) = 1.0 / fmax(sq(x), 1.0e-20); GM(3, 3) = 1.0;
}
GRHD_HD inline void chris_cylindrical(double x, double *ch) {
  CH(1, 2, 2) = -x;
  CH(2, 1, 2) = 1.0 / fmax(x, 1.0e-15);
  CH(2, 2, 1) = 1.0 / fmax(x, 1.0e-15);
}
GRHD_HD inline void derivs_cylindrical(double x, double *dg) { DG(2, 2, 1) = 2.0 * x; }
// metrics.f90:265-333
GRHD_HD inline void metric_mink_sph_phys(double r, double th, MetricOut &m) {
  double r2 = sq(r), s = sin(th), s2 = sq(s);
  m.alpha = 1.0;
  GG(1, 1) = 1.0; GG(2, 2) = r2; GG(3, 3) = r2 * s2;
  m.det = r2 * r2 * s2;
  GM(0, 0) = -1.0; GM(1, 1) = 1.0; GM(2, 2) = 1.0 / r2; GM(3, 3) = 1.0 / fmax(r2 * s2, 1.0e-30);
}
GRHD_HD inline void derivs_mink_sph_phys(double r, double th, int ny, double *dg) {
  double s = sin(th), c = cos(th);
  DG(2, 2, 1) = 2.0 * r;
  DG(3, 3, 1) = 2.0 * r * sq(s);
  DG(3, 3, 2) = 2.0 * sq(r) * s * c;
  if (ny == 1) for (int a = 0; a < 16; ++a) dg[a + 16] = 0.0;
}
GRHD_HD inline void chris_mink_sph_phys(double r, double th, double *ch) {
  double s = sin(th), c = cos(th);
  double safe = copysign(fmax(fabs(s), 1.0e-20), s);
  CH(1, 2, 2) = -r;
  CH(1, 3, 3) = -r * sq(s);
  CH(2, 1, 2) = 1.0 / r; CH(2, 2, 1) = CH(2, 1, 2);
  CH(2, 3, 3) = -s * c;
  CH(3, 1, 3) = 1.0 / r; CH(3, 3, 1) = CH(3, 1, 3);
  CH(3, 2, 3) = c / safe; CH(3, 3, 2) = CH(3, 2, 3);
}
// metrics.f90:338-411
GRHD_HD inline void metric_mink_sph_log(double x, double th, MetricOut &m) {
  double r = exp(x), r2 = sq(r), s = sin(th), s2 = sq(s);
  m.alpha = 1.0;
  GG(1, 1) = r2; GG(2, 2) = r2; GG(3, 3) = r2 * s2;
  m.det = r2 * r2 * r2 * s2;
  GM(0, 0) = -1.0; GM(1, 1) = 1.0 / r2; GM(2, 2) = 1.0 / r2; GM(3, 3) = 1.0 / fmax(r2 * s2, 1.0e-30);
}
GRHD_HD inline void derivs_mink_sph_log(double x, double th, int ny, double *dg) {
  double r2 = exp(2.0 * x), s = sin(th), c = cos(th);
  DG(1, 1, 1) = 2.0 * r2;
  DG(2, 2, 1) = 2.0 * r2;
  DG(3, 3, 1) = 2.0 * r2 * sq(s);
  DG(3, 3, 2) = 2.0 * r2 * s * c;
  if (ny == 1) for (int a = 0; a < 16; ++a) dg[a + 16] = 0.0;
}
GRHD_HD inline void chris_mink_sph_log(double th, double *ch) {
  double s = sin(th), c = cos(th);
  double safe = copysign(fmax(fabs(s), 1.0e-20), s);
  CH(1, 1, 1) = 1.0;
  CH(1, 2, 2) = -1.0;
  CH(1, 3, 3) = -sq(s);
  CH(2, 1, 2) = 1.0; CH(2, 2, 1) = CH(2, 1, 2);
  CH(2, 3, 3) = -s * c;
  CH(3, 1, 3) = 1.0; CH(3, 3, 1) = CH(3, 1, 3);
  CH(3, 2, 3) = c / safe; CH(3, 3, 2) = CH(3, 2, 3);
}
// metrics.f90:492-610 (EF, physical r)
GRHD_HD inline void metric_ef_phys(double r, double th, double M, bool want_gmunu, MetricOut &m) {
  double s = sin(th);
  m.alpha = 1.0 / sqrt(1.0 + 2.0 * M / r);
  m.beta[0] = 2.0 * M / r / (1.0 + 2.0 * M / r);
  double g11 = 1.0 + 2.0 * M / r, g22 = sq(r), g33 = sq(r) * sq(s);
  m.det = g11 * g22 * g33;
  GG(1, 1) = g11; GG(2, 2) = g22; GG(3, 3) = g33;
  if (want_gmunu) {
    GM(0, 0) = -1.0 / sq(m.alpha);
    for (int d = 1; d <= 3; ++d) { GM(0, d) = m.beta[d - 1] / sq(m.alpha); GM(d, 0) = GM(0, d); }
    GM(1, 1) = 1.0 / g11 - sq(m.beta[0]) / sq(m.alpha);
    GM(2, 2) = 1.0 / g22 - sq(m.beta[1]) / sq(m.alpha);
    GM(3, 3) = 1.0 / g33 - sq(m.beta[2]) / sq(m.alpha);
  }
  m.dlna[1] = M / (sq(r) + 2.0 * M * r);
}
GRHD_HD inline void chris_ef_phys(double r, double th, double M, double *ch) {
  double s = sin(th), c = cos(th);
  double safe = copysign(fmax(fabs(s), 1.0e-20), s);
  double r3 = r * r * r;
  CH(0, 0, 0) = 2.0 * sq(M) / r3;
  CH(0, 0, 1) = M * (1.0 + 2.0 * M / r) / sq(r);
  CH(0, 1, 0) = CH(0, 0, 1);
  CH(0, 1, 1) = 2.0 * M * (1.0 + M / r) / sq(r);
  CH(0, 2, 2) = -2.0 * M;
  CH(0, 3, 3) = CH(0, 2, 2) * sq(s);
  CH(1, 0, 0) = M / sq(r) * (1.0 - 2.0 * M / r);
  CH(1, 0, 1) = -CH(0, 0, 0);
  CH(1, 1, 0) = CH(1, 0, 1);
  CH(1, 1, 1) = -CH(0, 0, 1);
  CH(1, 2, 2) = 2.0 * M - r;
  CH(1, 3, 3) = CH(1, 2, 2) * sq(s);
  CH(2, 1, 2) = 1.0 / r; CH(2, 2, 1) = CH(2, 1, 2);
  CH(2, 3, 3) = -s * c;
  CH(3, 1, 3) = 1.0 / r; CH(3, 3, 1) = CH(3, 1, 3);
  CH(3, 2, 3) = c / safe; CH(3, 3, 2) = CH(3, 2, 3);
}
GRHD_HD inline void derivs_ef_phys(double r, double th, double M, int ny, double *dg) {
  double s = sin(th), c = cos(th);
  DG(0, 0, 1) = -2.0 * M / sq(r);
  DG(0, 1, 1) = -2.0 * M / sq(r); DG(1, 0, 1) = DG(0, 1, 1);
  DG(1, 1, 1) = -2.0 * M / sq(r);
  DG(2, 2, 1) = 2.0 * r;
  DG(3, 3, 1) = 2.0 * r * sq(s);
  DG(3, 3, 2) = sq(r) * 2.0 * s * c;
  if (ny == 1) for (int a = 0; a < 16; ++a) dg[a + 16] = 0.0;
}
// metrics.f90:612-746 (EF, x = ln r)
GRHD_HD inline void metric_ef_log(double x, double th, double M, bool want_gmunu, MetricOut &m) {
  double r = exp(x), s = sin(th);
  m.alpha = 1.0 / sqrt(1.0 + 2.0 * M / r);
  m.beta[0] = (2.0 * M / r / (1.0 + 2.0 * M / r)) / r;
  double g11 = (1.0 + 2.0 * M / r) * sq(r), g22 = sq(r), g33 = sq(r) * sq(s);
  m.det = g11 * g22 * g33;
  GG(1, 1) = g11; GG(2, 2) = g22; GG(3, 3) = g33;
  if (want_gmunu) {
    GM(0, 0) = -1.0 / sq(m.alpha);
    for (int d = 1; d <= 3; ++d) { GM(0, d) = m.beta[d - 1] / sq(m.alpha); GM(d, 0) = GM(0, d); }
    GM(1, 1) = 1.0 / g11 - sq(m.beta[0]) / sq(m.alpha);
    GM(2, 2) = 1.0 / g22 - sq(m.beta[1]) / sq(m.alpha);
    GM(3, 3) = 1.0 / g33 - sq(m.beta[2]) / sq(m.alpha);
  }
  m.dlna[1] = M / (r + 2.0 * M);
}
GRHD_HD inline void chris_ef_log(double x, double th, double M, double *ch) {
  double r = exp(x), s = sin(th), c = cos(th);
  double safe = copysign(fmax(fabs(s), 1.0e-20), s);
  double r3 = r * r * r;
  CH(0, 0, 0) = 2.0 * sq(M) / r3;
  CH(0, 0, 1) = M * (1.0 + 2.0 * M / r) / r;
  CH(0, 1, 0) = CH(0, 0, 1);
  CH(0, 1, 1) = 2.0 * M * (1.0 + M / r);
  CH(0, 2, 2) = -2.0 * M;
  CH(0, 3, 3) = CH(0, 2, 2) * sq(s);
  CH(1, 0, 0) = M / r3 * (1.0 - 2.0 * M / r);
  CH(1, 0, 1) = -2.0 * sq(M) / r3;
  CH(1, 1, 0) = CH(1, 0, 1);
  CH(1, 1, 1) = 1.0 - M / r - 2.0 * sq(M) / sq(r);
  CH(1, 2, 2) = 2.0 * M / r - 1.0;
  CH(1, 3, 3) = CH(1, 2, 2) * sq(s);
  CH(2, 1, 2) = 1.0; CH(2, 2, 1) = CH(2, 1, 2);
  CH(2, 3, 3) = -s * c;
  CH(3, 1, 3) = 1.0; CH(3, 3, 1) = CH(3, 1, 3);
  CH(3, 2, 3) = c / safe; CH(3, 3, 2) = CH(3, 2, 3);
}
GRHD_HD inline void derivs_ef_log(double x, double th, double M, int ny, double *dg) {
  double r = exp(x), s = sin(th), c = cos(th);
  DG(0, 0, 1) = -2.0 * M / r;
  DG(0, 1, 1) = 0.0; DG(1, 0, 1) = DG(0, 1, 1);
  DG(1, 1, 1) = 2.0 * sq(r) + 2.0 * M * r;
  DG(2, 2, 1) = 2.0 * sq(r);
  DG(3, 3, 1) = 2.0 * sq(r) * sq(s);
  DG(3, 3, 2) = 2.0 * sq(r) * s * c;
  if (ny == 1) for (int a = 0; a < 16; ++a) dg[a + 16] = 0.0;
}
// metrics.f90:753-921 (KS, physical r)
GRHD_HD inline void metric_ks_phys(double r, double th, double M, double a, bool want_gmunu, MetricOut &m) {
  double s = sin(th), c = cos(th), s2 = sq(s), c2 = sq(c);
  double Sigma = sq(r) + sq(a) * c2, H = M * r / Sigma, Delta = sq(r) - 2.0 * M * r + sq(a);
  m.alpha = 1.0 / sqrt(1.0 + 2.0 * H);
  m.beta[0] = 2.0 * H / (1.0 + 2.0 * H);
  GG(1, 1) = 1.0 + 2.0 * H;
  GG(1, 3) = -a * (1.0 + 2.0 * H) * s2; GG(3, 1) = GG(1, 3);
  GG(2, 2) = Sigma;
  GG(3, 3) = (sq(r) + sq(a) + 2.0 * H * sq(a) * s2) * s2;
  m.det = sq(Sigma) * s2 * (1.0 + 2.0 * H);
  if (want_gmunu) {
    GM(0, 0) = -(1.0 + 2.0 * H);
    GM(0, 1) = 2.0 * H; GM(1, 0) = GM(0, 1);
    GM(1, 1) = Delta / Sigma;
    GM(1, 3) = a / Sigma; GM(3, 1) = GM(1, 3);
    GM(2, 2) = 1.0 / Sigma;
    GM(3, 3) = (fabs(s) > 1.0e-15) ? 1.0 / (Sigma * s2) : 1.0 / (Sigma * 1.0e-30);
  }
  double dH_dr = M * (sq(a) * c2 - sq(r)) / sq(Sigma);
  double dH_dth = 2.0 * M * r * sq(a) * s * c / sq(Sigma);
  m.dlna[1] = -dH_dr / (1.0 + 2.0 * H);
  m.dlna[2] = -dH_dth / (1.0 + 2.0 * H);
}
GRHD_HD inline void derivs_ks_phys(double r, double th, double M, double a, int ny, double *dg) {
  double s = sin(th), c = cos(th), s2 = sq(s), c2 = sq(c);
  double Sigma = sq(r) + sq(a) * c2, H = M * r / Sigma;
  double dS_dr = 2.0 * r, dS_dth = -2.0 * sq(a) * s * c;
  double dH_dr = M * (sq(a) * c2 - sq(r)) / sq(Sigma);
  double dH_dth = 2.0 * M * r * sq(a) * s * c / sq(Sigma);
  DG(0, 0, 1) = 2.0 * dH_dr;
  DG(0, 1, 1) = 2.0 * dH_dr; DG(1, 0, 1) = DG(0, 1, 1);
  DG(0, 3, 1) = -2.0 * a * s2 * dH_dr; DG(3, 0, 1) = DG(0, 3, 1);
  DG(1, 1, 1) = 2.0 * dH_dr;
  DG(1, 3, 1) = -a * s2 * (2.0 * dH_dr); DG(3, 1, 1) = DG(1, 3, 1);
  DG(2, 2, 1) = dS_dr;
  DG(3, 3, 1) = 2.0 * r * s2 + 2.0 * sq(a) * sq(s2) * dH_dr;
  DG(0, 0, 2) = 2.0 * dH_dth;
  DG(0, 1, 2) = 2.0 * dH_dth; DG(1, 0, 2) = DG(0, 1, 2);
  DG(0, 3, 2) = -2.0 * a * (s2 * dH_dth + 2.0 * H * s * c); DG(3, 0, 2) = DG(0, 3, 2);
  DG(1, 1, 2) = 2.0 * dH_dth;
  DG(1, 3, 2) = -a * ((1.0 + 2.0 * H) * 2.0 * s * c + s2 * 2.0 * dH_dth); DG(3, 1, 2) = DG(1, 3, 2);
  DG(2, 2, 2) = dS_dth;
  DG(3, 3, 2) = 2.0 * (sq(r) + sq(a)) * s * c + 2.0 * sq(a) * sq(s2) * dH_dth + 8.0 * sq(a) * H * s * c * s2;
  if (ny == 1) for (int q = 0; q < 16; ++q) dg[q + 16] = 0.0;
}
// metrics.f90:998-1180 (KS, x = ln r)
GRHD_HD inline void metric_ks_log(double x, double th, double M, double a, bool want_gmunu, MetricOut &m) {
  double r = exp(x), s = sin(th), c = cos(th), s2 = sq(s), c2 = sq(c);
  double Sigma = sq(r) + sq(a) * c2, H = M * r / Sigma, Delta = sq(r) - 2.0 * M * r + sq(a);
  m.alpha = 1.0 / sqrt(1.0 + 2.0 * H);
  m.beta[0] = (2.0 * H / (1.0 + 2.0 * H)) / r;
  GG(1, 1) = (1.0 + 2.0 * H) * sq(r);
  GG(1, 3) = -a * (1.0 + 2.0 * H) * s2 * r; GG(3, 1) = GG(1, 3);
  GG(2, 2) = Sigma;
  GG(3, 3) = (sq(r) + sq(a) + 2.0 * H * sq(a) * s2) * s2;
  m.det = (sq(Sigma) * s2 * (1.0 + 2.0 * H)) * sq(r);
  if (want_gmunu) {
    GM(0, 0) = -(1.0 + 2.0 * H);
    GM(0, 1) = (2.0 * H) / r; GM(1, 0) = GM(0, 1);
    GM(1, 1) = (Delta / Sigma) / sq(r);
    GM(1, 3) = (a / Sigma) / r; GM(3, 1) = GM(1, 3);
    GM(2, 2) = 1.0 / Sigma;
    GM(3, 3) = (fabs(s) > 1.0e-15) ? 1.0 / (Sigma * s2) : 1.0 / (Sigma * 1.0e-30);
  }
  double dH_dr = M * (sq(a) * c2 - sq(r)) / sq(Sigma);
  double dH_dth = 2.0 * M * r * sq(a) * s * c / sq(Sigma);
  m.dlna[1] = -(dH_dr * r) / (1.0 + 2.0 * H);
  m.dlna[2] = -dH_dth / (1.0 + 2.0 * H);
}
GRHD_HD inline void derivs_ks_log(double x, double th, double M, double a, int ny, double *dg) {
  double r = exp(x), s = sin(th), c = cos(th), s2 = sq(s), c2 = sq(c);
  double Sigma = sq(r) + sq(a) * c2, H = M * r / Sigma;
  double dS_dth = -2.0 * sq(a) * s * c;
  double dH_dr = M * (sq(a) * c2 - sq(r)) / sq(Sigma);
  double dH_dth = 2.0 * M * r * sq(a) * s * c / sq(Sigma);
  double g_tr = 2.0 * H, g_rr = 1.0 + 2.0 * H, g_rphi = -a * (1.0 + 2.0 * H) * s2;
  double r3 = r * r * r;
  DG(0, 0, 1) = r * (2.0 * dH_dr);
  DG(0, 1, 1) = r * g_tr + sq(r) * (2.0 * dH_dr); DG(1, 0, 1) = DG(0, 1, 1);
  DG(0, 3, 1) = r * (-2.0 * a * s2 * dH_dr); DG(3, 0, 1) = DG(0, 3, 1);
  DG(1, 1, 1) = 2.0 * sq(r) * g_rr + r3 * (2.0 * dH_dr);
  DG(1, 3, 1) = r * g_rphi + sq(r) * (-2.0 * a * s2 * dH_dr); DG(3, 1, 1) = DG(1, 3, 1);
  DG(2, 2, 1) = 2.0 * sq(r);
  DG(3, 3, 1) = r * (2.0 * r * s2 + 2.0 * sq(a) * sq(s2) * dH_dr);
  DG(0, 0, 2) = 2.0 * dH_dth;
  DG(0, 1, 2) = r * (2.0 * dH_dth); DG(1, 0, 2) = DG(0, 1, 2);
  DG(0, 3, 2) = -2.0 * a * (s2 * dH_dth + 2.0 * H * s * c); DG(3, 0, 2) = DG(0, 3, 2);
  DG(1, 1, 2) = sq(r) * (2.0 * dH_dth);
  DG(1, 3, 2) = r * (-a * ((1.0 + 2.0 * H) * 2.0 * s * c + s2 * 2.0 * dH_dth)); DG(3, 1, 2) = DG(1, 3, 2);
  DG(2, 2, 2) = dS_dth;
  DG(3, 3, 2) = 2.0 * (sq(r) + sq(a)) * s * c + 2.0 * sq(a) * sq(s2) * dH_dth + 8.0 * sq(a) * H * s * c * s2;
  if (ny == 1) for (int q = 0; q < 16; ++q) dg[q + 16] = 0.0;
}
// metrics.f90:926-990 / 1186-1242: Gamma^l_{mn} = 1/2 g^{lr}(d_m g_rn + d_n g_rm - d_r g_mn)
GRHD_HD inline void chris_from_dg(const double *gmunu, const double *dg, double *ch) {
  for (int l = 0; l <= 3; ++l)
    for (int mu = 0; mu <= 3; ++mu)
      for (int nu = mu; nu <= 3; ++nu) {
        for (int rho = 0; rho <= 3; ++rho) {
          double dm = 0.0, dn = 0.0, dr = 0.0;
          if (mu == 1) dm = DG(rho, nu, 1); else if (mu == 2) dm = DG(rho, nu, 2);
          if (nu == 1) dn = DG(rho, mu, 1); else if (nu == 2) dn = DG(rho, mu, 2);
          if (rho == 1) dr = DG(mu, nu, 1); else if (rho == 2) dr = DG(mu, nu, 2);
          CH(l, mu, nu) = CH(l, mu, nu) + 0.5 * gmunu[l + 4 * rho] * (dm + dn - dr);
        }
        if (mu != nu) CH(l, nu, mu) = CH(l, mu, nu);
      }
}
#undef GG
#undef GM
#undef CH
#undef DG

// set_metric_type dispatch (metrics.f90:94-201): the 3+1 quantities at (x, y)
GRHD_HD inline void eval_metric(const Kind &K, double x, double y, bool want_gmunu, MetricOut &m) {
  clear(m);
  switch (K.metric) {
  case MINK:
    if (K.geom == CART) metric_minkowski(m);
    else if (K.geom == CYL) metric_cylindrical(x, m);
    else if (K.log_r) metric_mink_sph_log(x, y, m);
    else metric_mink_sph_phys(x, y, m);
    break;
  case EF:
    if (K.log_r) metric_ef_log(x, y, K.bh_mass, want_gmunu, m);
    else metric_ef_phys(x, y, K.bh_mass, want_gmunu, m);
    break;
  case KS:
    if (K.log_r) metric_ks_log(x, y, K.bh_mass, K.a_spin, want_gmunu, m);
    else metric_ks_phys(x, y, K.bh_mass, K.a_spin, want_gmunu, m);
    break;
  }
}
// Christoffel symbols (64) and metric derivatives (48) at (x, y); KS contracts them from
// the derivatives (metrics.f90:926-990), the others are closed forms
GRHD_HD inline void eval_chris_dg(const Kind &K, double x, double y, double *ch, double *dg) {
  for (int q = 0; q < 64; ++q) ch[q] = 0.0;
  for (int q = 0; q < 48; ++q) dg[q] = 0.0;
  switch (K.metric) {
  case MINK:
    if (K.geom == CART) {
    } else if (K.geom == CYL) {
      chris_cylindrical(x, ch); derivs_cylindrical(x, dg);
    } else if (K.log_r) {
      chris_mink_sph_log(y, ch); derivs_mink_sph_log(x, y, K.ny, dg);
    } else {
      chris_mink_sph_phys(x, y, ch); derivs_mink_sph_phys(x, y, K.ny, dg);
    }
    break;
  case EF:
    if (K.log_r) { chris_ef_log(x, y, K.bh_mass, ch); derivs_ef_log(x, y, K.bh_mass, K.ny, dg); }
    else { chris_ef_phys(x, y, K.bh_mass, ch); derivs_ef_phys(x, y, K.bh_mass, K.ny, dg); }
    break;
  case KS: {
    MetricOut m;
    clear(m);
    if (K.log_r) {
      metric_ks_log(x, y, K.bh_mass, K.a_spin, true, m);
      derivs_ks_log(x, y, K.bh_mass, K.a_spin, K.ny, dg);
    } else {
      metric_ks_phys(x, y, K.bh_mass, K.a_spin, true, m);
      derivs_ks_phys(x, y, K.bh_mass, K.a_spin, K.ny, dg);
    }
    chris_from_dg(m.gmunu, dg, ch);
    break;
  }
  }
}

}  // namespace grhd2_metric
