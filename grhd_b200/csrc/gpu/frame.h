// frame.h -- per-face geometry that the reference recomputes at every Riemann call and
// that depends only on the face metric: the Cramer gamma^dd used by
// calc_wavespeeds_grhd (fluxes.f90:760-774) and the orthonormal face frame of
// build_face_orthonormal_frame (fluxes.f90:402-473).  Evaluated once per face on the host
// when the metric tables are uploaded; same arithmetic, same order, IEEE double.  The
// functions also compile for the device (the allocation-free face entry point builds its
// per-face table there).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define GRHD_HD __host__ __device__
#else
#define GRHD_HD
#endif

namespace grhd {

// g: Fortran (3,3) array g[(a-1)+3(b-1)]
GRHD_HD inline double det3(const double *g) {
#define GA(a, b) g[((a) - 1) + 3 * ((b) - 1)]
  return GA(1, 1) * (GA(2, 2) * GA(3, 3) - GA(2, 3) * GA(3, 2)) - GA(1, 2) * (GA(2, 1) * GA(3, 3) - GA(2, 3) * GA(3, 1)) +
         GA(1, 3) * (GA(2, 1) * GA(3, 2) - GA(2, 2) * GA(3, 1));
}
// gamma^dd of calc_wavespeeds_grhd
GRHD_HD inline double gamma_up_dd(const double *g, int dir) {
  const double det = det3(g);
  if (dir == 1) return (GA(2, 2) * GA(3, 3) - GA(2, 3) * GA(3, 2)) / det;
  if (dir == 2) return (GA(1, 1) * GA(3, 3) - GA(1, 3) * GA(3, 1)) / det;
  return (GA(1, 1) * GA(2, 2) - GA(1, 2) * GA(2, 1)) / det;
}
GRHD_HD inline double metric_dot3(const double *a, const double *b, const double *g) {
  double s = 0.0;
  for (int i = 1; i <= 3; ++i)
    for (int j = 1; j <= 3; ++j) s = s + GA(i, j) * a[i - 1] * b[j - 1];
  return s;
}
// cof[3a+i] = coframe(a+1,i+1); returns ok
GRHD_HD inline bool face_frame(const double *g, int dir, double *cof, double *gup) {
  double frame[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 9; ++q) cof[q] = 0.0;
  *gup = 0.0;
  for (int q = 0; q < 9; ++q) if (!std::isfinite(g[q])) return false;
  const double det = det3(g);
  if (!std::isfinite(det) || det <= 1.0e-30) return false;
  double gi[9];
#define GI(a, b) gi[((a) - 1) + 3 * ((b) - 1)]
  GI(1, 1) = (GA(2, 2) * GA(3, 3) - GA(2, 3) * GA(3, 2)) / det;
  GI(1, 2) = (GA(1, 3) * GA(3, 2) - GA(1, 2) * GA(3, 3)) / det;
  GI(1, 3) = (GA(1, 2) * GA(2, 3) - GA(1, 3) * GA(2, 2)) / det;
  GI(2, 1) = (GA(2, 3) * GA(3, 1) - GA(2, 1) * GA(3, 3)) / det;
  GI(2, 2) = (GA(1, 1) * GA(3, 3) - GA(1, 3) * GA(3, 1)) / det;
  GI(2, 3) = (GA(1, 3) * GA(2, 1) - GA(1, 1) * GA(2, 3)) / det;
  GI(3, 1) = (GA(2, 1) * GA(3, 2) - GA(2, 2) * GA(3, 1)) / det;
  GI(3, 2) = (GA(1, 2) * GA(3, 1) - GA(1, 1) * GA(3, 2)) / det;
  GI(3, 3) = (GA(1, 1) * GA(2, 2) - GA(1, 2) * GA(2, 1)) / det;
  for (int q = 0; q < 9; ++q) if (!std::isfinite(gi[q])) return false;
  *gup = GI(dir, dir);
  if (*gup <= 1.0e-30 || !std::isfinite(*gup)) return false;
  for (int i = 1; i <= 3; ++i) frame[i - 1] = GI(i, dir) / std::sqrt(*gup);
#undef GI
  int t0, t1;
  if (dir == 1) { t0 = 2; t1 = 3; } else if (dir == 2) { t0 = 3; t1 = 1; } else { t0 = 1; t1 = 2; }
  const int tan_dirs[2] = {t0, t1};
  for (int b = 2; b <= 3; ++b) {
    double seed[3] = {0.0, 0.0, 0.0};
    seed[tan_dirs[b - 2] - 1] = 1.0;
    for (int a = 1; a <= b - 1; ++a) {
      const double pr = metric_dot3(seed, &frame[3 * (a - 1)], g);
      for (int i = 0; i < 3; ++i) seed[i] = seed[i] - pr * frame[3 * (a - 1) + i];
    }
    const double nsq = metric_dot3(seed, seed, g);
    if (!std::isfinite(nsq) || nsq <= 1.0e-28) return false;
    for (int i = 0; i < 3; ++i) frame[3 * (b - 1) + i] = seed[i] / std::sqrt(nsq);
  }
  for (int a = 1; a <= 3; ++a)
    for (int i = 1; i <= 3; ++i) {
      double s = 0.0;
      for (int j = 1; j <= 3; ++j) s = s + GA(i, j) * frame[3 * (a - 1) + (j - 1)];
      cof[3 * (a - 1) + (i - 1)] = s;
    }
  for (int q = 0; q < 9; ++q) if (!std::isfinite(frame[q]) || !std::isfinite(cof[q])) return false;
  return true;
#undef GA
}

}  // namespace grhd
