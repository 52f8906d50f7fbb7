// metric_build.cuh -- the metric cache built on the device (grhd2_gpu_set_metric_analytic).
//
// precalculate_metric_cache (initialization.f90:265-391) evaluates the analytic metric
// (metrics.f90:94-1242) at every cell centre and face of the (i, j) plane -- the cache is
// k-invariant -- and the Riemann solver rebuilds the face frame from it at every call
// (fluxes.f90:402-473, :760-774).  Here one thread per table entry evaluates the same
// functions (metric_eval.h, shared with the host set-up) and writes the packed centre and
// face tables the stage kernels read, with the same fields and arithmetic as the host-side
// packing of grhd2_gpu_set_metric.  Compiled without FMA contraction, so only the device's
// sin, cos and exp separate the result from a host-built cache.
#pragma once

#include <cfloat>

#include "frame.h"
#include "metric_eval.h"
#include "state.cuh"

namespace grhd {

// the cell-centred grid of the (i, j) plane: centres x_min + (i - 1/2) dx, faces x_min + i dx
// (allocate_and_grid, initialization.f90:84-215)
struct MetricGrid {
  grhd2_metric::Kind kind;
  int nx, ny;
  double x_min, y_min, dx, dy;
};

// status bits: a table entry that is not exactly symmetric (the host path's upload check),
// a face whose frame gamma^dd differs from its wavespeed gamma^dd
constexpr unsigned long long MB_ASYM = 1ull, MB_FRAME = 2ull;

__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}

__device__ __forceinline__ double centre_x(const MetricGrid &g, int i) { return g.x_min + ((double)i - 0.5) * g.dx; }
__device__ __forceinline__ double centre_y(const MetricGrid &g, int j) { return g.y_min + ((double)j - 0.5) * g.dy; }

// centre table: entry q = (i - 1) + nx (j - 1) of the NCF x nx*ny planes
__global__ void __launch_bounds__(128) k_metric_centre(MetricGrid g, double *__restrict__ C,
                                                       unsigned long long *status) {
  const int nij = g.nx * g.ny;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nij) return;
  const int i = q % g.nx + 1, j = q / g.nx + 1;
  const double x = centre_x(g, i), y = centre_y(g, j);
  grhd2_metric::MetricOut m;
  double ch[64], dg[48];
  grhd2_metric::eval_metric(g.kind, x, y, true, m);
  grhd2_metric::eval_chris_dg(g.kind, x, y, ch, dg);
  // gamma^ij = g^ij + beta^i beta^j / alpha^2 (initialization.f90:297)
  double gi[9];
  for (int a = 1; a <= 3; ++a)
    for (int b = 1; b <= 3; ++b)
      gi[(a - 1) + 3 * (b - 1)] = m.gmunu[a + 4 * b] + (m.beta[a - 1] * m.beta[b - 1]) / grhd2_metric::sq(m.alpha);
  bool sym = same_bits(m.gamma[1], m.gamma[3]) && same_bits(m.gamma[2], m.gamma[6]) &&
             same_bits(m.gamma[5], m.gamma[7]) && same_bits(gi[1], gi[3]) && same_bits(gi[2], gi[6]) &&
             same_bits(gi[5], gi[7]);
  const size_t n = (size_t)nij;
  C[CF_ALPHA * n + q] = m.alpha;
  for (int d = 0; d < 3; ++d) C[(CF_B1 + d) * n + q] = m.beta[d];
  const int sidx[6] = {0, 3, 6, 4, 7, 8};  // (1,1) (1,2) (1,3) (2,2) (2,3) (3,3)
  for (int s = 0; s < 6; ++s) {
    C[(CF_G11 + s) * n + q] = m.gamma[sidx[s]];
    C[(CF_I11 + s) * n + q] = gi[sidx[s]];
  }
  C[CF_SQG * n + q] = sqrt(m.det);
  for (int mu = 0; mu < 4; ++mu)
    for (int nu = mu; nu < 4; ++nu) {
      sym = sym && same_bits(m.gmunu[mu + 4 * nu], m.gmunu[nu + 4 * mu]) &&
            same_bits(ch[4 * mu + 16 * nu], ch[4 * nu + 16 * mu]);
      C[(CF_GM + sym4(mu, nu)) * n + q] = m.gmunu[mu + 4 * nu];
      C[(CF_CH0 + sym4(mu, nu)) * n + q] = ch[4 * mu + 16 * nu];
      for (int d = 0; d < 3; ++d) {
        sym = sym && same_bits(dg[mu + 4 * nu + 16 * d], dg[nu + 4 * mu + 16 * d]);
        C[(CF_DG + 10 * d + sym4(mu, nu)) * n + q] = dg[mu + 4 * nu + 16 * d];
      }
    }
  for (int mu = 0; mu < 4; ++mu) C[(CF_DLNA + mu) * n + q] = m.dlna[mu];
  for (int d = 0; d < 3; ++d) C[(CF_VA + d) * n + q] = m.beta[d] / m.alpha;
  if (!sym) atomicOr(status, MB_ASYM);
}

// face table of direction dir (1 x, 2 y, 3 z) with n faces, laid out as set_metric lays it
// out: x faces f = (i - 1) + (nx + 1)(j - 1), y faces f = (i - 1) + nx (j - 1) with
// j = 1..ny+1, z faces at the cell centres of the plane
__global__ void __launch_bounds__(128) k_metric_face(MetricGrid g, int dir, int n, double *__restrict__ T,
                                                     unsigned long long *status) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  double x, y;
  bool zero = false, pole = false;
  if (dir == 1) {
    const int i = f % (g.nx + 1) + 1, j = f / (g.nx + 1) + 1;
    x = g.x_min + (double)(i - 1) * g.dx;
    y = centre_y(g, j);
    // the cylindrical axis face (evolution.f90:69-71)
    zero = g.kind.geom == grhd2_metric::CYL && fabs(x) <= 64.0 * DBL_EPSILON;
  } else if (dir == 2) {
    const int i = f % g.nx + 1, j = f / g.nx + 1;
    x = centre_x(g, i);
    y = g.y_min + (double)(j - 1) * g.dy;
    // polar faces: sqrt(gamma) set to exactly zero (initialization.f90:356-363) and the
    // flux zeroed (evolution.f90:122-124)
    pole = (g.kind.geom == grhd2_metric::SPH || g.kind.geom == grhd2_metric::SPHEROID) &&
           fabs(sin(y)) <= 64.0 * DBL_EPSILON;
    zero = pole;
  } else {
    const int i = f % g.nx + 1, j = f / g.nx + 1;
    x = centre_x(g, i);
    y = centre_y(g, j);
  }
  grhd2_metric::MetricOut m;
  grhd2_metric::eval_metric(g.kind, x, y, false, m);
  const double *gm = m.gamma;
  bool sym = same_bits(gm[1], gm[3]) && same_bits(gm[2], gm[6]) && same_bits(gm[5], gm[7]);
  const size_t s = (size_t)n;
  T[FF_ALPHA * s + f] = m.alpha;
  T[FF_BETA_N * s + f] = m.beta[dir - 1];
  T[FF_G11 * s + f] = gm[0]; T[FF_G12 * s + f] = gm[3]; T[FF_G13 * s + f] = gm[6];
  T[FF_G22 * s + f] = gm[4]; T[FF_G23 * s + f] = gm[7]; T[FF_G33 * s + f] = gm[8];
  T[FF_SQG * s + f] = pole ? 0.0 : sqrt(m.det);
  const double gup_w = gamma_up_dd(gm, dir);
  T[FF_GUP * s + f] = gup_w;
  double cof[9], gup;
  const bool ok = face_frame(gm, dir, cof, &gup);
  for (int q = 0; q < 9; ++q) T[(FF_COF + q) * s + f] = cof[q];
  T[FF_FRAME_OK * s + f] = ok ? 1.0 : 0.0;
  T[FF_ZERO * s + f] = zero ? 1.0 : 0.0;
  if (!sym) atomicOr(status, MB_ASYM);
  if (ok && !same_bits(gup, gup_w)) atomicOr(status, MB_FRAME);
}

// single-precision copies of the tables for the mixed policy (round to nearest, as the host
// path's conversion)
__global__ void k_metric_to_float(const double *__restrict__ src, float *__restrict__ dst, size_t n) {
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    dst[q] = __double2float_rn(src[q]);
}

}  // namespace grhd
