// diag.cuh -- diagnostics of the resident state as device reductions, so the state does
// not leave the GPU at diagnostic strides:
//   total mass        grhd2.f90:283-301   sum u(D) dx dy dz
//   accretion rate    output.f90:951-992  -sum_{j,k} up(D) (alpha v^x - beta^x) dy dz at i = idx_probe
//   PPI modes         output.f90:995-1049 per-k azimuthal mass of cells with rho > 1e3 rho_floor
//                                         (the host forms the m = 1..4 Fourier sums)
//   global diagnostics output.f90:1052-1125 masses, angular momentum, extrema, counts
// Every per-cell term is evaluated with the reference's operation order; the sums are
// reduced in a fixed tree (fixed block count, warp shuffles, one final block), so a result
// is reproducible run to run, and differs from a serial sum only by summation order.
#pragma once

#include "state.cuh"

namespace grhd {

constexpr int DIAG_BS = 256;
constexpr int DIAG_BLOCKS = 592;  // 4 x 148 SMs

// sum over the block (deterministic tree); result valid in thread 0
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[DIAG_BS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < DIAG_BS / 32 ? ws[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}
__device__ __forceinline__ double block_min(double v) {
  __shared__ double ws[DIAG_BS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < DIAG_BS / 32 ? ws[lane] : DBL_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  return v;
}
__device__ __forceinline__ double block_max(double v) {
  __shared__ double ws[DIAG_BS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < DIAG_BS / 32 ? ws[lane] : -DBL_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  return v;
}

// partial results of the global diagnostics
struct DiagGlobal {
  double mass, disk, angmom, rho_min, p_min, rho_max, p_max, vsq_max;
  double atmosphere, invalid;  // counts (exact in double below 2^53)
};

__device__ __forceinline__ DiagGlobal diag_reduce(DiagGlobal a) {
  DiagGlobal r;
  r.mass = block_sum(a.mass);
  r.disk = block_sum(a.disk);
  r.angmom = block_sum(a.angmom);
  r.rho_min = block_min(a.rho_min);
  r.p_min = block_min(a.p_min);
  r.rho_max = block_max(a.rho_max);
  r.p_max = block_max(a.p_max);
  r.vsq_max = block_max(a.vsq_max);
  r.atmosphere = block_sum(a.atmosphere);
  r.invalid = block_sum(a.invalid);
  return r;
}

// calc_global_diagnostics over the cells, grid-stride; one partial per block
template <class PT>
__global__ void __launch_bounds__(DIAG_BS) k_diag_global(const GridDev G, const PT *__restrict__ P,
                                                         const double *__restrict__ UP, DiagGlobal *__restrict__ part) {
  const double cell_volume = G.dx * G.dy * G.dz;
  const double density_cut = 1.0e3 * G.rho_floor;
  DiagGlobal a{0.0, 0.0, 0.0, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, 0.0, 0.0, 0.0};
  for (long long c = (long long)blockIdx.x * DIAG_BS + threadIdx.x; c < G.ncell; c += (long long)gridDim.x * DIAG_BS) {
    const long long ij = c % G.nij;
    const double rho = (double)P[c], pres = (double)P[G.pplane + c];
    const double v[3] = {(double)P[2 * G.pplane + c], (double)P[3 * G.pplane + c], (double)P[4 * G.pplane + c]};
    const double *T = G.centre;
    const long long S = G.nij;
    const int gi[3][3] = {{CF_G11, CF_G12, CF_G13}, {CF_G12, CF_G22, CF_G23}, {CF_G13, CF_G23, CF_G33}};
    double v_sq = 0.0;  // output.f90:1081-1086, loop order ii, jj
#pragma unroll
    for (int ii = 0; ii < 3; ++ii)
#pragma unroll
      for (int jj = 0; jj < 3; ++jj) v_sq = v_sq + T[gi[ii][jj] * S + ij] * v[ii] * v[jj];
    if (!isfinite(rho) || !isfinite(pres) || !isfinite(v_sq) || rho <= 0.0 || pres <= 0.0 || v_sq < 0.0 ||
        v_sq >= 1.0)
      a.invalid += 1.0;
    if (isfinite(rho)) { a.rho_min = fmin(a.rho_min, rho); a.rho_max = fmax(a.rho_max, rho); }
    if (isfinite(pres)) { a.p_min = fmin(a.p_min, pres); a.p_max = fmax(a.p_max, pres); }
    if (isfinite(v_sq)) a.vsq_max = fmax(a.vsq_max, v_sq);
    const double D = UP[c];
    a.mass += D * cell_volume;
    a.angmom += UP[4 * G.pplane + c] * cell_volume;
    if (rho > density_cut) a.disk += D * cell_volume;
    else a.atmosphere += 1.0;
  }
  const DiagGlobal r = diag_reduce(a);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void __launch_bounds__(DIAG_BS) k_diag_global_final(const DiagGlobal *__restrict__ part, int n,
                                                               DiagGlobal *__restrict__ out) {
  DiagGlobal a{0.0, 0.0, 0.0, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < n; b += DIAG_BS) {
    const DiagGlobal p = part[b];
    a.mass += p.mass; a.disk += p.disk; a.angmom += p.angmom;
    a.rho_min = fmin(a.rho_min, p.rho_min); a.p_min = fmin(a.p_min, p.p_min);
    a.rho_max = fmax(a.rho_max, p.rho_max); a.p_max = fmax(a.p_max, p.p_max);
    a.vsq_max = fmax(a.vsq_max, p.vsq_max);
    a.atmosphere += p.atmosphere; a.invalid += p.invalid;
  }
  const DiagGlobal r = diag_reduce(a);
  if (threadIdx.x == 0) *out = r;
}

// sum of u(D) dx dy dz (grhd2.f90:296: total_mass + u(eq_de) * dx * dy * dz)
__global__ void __launch_bounds__(DIAG_BS) k_diag_mass(const GridDev G, const double *__restrict__ U,
                                                       double *__restrict__ part) {
  double a = 0.0;
  for (long long c = (long long)blockIdx.x * DIAG_BS + threadIdx.x; c < G.ncell; c += (long long)gridDim.x * DIAG_BS)
    a += U[c] * G.dx * G.dy * G.dz;
  const double r = block_sum(a);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void __launch_bounds__(DIAG_BS) k_sum_final(const double *__restrict__ part, int n, double *__restrict__ out) {
  double a = 0.0;
  for (int b = threadIdx.x; b < n; b += DIAG_BS) a += part[b];
  const double r = block_sum(a);
  if (threadIdx.x == 0) *out = r;
}

// accretion rate through the shell of cells i = idx (0-based), one block
template <class PT>
__global__ void __launch_bounds__(DIAG_BS) k_diag_mdot(const GridDev G, const PT *__restrict__ P,
                                                       const double *__restrict__ UP, int idx, double *__restrict__ out) {
  double a = 0.0;
  const long long n = (long long)G.ny * G.nz;
  for (long long s = threadIdx.x; s < n; s += DIAG_BS) {
    const long long j = s % G.ny, k = s / G.ny;
    const long long c = idx + (long long)G.nx * (j + (long long)G.ny * k);
    const long long ij = idx + (long long)G.nx * j;
    const double alpha = G.centre[(long long)CF_ALPHA * G.nij + ij];
    const double beta1 = G.centre[(long long)CF_B1 * G.nij + ij];
    const double v_eff = alpha * (double)P[2 * G.pplane + c] - beta1;
    a += UP[c] * v_eff * G.dy * G.dz;
  }
  const double r = block_sum(a);
  if (threadIdx.x == 0) *out = -r;
}

// mass of the cells above the density cut in each k-plane (one block per k)
template <class PT>
__global__ void __launch_bounds__(DIAG_BS) k_diag_azimuthal(const GridDev G, const PT *__restrict__ P,
                                                            const double *__restrict__ UP, double *__restrict__ out) {
  const double cell_volume = G.dx * G.dy * G.dz;
  const double density_cut = 1.0e3 * G.rho_floor;
  const long long k = blockIdx.x;
  double a = 0.0;
  for (long long ij = threadIdx.x; ij < G.nij; ij += DIAG_BS) {
    const long long c = ij + G.nij * k;
    if ((double)P[c] > density_cut) a += UP[c] * cell_volume;
  }
  const double r = block_sum(a);
  if (threadIdx.x == 0) out[k] = r;
}

// calc_gw_strain (output.f90:852-948): Finn-Evans stresses of the cells outside the horizon
// with the numerical atmosphere subtracted.  tab = r(nx) | sin th, cos th (ny) | sin ph,
// cos ph (nz), evaluated on the host with the C library so every per-cell term equals the
// reference's.  One partial (Ixx, Iyy, Ixy) per block.
template <class PT>
__global__ void __launch_bounds__(DIAG_BS) k_diag_gw(const GridDev G, const PT *__restrict__ P,
                                                     const double *__restrict__ tab, int use_log_r, double r_h,
                                                     double bh_mass, double spin, double *__restrict__ part) {
  const double *rr = tab, *sth = tab + G.nx, *cth = sth + G.ny, *sph = cth + G.ny, *cph = sph + G.nz;
  double ixx = 0.0, iyy = 0.0, ixy = 0.0;
  for (long long c = (long long)blockIdx.x * DIAG_BS + threadIdx.x; c < G.ncell; c += (long long)gridDim.x * DIAG_BS) {
    const long long ij = c % G.nij, i = ij % G.nx, j = ij / G.nx, k = c / G.nij;
    const double r = rr[i];
    if (r <= r_h) continue;
    double rho = (double)P[c] - G.rho_floor, pres = (double)P[G.pplane + c] - G.p_floor;
    if (!(rho > 0.0)) rho = 0.0;
    if (!(pres > 0.0)) pres = 0.0;
    if (rho <= 0.0 && pres <= 0.0) continue;
    const double alpha = G.centre[(long long)CF_ALPHA * G.nij + ij];
    double rates[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      rates[d] = alpha * (double)P[(2 + d) * G.pplane + c] - G.centre[(long long)(CF_B1 + d) * G.nij + ij];
    if (use_log_r) rates[0] = r * rates[0];
    const double st = sth[j], ct = cth[j], sp = sph[k], cp = cph[k];
    double pos[3], vel[3];
    if (fabs(st) <= 64.0 * DBL_EPSILON) {
      pos[0] = 0.0; pos[1] = 0.0; pos[2] = copysign(fabs(r), ct);
    } else {
      pos[0] = (r * cp - spin * sp) * st;
      pos[1] = (r * sp + spin * cp) * st;
      pos[2] = r * ct;
    }
    vel[0] = rates[0] * cp * st + rates[1] * (r * cp - spin * sp) * ct - rates[2] * (r * sp + spin * cp) * st;
    vel[1] = rates[0] * sp * st + rates[1] * (r * sp + spin * cp) * ct + rates[2] * (r * cp - spin * sp) * st;
    vel[2] = rates[0] * ct - r * rates[1] * st;
    const double sigma = r * r + spin * spin * (ct * ct);
    const double jac = sigma * st;
    const double dV = jac * (use_log_r ? r : 1.0) * G.dx * G.dy * G.dz;
    const double r2 = pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2];
    const double mr3 = bh_mass / (r2 * sqrt(r2));
    ixx += (2.0 * rho * (vel[0] * vel[0]) + 2.0 * pres - 2.0 * rho * mr3 * (pos[0] * pos[0])) * dV;
    iyy += (2.0 * rho * (vel[1] * vel[1]) + 2.0 * pres - 2.0 * rho * mr3 * (pos[1] * pos[1])) * dV;
    ixy += (2.0 * rho * vel[0] * vel[1] - 2.0 * rho * mr3 * pos[0] * pos[1]) * dV;
  }
  ixx = block_sum(ixx);
  iyy = block_sum(iyy);
  ixy = block_sum(ixy);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = ixx;
    part[3 * blockIdx.x + 1] = iyy;
    part[3 * blockIdx.x + 2] = ixy;
  }
}

__global__ void __launch_bounds__(DIAG_BS) k_sum3_final(const double *__restrict__ part, int n, double *__restrict__ out) {
  double a[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < n; b += DIAG_BS)
#pragma unroll
    for (int q = 0; q < 3; ++q) a[q] += part[3 * b + q];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double r = block_sum(a[q]);
    if (threadIdx.x == 0) out[q] = r;
  }
}

// write_vtk_cell_data (output.f90:398-453): the 7 cell fields of a VTK frame exactly as
// the file holds them -- rho, p, v^r (x r_scale on log-r grids), v^theta, v^phi, the lapse,
// beta^r (x r_scale) -- each nx*ny*nz doubles in i-fastest order, big-endian.
__device__ __forceinline__ unsigned long long bswap64(unsigned long long x) {
  const unsigned lo = (unsigned)x, hi = (unsigned)(x >> 32);
  const unsigned slo = __byte_perm(lo, 0, 0x0123), shi = __byte_perm(hi, 0, 0x0123);
  return ((unsigned long long)slo << 32) | shi;
}
template <class PT>
__global__ void __launch_bounds__(DIAG_BS) k_vtk_cells(const GridDev G, const PT *__restrict__ P,
                                                       const double *__restrict__ r_scale,
                                                       unsigned long long *__restrict__ out) {
  for (long long c = (long long)blockIdx.x * DIAG_BS + threadIdx.x; c < G.ncell; c += (long long)gridDim.x * DIAG_BS) {
    const long long ij = c % G.nij, i = ij % G.nx;
    double f[7];
#pragma unroll
    for (int v = 0; v < 5; ++v) f[v] = (double)P[v * G.pplane + c];
    f[5] = G.centre[(long long)CF_ALPHA * G.nij + ij];
    f[6] = G.centre[(long long)CF_B1 * G.nij + ij];
    if (r_scale) {
      f[2] = f[2] * r_scale[i];
      f[6] = f[6] * r_scale[i];
    }
#pragma unroll
    for (int q = 0; q < 7; ++q) out[q * G.ncell + c] = bswap64(__double_as_longlong(f[q]));
  }
}

}  // namespace grhd
