// kernels.cuh -- sm_100a kernels of the per-stage path.
//
//   (face fluxes: flux.cuh)
//   cell_update      one thread per cell: flux divergence + sources in calc_rhs's order,
//                    SSP-RK3 stage combination (grhd2.f90:243-249) and con2prim
//                    (equations.f90:94), or the bare RHS for grhd2_gpu_calc_rhs
//   c2p_all/p2c_all  con2prim / prim2con sweeps
//   cfl_reduce       update_adaptive_dt's max-reductions (warp shuffles + atomics)
//   convert kernels  reference (Fortran AoS, ghosted) <-> device (SoA, interior) layouts
#pragma once

#include "cell.cuh"

namespace grhd {

// Riemann flux of one face given its interface states (resolve_riemann_problem)
template <class R>
__device__ __forceinline__ bool riemann(const Phys &P, const R (&qL)[NEQ], const R (&qR)[NEQ], int dir,
                                        const double *__restrict__ T, long long nf, long long f, R (&flux)[NEQ]) {
  const FaceMetric<R> m = load_face_metric<R>(T, nf, f);
  if (P.rs == RS_HLLC) {
    const FaceFrame<R> fr = load_face_frame<R>(T, nf, f);
    return hllc(P, qL, qR, dir, m, fr, flux);
  }
  hlle(P, qL, qR, dir, m, flux);
  return false;
}



// end of a step: t = t + dt, steps += 1 (grhd2.f90:229-230); deactivate grids that reached
// their final time or step limit
__global__ void k_advance_clocks(const GridDev *__restrict__ grids, int n) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  advance_clock(grids[g].clock);
}

template <class PT>
__global__ void k_c2p_all(const GridDev G, const Phys P, PT *__restrict__ Pout, double *__restrict__ UP,
                          unsigned long long *__restrict__ cnt) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const long long ij = c % ((long long)G.nx * G.ny);
  double cs[NEQ], pr[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) cs[v] = UP[v * G.pplane + c];
  const unsigned fl = cons_to_prim(P, load_cell_metric(G, ij), cs, pr);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) { UP[v * G.pplane + c] = cs[v]; Pout[v * G.pplane + c] = (PT)pr[v]; }
  c2p_count(cnt, fl);
}

// The same con2prim over every cell of a batch's scheme group in one launch (the block map
// of the cell update's tiles).  A 400x1x200 torus alone is one wave of ~18 us, bound by
// the latency of its torus cells' ~30 residual evaluations; launched together, the grids'
// waves overlap instead of running one after another.
template <class PT>
__global__ void __launch_bounds__(CELL_BS_STAGE, 8)
    k_c2p_batch(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  unsigned ia, jb, kc;
  if (!tile_item<7>(G.tiles[TILE_CELL], (unsigned)bm.first >> 7, threadIdx.x, (unsigned)G.nx, (unsigned)G.ny,
                    (unsigned)G.nz, ia, jb, kc))
    return;
  const CellIndex x = cell_index_of(G, ia, jb, kc);
  const long long ij = (long long)ia + (long long)G.nx * jb;
  double *__restrict__ UP = G.UP;
  PT *__restrict__ Pout = (PT *)G.P;
  const long long pl = G.pplane;
  double cs[NEQ], pr[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) cs[v] = UP[v * pl + x.c];
  const unsigned fl = cons_to_prim(G.phys, load_cell_metric(G, ij), cs, pr);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) { UP[v * pl + x.c] = cs[v]; Pout[v * pl + x.c] = (PT)pr[v]; }
  c2p_count(G.cnt, fl);
}

template <class PT>
__global__ void k_p2c_all(const GridDev G, const Phys P, const PT *__restrict__ Pin, double *__restrict__ UP) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const long long ij = c % ((long long)G.nx * G.ny);
  double q[NEQ], u[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) q[v] = (double)Pin[v * G.pplane + c];
  prim_to_cons(P, load_cell_metric(G, ij), q, u);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) UP[v * G.pplane + c] = u[v];
}

// update_adaptive_dt (evolution.f90:218-255): out[0..2] = max speeds as ordered bits,
// out[3] = invalid cells.  Speeds are finite and >= 0, so their IEEE bit patterns order
// like the values and the max is exact in any reduction order.
__global__ void k_cfl_reduce(const GridDev G, unsigned long long *__restrict__ out) {
  unsigned long long mx = 0, my = 0, mz = 0, bad = 0;
  for (long long ij = (long long)blockIdx.x * blockDim.x + threadIdx.x; ij < G.nij; ij += (long long)gridDim.x * blockDim.x) {
    const double *C = G.centre;
    const long long S = G.nij;
    const double a = C[CF_ALPHA * S + ij], b1 = C[CF_B1 * S + ij], b2 = C[CF_B2 * S + ij], b3 = C[CF_B3 * S + ij];
    const double i11 = C[CF_I11 * S + ij], i22 = C[CF_I22 * S + ij], i33 = C[CF_I33 * S + ij];
    if (!isfinite(a) || a <= 0.0 || !isfinite(b1) || !isfinite(b2) || !isfinite(b3) || !isfinite(i11) || i11 <= 0.0 ||
        (G.ny > 1 && (!isfinite(i22) || i22 <= 0.0)) || (G.nz > 1 && (!isfinite(i33) || i33 <= 0.0))) {
      bad += (unsigned long long)G.nz;
      continue;
    }
    const double vx = a * sqrt(i11) + fabs(b1);
    mx = max(mx, (unsigned long long)__double_as_longlong(vx));
    if (G.ny > 1) my = max(my, (unsigned long long)__double_as_longlong(a * sqrt(i22) + fabs(b2)));
    if (G.nz > 1) mz = max(mz, (unsigned long long)__double_as_longlong(a * sqrt(i33) + fabs(b3)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    my = max(my, __shfl_xor_sync(0xffffffffu, my, o));
    mz = max(mz, __shfl_xor_sync(0xffffffffu, mz, o));
    bad += __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], mx); atomicMax(&out[1], my); atomicMax(&out[2], mz);
    if (bad) atomicAdd(&out[3], bad);
  }
}

// ------------------------------------------------------------------------------------
// layout conversion: reference arrays (Fortran AoS) <-> device (SoA interior)
// ------------------------------------------------------------------------------------
struct FortranLayout {
  int nx, ny, nz, ng;
  __host__ __device__ long long pidx(int v, int i, int j, int k) const {  // p(v+1, i, j, k)
    const long long sx = 5, sy = 5LL * (nx + 2 * ng + 1), sz = sy * (ny + 2 * ng + 1);
    return v + sx * (i + ng) + sy * (j + ng) + sz * (k + ng);
  }
};

template <class PT>
__global__ void k_prims_in(const GridDev G, const double *__restrict__ pf, PT *__restrict__ Pout,
                           double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
  const FortranLayout L{G.nx, G.ny, G.nz, G.ng};
  const int i = (int)(c % G.nx) + 1;
  const long long r = c / G.nx;
  const int j = (int)(r % G.ny) + 1, k = (int)(r / G.ny) + 1;
#pragma unroll
  for (int v = 0; v < NEQ; ++v) Pout[v * G.pplane + c] = (PT)pf[L.pidx(v, i, j, k)];
  if (G.ng == 2) {  // the never-filled -nghost slabs (see state.cuh)
    if (i == 1) {
      const long long s = (j - 1) + (long long)G.ny * (k - 1), ns = (long long)G.ny * G.nz;
      for (int v = 0; v < NEQ; ++v) fx[v * ns + s] = pf[L.pidx(v, -G.ng, j, k)];
    }
    if (j == 1 && fy) {
      const long long s = (i - 1) + (long long)G.nx * (k - 1), ns = (long long)G.nx * G.nz;
      for (int v = 0; v < NEQ; ++v) fy[v * ns + s] = pf[L.pidx(v, i, -G.ng, k)];
    }
    if (k == 1 && fz) {
      const long long s = (i - 1) + (long long)G.nx * (j - 1), ns = (long long)G.nx * G.ny;
      for (int v = 0; v < NEQ; ++v) fz[v * ns + s] = pf[L.pidx(v, i, j, -G.ng)];
    }
  }
}

// interior cells and every ghost outside the domain in exactly one direction
template <class PT>
__global__ void k_prims_out(const GridDev G, const PT *__restrict__ Pin, double *__restrict__ pf) {
  const int NX = G.nx + 2 * G.ng + 1, NY = G.ny + 2 * G.ng + 1, NZ = G.nz + 2 * G.ng + 1;
  const long long n = (long long)NX * NY * NZ;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = (int)(t % NX) - G.ng;
  const long long r = t / NX;
  const int j = (int)(r % NY) - G.ng, k = (int)(r / NY) - G.ng;
  const bool oi = i < 1 || i > G.nx, oj = j < 1 || j > G.ny, ok = k < 1 || k > G.nz;
  if ((int)oi + (int)oj + (int)ok > 1) return;
  // index -nghost is never written by set_boundary_conditions (it keeps the caller's
  // value), except in the jet case, which resets every ghost to the ambient state
  if (G.case_id != 5 && (i == -G.ng || j == -G.ng || k == -G.ng)) return;
  double q[NEQ];
  if (oj) load_cell<2>(Pin, G, i, j, k, q);
  else if (ok) load_cell<3>(Pin, G, i, j, k, q);
  else load_cell<1>(Pin, G, i, j, k, q);
  const FortranLayout L{G.nx, G.ny, G.nz, G.ng};
#pragma unroll
  for (int v = 0; v < NEQ; ++v) pf[L.pidx(v, i, j, k)] = q[v];
}

// u(5,nx,ny,nz) AoS <-> SoA
// Conserved state between the reference's layout u(5, nx, ny, nz) (variable fastest: the
// upload/download staging and the checkpoint snapshot) and the SoA planes.  Launched with
// LAYOUT_BS threads per block, one cell each.  A block's LAYOUT_BS x 5 doubles (10 KB) are
// contiguous and start on a 16-byte boundary (a multiple of 256 cells x 40 bytes from a
// 16-byte aligned buffer, checked), so they move between HBM and shared memory as 128-bit
// vectors (ld/st.global.v2.f64), while each plane is read or written one coalesced row per
// variable.  Thread t's cell sits at s[5 t .. 5 t + 4] (stride 5 doubles: two-way bank
// conflicts at most).
constexpr int LAYOUT_BS = 256;
__global__ void __launch_bounds__(LAYOUT_BS) k_cons_in(const GridDev G, const double *__restrict__ uf,
                                                       double *__restrict__ U) {
  __shared__ __align__(16) double s[NEQ * LAYOUT_BS];
  const long long c0 = (long long)blockIdx.x * LAYOUT_BS;
  const int cells = (int)min((long long)LAYOUT_BS, G.ncell - c0);
  const int nd = cells * NEQ;
  const double *src = uf + c0 * NEQ;
  if (((uintptr_t)uf & 15u) == 0) {
    const double2 *src2 = reinterpret_cast<const double2 *>(src);
    double2 *s2 = reinterpret_cast<double2 *>(s);
    for (int q = (int)threadIdx.x; q < nd / 2; q += LAYOUT_BS) s2[q] = __ldg(&src2[q]);
    if ((nd & 1) && threadIdx.x == 0) s[nd - 1] = src[nd - 1];
  } else {
    for (int q = (int)threadIdx.x; q < nd; q += LAYOUT_BS) s[q] = src[q];
  }
  __syncthreads();
  const int t = (int)threadIdx.x;
  if (t >= cells) return;
#pragma unroll
  for (int v = 0; v < NEQ; ++v) U[v * G.pplane + c0 + t] = s[NEQ * t + v];
}
__global__ void __launch_bounds__(LAYOUT_BS) k_cons_out(const GridDev G, const double *__restrict__ U,
                                                        double *__restrict__ uf) {
  __shared__ __align__(16) double s[NEQ * LAYOUT_BS];
  const long long c0 = (long long)blockIdx.x * LAYOUT_BS;
  const int cells = (int)min((long long)LAYOUT_BS, G.ncell - c0);
  const int nd = cells * NEQ;
  const int t = (int)threadIdx.x;
  if (t < cells) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) s[NEQ * t + v] = U[v * G.pplane + c0 + t];
  }
  __syncthreads();
  double *dst = uf + c0 * NEQ;
  if (((uintptr_t)uf & 15u) == 0) {
    double2 *dst2 = reinterpret_cast<double2 *>(dst);
    const double2 *s2 = reinterpret_cast<const double2 *>(s);
    for (int q = t; q < nd / 2; q += LAYOUT_BS) dst2[q] = s2[q];
    if ((nd & 1) && t == 0) dst[nd - 1] = s[nd - 1];
  } else {
    for (int q = t; q < nd; q += LAYOUT_BS) dst[q] = s[q];
  }
}

// independent faces with explicit states (the Riemann entry point of the C-ABI)
template <class R>
__global__ void k_riemann_faces(const Phys P, int n, int dir, const double *__restrict__ qL, const double *__restrict__ qR,
                                const double *__restrict__ T, double *__restrict__ flux, int physical_only) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  R l[NEQ], r[NEQ], out[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) { l[v] = R(qL[5 * f + v]); r[v] = R(qR[5 * f + v]); }
  if (physical_only) {
    R u[NEQ];
    flux_and_cons(P, l, dir, load_face_metric<R>(T, n, f), out, u);
  } else {
    riemann(P, l, r, dir, T, n, f, out);
  }
#pragma unroll
  for (int v = 0; v < NEQ; ++v) flux[5 * f + v] = (double)out[v];
}

}  // namespace grhd
