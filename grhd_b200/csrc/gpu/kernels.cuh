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

#include "common.cuh"

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

// ------------------------------------------------------------------------------------
// calc_sources (equations.f90:509-552) + calculate_stress_energy_tensor (metrics.f90:1251)
// ------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void sources(const GridDev &G, const Phys &P, long long ij, const double (&qd)[NEQ],
                                        R (&src)[NEQ]) {
#pragma unroll
  for (int n = 0; n < NEQ; ++n) src[n] = R(0);
  if (P.srhd) return;
  const double *__restrict__ C = G.centre;
  const long long S = G.nij;
  auto ld = [&](int fld) { return R(__ldg(&C[fld * S + ij])); };
  const R alpha = ld(CF_ALPHA), sqg = ld(CF_SQG);
  FaceMetric<R> m;
  m.g11 = ld(CF_G11); m.g12 = ld(CF_G12); m.g13 = ld(CF_G13); m.g22 = ld(CF_G22); m.g23 = ld(CF_G23); m.g33 = ld(CF_G33);
  R q[NEQ];
#pragma unroll
  for (int n = 0; n < NEQ; ++n) q[n] = R(qd[n]);
  R v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]};
  const R vsq = cap_velocity(m, v, R(P.v_max));
  const R h = R(1) + R(P.g1) * q[EQ_PR] / q[EQ_DE];
  const R W = R(1) / sqrt(R(1) - vsq);
  R uf[4];
  uf[0] = W / alpha;
  uf[1] = W * (v[0] - ld(CF_B1) / alpha);
  uf[2] = W * (v[1] - ld(CF_B2) / alpha);
  uf[3] = W * (v[2] - ld(CF_B3) / alpha);
  R T[10];
#pragma unroll
  for (int mu = 0; mu <= 3; ++mu)
#pragma unroll
    for (int nu = mu; nu <= 3; ++nu)
      T[sym4(mu, nu)] = (q[EQ_DE] * h * uf[mu] * uf[nu]) + (q[EQ_PR] * ld(CF_GM + sym4(mu, nu)));
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R s = R(0);
#pragma unroll
    for (int mu = 0; mu <= 3; ++mu)
#pragma unroll
      for (int nu = 0; nu <= 3; ++nu) s = s + R(0.5) * T[sym4(mu, nu)] * ld(CF_DG + 10 * d + sym4(mu, nu));
    src[EQ_VX + d] = s;
  }
  R st = R(0);
#pragma unroll
  for (int mu = 0; mu <= 3; ++mu) {
    st = st + T[sym4(mu, 0)] * ld(CF_DLNA + mu);
#pragma unroll
    for (int nu = 0; nu <= 3; ++nu) st = st - T[sym4(mu, nu)] * ld(CF_CH0 + sym4(mu, nu));
  }
  src[EQ_PR] = st;
#pragma unroll
  for (int n = 0; n < NEQ; ++n) src[n] = src[n] * alpha * sqg;
  src[EQ_PR] = src[EQ_PR] * alpha;
}

__device__ __forceinline__ CellMetric load_cell_metric(const GridDev &G, long long ij) {
  const double *__restrict__ C = G.centre;
  const long long S = G.nij;
  CellMetric m;
  m.g11 = __ldg(&C[CF_G11 * S + ij]); m.g12 = __ldg(&C[CF_G12 * S + ij]); m.g13 = __ldg(&C[CF_G13 * S + ij]);
  m.g22 = __ldg(&C[CF_G22 * S + ij]); m.g23 = __ldg(&C[CF_G23 * S + ij]); m.g33 = __ldg(&C[CF_G33 * S + ij]);
  m.i11 = __ldg(&C[CF_I11 * S + ij]); m.i12 = __ldg(&C[CF_I12 * S + ij]); m.i13 = __ldg(&C[CF_I13 * S + ij]);
  m.i22 = __ldg(&C[CF_I22 * S + ij]); m.i23 = __ldg(&C[CF_I23 * S + ij]); m.i33 = __ldg(&C[CF_I33 * S + ij]);
  m.sqg = __ldg(&C[CF_SQG * S + ij]);
  return m;
}

__device__ __forceinline__ void c2p_count(unsigned long long *cnt, unsigned fl) {
  count_add(cnt, CNT_FLOOR_PRE, (fl & C2P_FLOOR_PRE) ? 1u : 0u);
  count_add(cnt, CNT_CAUSAL, (fl & C2P_CAUSAL) ? 1u : 0u);
  count_add(cnt, CNT_BRENT, (fl & C2P_BRENT) ? 1u : 0u);
  count_add(cnt, CNT_ROOT_FAIL, (fl & C2P_ROOT_FAIL) ? 1u : 0u);
  count_add(cnt, CNT_BAD_V, (fl & C2P_BAD_V) ? 1u : 0u);
  count_add(cnt, CNT_SANITISE, (fl & C2P_SANITISE) ? 1u : 0u);
}

// ------------------------------------------------------------------------------------
// cell update: RHS (evolution.f90:85-88, :137-139, :180-182) -> stage -> con2prim
// MODE 0 writes the RHS only; MODE 1..3 are the SSP-RK3 stages (stage 1 also copies
// up into u, the "u = up" of grhd2.f90:232).
// ------------------------------------------------------------------------------------
// Batched: block b works on grid map[b].grid, cell tile map[b].first / 128.
// Resident 128-thread blocks per SM the register allocation must allow.  The kernel waits
// on dependent FP64 chains (con2prim) and scattered table loads, so more warps in flight
// pay for a few spilled registers: measured on the 2.5D torus batch, 8 blocks (64
// registers) is fastest for FP64 and 6 (80 registers) for the mixed policy.
template <class PT>
constexpr int cell_min_blocks() { return sizeof(PT) == sizeof(double) ? 8 : 6; }

template <int MODE, class R, class PT>
__global__ void __launch_bounds__(128, cell_min_blocks<PT>())
    k_cell_update(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  unsigned ia, jb, kc;
  if (!tile_item<7>(G.tiles[TILE_CELL], (unsigned)bm.first >> 7, threadIdx.x, (unsigned)G.nx, (unsigned)G.ny,
                    (unsigned)G.nz, ia, jb, kc))
    return;
  const long long c = (long long)ia + (long long)G.nx * ((long long)jb + (long long)G.ny * kc);
  const Phys P = G.phys;
  PT *__restrict__ Pio = (PT *)G.P;
  const R *__restrict__ Fx = (const R *)G.F[0];
  const R *__restrict__ Fy = (const R *)G.F[1];
  const R *__restrict__ Fz = (const R *)G.F[2];
  double *__restrict__ U = G.U;
  double *__restrict__ UP = G.UP;
  double *__restrict__ rhs_out = G.RHS;
  const double dx = G.dx, dy = G.dy, dz = G.dz;
  double dt = 0.0;
  if (MODE != 0) {
    const GridClock ck = *G.clock;
    if (clock_skip(ck)) return;
    dt = clock_dt(ck);
  }
  unsigned long long *cnt = G.cnt;
  const int i0 = (int)ia, j0 = (int)jb, k0 = (int)kc;
  const long long ij = i0 + (long long)G.nx * j0;
  double q[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) q[v] = (double)Pio[v * G.pplane + c];
  R src[NEQ];
  sources<R>(G, P, ij, q, src);
  double rhs[NEQ];
  {
    const long long nfx = (long long)(G.nx + 1) * G.ny * G.nz;
    const long long fx = i0 + (long long)(G.nx + 1) * (j0 + (long long)G.ny * k0);
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      const R a = Fx[v * nfx + fx + 1], b = Fx[v * nfx + fx];
      rhs[v] = (double)(-(a - b) / R(dx) + src[v]);
    }
  }
  if (G.ny > 1) {
    const long long nfy = (long long)G.nx * (G.ny + 1) * G.nz;
    const long long fy = i0 + (long long)G.nx * (j0 + (long long)(G.ny + 1) * k0);
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      const R a = Fy[v * nfy + fy + G.nx], b = Fy[v * nfy + fy];
      rhs[v] = (double)(R(rhs[v]) - (a - b) / R(dy));
    }
  }
  if (G.nz > 1) {
    const long long nfz = (long long)G.nx * G.ny * (G.nz + 1);
    const long long fz = i0 + (long long)G.nx * (j0 + (long long)G.ny * k0);
    const long long st = (long long)G.nx * G.ny;
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      const R a = Fz[v * nfz + fz + st], b = Fz[v * nfz + fz];
      rhs[v] = (double)(R(rhs[v]) - (a - b) / R(dz));
    }
  }
  if (MODE == 0) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) rhs_out[v * G.pplane + c] = rhs[v];
    return;
  }
  double cs[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) {
    const double up = UP[v * G.pplane + c];
    double nv;
    if (MODE == 1) {
      U[v * G.pplane + c] = up;  // u = up (grhd2.f90:232)
      nv = up + rhs[v] * dt;
    } else if (MODE == 2) {
      nv = 0.75 * U[v * G.pplane + c] + 0.25 * (up + rhs[v] * dt);
    } else {
      nv = (U[v * G.pplane + c] + 2.0 * (up + rhs[v] * dt)) / 3.0;
    }
    cs[v] = nv;
  }
  const CellMetric cm = load_cell_metric(G, ij);
  // mixed policy: seed the root finder with the Lorentz factor of the current primitives
  double W_seed = 0.0;
  if (sizeof(PT) == sizeof(float)) {
    const double a = q[EQ_VX], b = q[EQ_VY], d = q[EQ_VZ];
    const double vsq = cm.g11 * a * a + cm.g22 * b * b + cm.g33 * d * d +
                       2.0 * (cm.g12 * a * b + cm.g13 * a * d + cm.g23 * b * d);
    W_seed = vsq < 1.0 ? 1.0 / sqrt(1.0 - vsq) : 0.0;
  }
  double pr[NEQ];
  const unsigned fl = cons_to_prim(P, cm, cs, pr, W_seed);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) {
    UP[v * G.pplane + c] = cs[v];
    Pio[v * G.pplane + c] = (PT)pr[v];
  }
  c2p_count(cnt, fl);
}

// end of a step: t = t + dt, steps += 1 (grhd2.f90:229-230); deactivate grids that reached
// their final time or step limit
__global__ void k_advance_clocks(const GridDev *__restrict__ grids, int n) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  GridClock *c = grids[g].clock;
  if (c->mode == 1) {
    if (!c->active) return;
    c->t = c->t + clock_dt(*c);
    c->steps += 1;
    c->active = c->t < c->final_time && (c->max_steps < 0 || c->steps < c->max_steps);
  } else {
    c->steps += 1;
  }
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
__global__ void k_cons_in(const GridDev G, const double *__restrict__ uf, double *__restrict__ U) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
#pragma unroll
  for (int v = 0; v < NEQ; ++v) U[v * G.pplane + c] = uf[5 * c + v];
}
__global__ void k_cons_out(const GridDev G, const double *__restrict__ U, double *__restrict__ uf) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= G.ncell) return;
#pragma unroll
  for (int v = 0; v < NEQ; ++v) uf[5 * c + v] = U[v * G.pplane + c];
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
