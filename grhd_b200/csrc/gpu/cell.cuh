// cell.cuh -- per-cell device code of the stage update: metric sources, the RK stage
// combination and con2prim for one cell (cell_item), shared by the stage kernels and the
// persistent step kernel.
#pragma once

#include "common.cuh"

namespace grhd {

// ------------------------------------------------------------------------------------
// calc_sources (equations.f90:509-552) + calculate_stress_energy_tensor (metrics.f90:1251)
// ------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void sources(const GridDev &G, const Phys &P, long long ij, const double (&qd)[NEQ],
                                        R (&src)[NEQ]) {
#pragma unroll
  for (int n = 0; n < NEQ; ++n) src[n] = R(0);
  if (P.srhd) return;
  const R *__restrict__ C = centre_table<R>(G);
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
  uf[1] = W * (v[0] - ld(CF_VA));  // beta^i / alpha: per (i,j), rounded once (the same quotient)
  uf[2] = W * (v[1] - ld(CF_VA + 1));
  uf[3] = W * (v[2] - ld(CF_VA + 2));
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
  const unsigned mask = __match_any_sync(__activemask(), (unsigned long long)cnt);
  if (!__any_sync(mask, fl != 0u)) return;  // the common case: no floor, no failure
  const bool lead = (threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1);
  const unsigned flag[6] = {C2P_FLOOR_PRE, C2P_CAUSAL, C2P_BRENT, C2P_ROOT_FAIL, C2P_BAD_V, C2P_SANITISE};
  const int idx[6] = {CNT_FLOOR_PRE, CNT_CAUSAL, CNT_BRENT, CNT_ROOT_FAIL, CNT_BAD_V, CNT_SANITISE};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const unsigned tot = __reduce_add_sync(mask, (fl & flag[q]) ? 1u : 0u);
    if (tot && lead) atomicAdd(&cnt[idx[q]], (unsigned long long)tot);
  }
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

// One cell (ia, jb, kc), 0-based.  MODE 0 writes the RHS; 1..3 run the RK stage.  The
// mode is a run-time argument so a persistent kernel needs one copy of the code; the
// stage kernels pass a constant and the compiler folds it.
template <class R, class PT>
__device__ __forceinline__ void cell_item(const GridDev &G, unsigned ia, unsigned jb, unsigned kc, const int MODE) {
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

template <int MODE, class R, class PT>
__global__ void __launch_bounds__(128, cell_min_blocks<PT>())
    k_cell_update(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  unsigned ia, jb, kc;
  if (!tile_item<7>(G.tiles[TILE_CELL], (unsigned)bm.first >> 7, threadIdx.x, (unsigned)G.nx, (unsigned)G.ny,
                    (unsigned)G.nz, ia, jb, kc))
    return;
  cell_item<R, PT>(G, ia, jb, kc, MODE);
}

}  // namespace grhd
