// cell.cuh -- per-cell device code of the stage update: metric sources, the RK stage
// combination and con2prim for one cell (cell_core), fed directly from global memory
// (cell_item: the persistent step kernel, and the stage kernel without a table slice) or
// through shared-memory staging (k_cell_update).
#pragma once

#include "common.cuh"

namespace grhd {

// Field fld of one (i,j) column of a centre table: from global memory, or from a block's
// shared-memory slice of the table (SliceCol, below).
template <class T>
struct GlobalCol {
  const T *__restrict__ C;
  long long S, ij;
  __device__ __forceinline__ T operator()(int fld) const { return __ldg(&C[fld * S + ij]); }
};
template <class T>
__device__ __forceinline__ GlobalCol<T> global_col(const T *C, const GridDev &G, long long ij) {
  return GlobalCol<T>{C, G.nij, ij};
}

// ------------------------------------------------------------------------------------
// calc_sources (equations.f90:509-552) + calculate_stress_energy_tensor (metrics.f90:1251)
// ------------------------------------------------------------------------------------
// Under the mixed policy (R = float) the contraction of T^{mu nu} with the metric
// derivatives runs in FP32, while the lapse and sqrt(gamma) factors -- the time component
// of the four-velocity W / alpha and the closing alpha sqrt(gamma) (alpha) scaling of
// equations.f90:550-551, which grow steep near the horizon -- are applied in FP64 from the
// FP64 centre table (alpha64, sqg64) in every cell.  The result is FP64 in both policies.
template <class R, class Col>
__device__ __forceinline__ void sources(const Phys &P, const Col &col, const double (&qd)[NEQ], double (&out)[NEQ],
                                        double alpha64, double sqg64) {
#pragma unroll
  for (int n = 0; n < NEQ; ++n) out[n] = 0.0;
  if (P.srhd) return;
  auto ld = [&](int fld) { return R(col(fld)); };
  constexpr bool mixed = sizeof(R) == sizeof(float);
  R src[NEQ] = {R(0), R(0), R(0), R(0), R(0)};  // D has no source
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
  uf[0] = mixed ? R((double)W / alpha64) : W / alpha;
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
  if constexpr (mixed) {
#pragma unroll
    for (int n = 0; n < NEQ; ++n) out[n] = (double)src[n] * alpha64 * sqg64;
    out[EQ_PR] = out[EQ_PR] * alpha64;
  } else {
#pragma unroll
    for (int n = 0; n < NEQ; ++n) src[n] = src[n] * alpha * sqg;
    src[EQ_PR] = src[EQ_PR] * alpha;
#pragma unroll
    for (int n = 0; n < NEQ; ++n) out[n] = (double)src[n];
  }
}

template <class Col>
__device__ __forceinline__ CellMetric load_cell_metric(const Col &C) {
  CellMetric m;
  m.g11_ = C(CF_G11); m.g12_ = C(CF_G12); m.g13_ = C(CF_G13);
  m.g22_ = C(CF_G22); m.g23_ = C(CF_G23); m.g33_ = C(CF_G33);
  m.i11_ = C(CF_I11); m.i12_ = C(CF_I12); m.i13_ = C(CF_I13);
  m.i22_ = C(CF_I22); m.i23_ = C(CF_I23); m.i33_ = C(CF_I33);
  m.sqg_ = C(CF_SQG);
  return m;
}

__device__ __forceinline__ CellMetric load_cell_metric(const GridDev &G, long long ij) {
  return load_cell_metric(global_col(G.centre, G, ij));
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
// pay for a few spilled registers: measured on the 2.5D and 3D torus batches, 8 blocks
// (64 registers) is fastest for FP64 (6: -4 %, 4: -14 %) and 5 (96 registers, a third of
// the spills of 6) for the mixed policy (6: -1 %, 4, 7 and 8 slower).
template <class PT>
constexpr int cell_min_blocks() { return sizeof(PT) == sizeof(double) ? 8 : 5; }

// cp.async (sm_80+ asynchronous global->shared copy, cp-size 4, 8 or 16 bytes) and its
// commit/wait; a thread waits for its own groups only.
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- the block's slice of a centre table ------------------------------------------------
// Cell tiles of grids with a k extent are 32 cells along i x 4 along k, so the four warps
// of a block share 32 (i,j) columns.  The block copies the NCF fields of those columns
// into shared memory once ([NCF][32], with cp.async) and every thread reads its column
// from there: ~70 table loads per cell that would otherwise go to L1/L2.
constexpr int SLICE_COLS = 32;
static_assert(SLICE_COLS == 32, "stage_slice copies one column per lane of a warp");
template <class T>
__host__ __device__ constexpr size_t slice_bytes() { return (size_t)NCF * SLICE_COLS * sizeof(T); }
template <class T>
struct SliceCol {
  const T *s;
  unsigned lane;
  __device__ __forceinline__ T operator()(int fld) const { return s[fld * SLICE_COLS + lane]; }
};
// a cell's metric read field by field from a table column where con2prim uses it (for a
// column in shared memory: no registers held across the root finder)
template <class Col>
struct ColMetric {
  Col c;
  __device__ __forceinline__ double g11() const { return c(CF_G11); }
  __device__ __forceinline__ double g12() const { return c(CF_G12); }
  __device__ __forceinline__ double g13() const { return c(CF_G13); }
  __device__ __forceinline__ double g22() const { return c(CF_G22); }
  __device__ __forceinline__ double g23() const { return c(CF_G23); }
  __device__ __forceinline__ double g33() const { return c(CF_G33); }
  __device__ __forceinline__ double i11() const { return c(CF_I11); }
  __device__ __forceinline__ double i12() const { return c(CF_I12); }
  __device__ __forceinline__ double i13() const { return c(CF_I13); }
  __device__ __forceinline__ double i22() const { return c(CF_I22); }
  __device__ __forceinline__ double i23() const { return c(CF_I23); }
  __device__ __forceinline__ double i33() const { return c(CF_I33); }
  __device__ __forceinline__ double sqg() const { return c(CF_SQG); }
};
// the metric con2prim works with: loaded into registers from global memory, read in place
// from a shared-memory slice
template <class T>
__device__ __forceinline__ CellMetric metric_of(const GlobalCol<T> &c) { return load_cell_metric(c); }
// A global table column whose con2prim metric is read field by field where used (the
// mixed cell update: its registers go to the staged inputs; measured +7 % on the 2.5D
// torus batch against loading the 13 fields up front)
template <class T>
struct LazyCol : GlobalCol<T> {};
template <class T>
__device__ __forceinline__ ColMetric<LazyCol<T>> metric_of(const LazyCol<T> &c) { return ColMetric<LazyCol<T>>{c}; }
template <class T>
__device__ __forceinline__ ColMetric<SliceCol<T>> metric_of(const SliceCol<T> &c) { return ColMetric<SliceCol<T>>{c}; }
// whether the block's warps share their (i,j) columns (the tile layout above)
__device__ __forceinline__ bool cell_tile_sliced(const GridDev &G) {
  return G.nz > 1 && G.tiles[TILE_CELL].lx == 5 && G.tiles[TILE_CELL].ly == 0;
}
// every thread of the block takes part: a thread copies column `lane` of the fields
// warp, warp + W, ... (W warps in the block), walking both pointers; columns beyond nx are
// left unset (no cell reads them)
template <class T>
__device__ __forceinline__ void stage_slice(T *slice, const T *C, const GridDev &G, unsigned i0, unsigned j) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const unsigned ncols = min((unsigned)SLICE_COLS, (unsigned)G.nx - i0);
  if (lane < ncols) {
    const T *src = C + ((long long)warp * G.nij + (long long)i0 + (long long)G.nx * j + lane);
    T *dst = slice + warp * SLICE_COLS + lane;
    const long long src_step = (long long)nwarps * G.nij;
    const unsigned dst_step = nwarps * SLICE_COLS;
#pragma unroll 4
    for (unsigned fld = warp; fld < (unsigned)NCF; fld += nwarps) {
      cp_async<sizeof(T)>(dst, src);
      src += src_step;
      dst += dst_step;
    }
  }
  cp_async_commit();
}

// Where cell_core reads a cell's streamed inputs: the primitives, the two faces of each
// active direction, and up, u.  DirectIn loads them from global memory where they are
// used; StagedIn (below) has them copied into shared memory ahead of use.
struct CellIndex {
  long long c;     // cell index in the state planes
  unsigned i, j, k;
};
__device__ __forceinline__ CellIndex cell_index_of(const GridDev &G, unsigned ia, unsigned jb, unsigned kc) {
  return CellIndex{(long long)ia + (long long)G.nx * ((long long)jb + (long long)G.ny * kc), ia, jb, kc};
}
// lower face of the cell along direction d (0..2), the face count, the upper face's offset
__device__ __forceinline__ long long face_lo(const GridDev &G, const CellIndex &x, int d) {
  if (d == 0) return x.i + (long long)(G.nx + 1) * (x.j + (long long)G.ny * x.k);
  if (d == 1) return x.i + (long long)G.nx * (x.j + (long long)(G.ny + 1) * x.k);
  return x.i + (long long)G.nx * (x.j + (long long)G.ny * x.k);
}
__device__ __forceinline__ long long face_n(const GridDev &G, int d) {
  if (d == 0) return (long long)(G.nx + 1) * G.ny * G.nz;
  if (d == 1) return (long long)G.nx * (G.ny + 1) * G.nz;
  return (long long)G.nx * G.ny * (G.nz + 1);
}
__device__ __forceinline__ long long face_up(const GridDev &G, int d) {
  return d == 0 ? 1LL : (d == 1 ? (long long)G.nx : (long long)G.nx * G.ny);
}

template <class R, class PT, class ColR = GlobalCol<R>, class Col64 = GlobalCol<double>>
struct DirectIn {
  const GridDev &G;
  const CellIndex &x;
  ColR cr;     // the centre table of arithmetic type R (sources)
  Col64 c64;   // the FP64 centre table (con2prim metric)
  __device__ __forceinline__ void wait_prims() const {}
  __device__ __forceinline__ void wait_fluxes() const {}
  __device__ __forceinline__ void wait_state() const {}
  __device__ __forceinline__ const ColR &table_r() const { return cr; }
  __device__ __forceinline__ const Col64 &table64() const { return c64; }
  __device__ __forceinline__ double prim(int v) const { return (double)((const PT *)G.P)[v * G.pplane + x.c]; }
  __device__ __forceinline__ R flux(int d, int upper, int v) const {
    return ((const R *)G.F[d])[v * face_n(G, d) + face_lo(G, x, d) + (upper ? face_up(G, d) : 0)];
  }
  __device__ __forceinline__ double up(int v) const { return G.UP[v * G.pplane + x.c]; }
  __device__ __forceinline__ double u(int v) const { return G.U[v * G.pplane + x.c]; }
};

// Seed of the mixed policy's root finder: the Lorentz factor of the cell's primitives at
// the start of the stage (re-read from the cell's inputs when a cell reaches the root
// finder; 0, no seed, for v^2 >= 1).
template <class In, class CM>
struct PrimSeed {
  static constexpr bool seeded = true;
  const In &in;
  const CM &cm;
  __device__ __forceinline__ double operator()() const {
    const double a = in.prim(EQ_VX), b = in.prim(EQ_VY), d = in.prim(EQ_VZ);
    const double vsq = cm.g11() * a * a + cm.g22() * b * b + cm.g33() * d * d +
                       2.0 * (cm.g12() * a * b + cm.g13() * a * d + cm.g23() * b * d);
    return vsq < 1.0 ? rcp_mixed(sqrt(1.0 - vsq)) : 0.0;
  }
};

// One cell (ia, jb, kc), 0-based.  MODE 0 writes the RHS; 1..3 run the RK stage.  The
// mode is a run-time argument so a persistent kernel needs one copy of the code; the
// stage kernels pass a constant and the compiler folds it.  The clock has been checked
// by the caller (dt: the grid's step, 0 in MODE 0).
// ---- compensated RK3 accumulation (mixed policy with carries) ------------------------
// The state is a double-double: up + carry (and u + carry), the carry holding what the FP64
// rounding of each stage combination dropped.  Error-free transformations: Knuth's TwoSum
// (s = a + b exactly as s + e) and the FMA form of the exact product (p + e = a b).
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
// (ah, al) + (bh, bl), renormalised so that |l| <= ulp(h) / 2
__device__ __forceinline__ void dd_add(double ah, double al, double bh, double bl, double &h, double &l) {
  double s, e;
  two_sum(ah, bh, s, e);
  e = e + (al + bl);
  h = s + e;
  l = e - (h - s);
}
// (ah, al) * b
__device__ __forceinline__ void dd_mul(double ah, double al, double b, double &h, double &l) {
  const double p = ah * b;
  const double e = fma(ah, b, -p) + al * b;
  h = p + e;
  l = e - (h - p);
}
__device__ __forceinline__ double load_carry(const GridDev &G, const void *C, long long i) {
  return G.carry == 1 ? ((const double *)C)[i] : (double)((const float *)C)[i];
}
__device__ __forceinline__ void store_carry(const GridDev &G, void *C, long long i, double x) {
  if (G.carry == 1) ((double *)C)[i] = x;
  else ((float *)C)[i] = (float)x;
}
// The SSP-RK3 combination of grhd2.f90:243-249 in double-double arithmetic: rhs*dt with its
// rounding error, up + rhs*dt, then u = up (stage 1), 0.75 u + 0.25 (...) (stage 2) or
// (u + 2 (...)) / 3 (stage 3).  hi goes to con2prim as the stage's FP64 state, lo to the
// carry.
template <class In>
__device__ __forceinline__ void rk_stage_compensated(const GridDev &G, long long c, int MODE, double dt, const In &in,
                                                     const double (&rhs)[NEQ], double (&hi)[NEQ], double (&lo)[NEQ]) {
#pragma unroll
  for (int v = 0; v < NEQ; ++v) {
    const long long k = v * G.pplane + c;
    const double up = in.up(v), upl = load_carry(G, G.UPc, k);
    const double d = rhs[v] * dt, dl = fma(rhs[v], dt, -d);
    double th, tl;
    dd_add(up, upl, d, dl, th, tl);  // up + rhs*dt
    if (MODE == 1) {
      G.U[k] = up;  // u = up (grhd2.f90:232), carry included
      store_carry(G, G.Uc, k, upl);
      hi[v] = th;
      lo[v] = tl;
    } else if (MODE == 2) {
      double ah, al, bh, bl;
      dd_mul(in.u(v), load_carry(G, G.Uc, k), 0.75, ah, al);
      dd_mul(th, tl, 0.25, bh, bl);
      dd_add(ah, al, bh, bl, hi[v], lo[v]);
    } else {
      double sh, sl;
      dd_add(in.u(v), load_carry(G, G.Uc, k), 2.0 * th, 2.0 * tl, sh, sl);
      const double q = sh / 3.0;
      const double ql = (fma(-q, 3.0, sh) + sl) / 3.0;
      hi[v] = q + ql;
      lo[v] = ql - (hi[v] - q);
    }
  }
}

// The new primitives go to Pout (the stage kernel's next buffer), or to G.P in place.
template <class R, class PT, class In>
__device__ __forceinline__ void cell_core(const GridDev &G, unsigned ia, unsigned jb, const CellIndex &x, const int MODE,
                                          double dt, const In &in, PT *Pout = nullptr) {
  const long long c = x.c;
  const Phys P = G.phys;
  PT *__restrict__ Pio = Pout ? Pout : (PT *)G.P;
  double *__restrict__ U = G.U;
  double *__restrict__ UP = G.UP;
  double *__restrict__ rhs_out = G.RHS;
  const double dx = G.dx, dy = G.dy, dz = G.dz;
  unsigned long long *cnt = G.cnt;
  in.wait_prims();
  double q[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) q[v] = in.prim(v);
  double src[NEQ];
  if constexpr (sizeof(R) == sizeof(float))
    sources<R>(P, in.table_r(), q, src, in.table64()(CF_ALPHA), in.table64()(CF_SQG));
  else
    sources<R>(P, in.table_r(), q, src, 0.0, 0.0);
  in.wait_fluxes();
  // the flux differences in R; their sum with the (FP64) sources in FP64 (for R = double
  // the reference's order: -(F_i - F_{i-1})/dx + S, then - (G_j - G_{j-1})/dy, ...)
  double rhs[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) {
    const R a = in.flux(0, 1, v), b = in.flux(0, 0, v);
    rhs[v] = (double)(div_pos(-(a - b), R(dx)) + src[v]);
  }
  if (G.ny > 1) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      const R a = in.flux(1, 1, v), b = in.flux(1, 0, v);
      rhs[v] = rhs[v] - (double)div_pos(a - b, R(dy));
    }
  }
  if (G.nz > 1) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      const R a = in.flux(2, 1, v), b = in.flux(2, 0, v);
      rhs[v] = rhs[v] - (double)div_pos(a - b, R(dz));
    }
  }
  if (MODE == 0) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) rhs_out[v * G.pplane + c] = rhs[v];
    return;
  }
  in.wait_state();
  double cs[NEQ];
  constexpr bool mixed = sizeof(PT) == sizeof(float);
  const bool comp = mixed && G.carry != 0;  // compensated accumulation (mixed policy only)
  double lo[NEQ];
  if (comp) {
    rk_stage_compensated(G, c, MODE, dt, in, rhs, cs, lo);
  } else {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) {
      const double up = in.up(v);
      double nv;
      if (MODE == 1) {
        U[v * G.pplane + c] = up;  // u = up (grhd2.f90:232)
        nv = up + rhs[v] * dt;
      } else if (MODE == 2) {
        nv = 0.75 * in.u(v) + 0.25 * (up + rhs[v] * dt);
      } else {
        nv = (in.u(v) + 2.0 * (up + rhs[v] * dt)) / 3.0;
      }
      cs[v] = nv;
    }
  }
  double hi[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) hi[v] = cs[v];
  const auto cm = metric_of(in.table64());
  double pr[NEQ];
  unsigned fl;
  if constexpr (mixed)  // mixed policy: the seeded root finder
    fl = cons_to_prim(P, cm, cs, pr, PrimSeed<In, decltype(cm)>{in, cm});
  else
    fl = cons_to_prim(P, cm, cs, pr);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) {
    UP[v * G.pplane + c] = cs[v];
    Pio[v * G.pplane + c] = (PT)pr[v];
  }
  if (comp) {  // a value con2prim changed (floors, causal rescaling) starts without a carry
#pragma unroll
    for (int v = 0; v < NEQ; ++v) store_carry(G, G.UPc, v * G.pplane + c, cs[v] == hi[v] ? lo[v] : 0.0);
  }
  c2p_count(cnt, fl);
}

template <class R, class PT>
__device__ __forceinline__ void cell_item(const GridDev &G, unsigned ia, unsigned jb, unsigned kc, const int MODE) {
  double dt = 0.0;
  if (MODE != 0) {
    const GridClock ck = *G.clock;
    if (clock_skip(ck)) return;
    dt = clock_dt(ck);
  }
  const CellIndex x = cell_index_of(G, ia, jb, kc);
  const long long ij = (long long)ia + (long long)G.nx * jb;
  cell_core<R, PT>(G, ia, jb, x, MODE, dt,
                   DirectIn<R, PT>{G, x, global_col(centre_table<R>(G), G, ij), global_col(G.centre, G, ij)});
}

// ---- staged inputs ------------------------------------------------------------------
// Each thread copies its own cell's streamed inputs into shared memory with cp.async
// (sm_80+ asynchronous global->shared copies; a thread waits for its own groups, so no
// block barrier is needed) in three commit groups: primitives, face fluxes, then up and
// u.  All the copies are in flight at once without holding registers, and the sources
// (which need only the primitives and the metric tables) overlap the flux and RK-state
// fetches.  Layout per block, structure of arrays over the block's threads:
//   double up[NEQ][CELL_BS], u[NEQ][CELL_BS]; PT p[NEQ][CELL_BS];
//   R f[2 * dirs][NEQ][CELL_BS]   (lower, upper face of each active direction)
constexpr int CELL_BS_STAGE = 128;
static_assert(CELL_BS_STAGE % 32 == 0, "sliced cell tiles are whole warps along i");
// Staging pays for the mixed policy (measured on the 2.5D and 3D torus batches: cell
// update -7 %); the FP64 kernel is bound by its FP64 instruction stream and runs as fast
// with direct loads and no shared memory limiting its resident blocks.
template <class PT>
__host__ __device__ constexpr bool cell_staged() { return sizeof(PT) == sizeof(float); }
template <class R, class PT>
__host__ __device__ constexpr size_t cell_stage_bytes(int dirs) {
  return cell_staged<PT>()
             ? (size_t)CELL_BS_STAGE * (2 * NEQ * sizeof(double) + NEQ * sizeof(PT) + 2 * dirs * NEQ * sizeof(R))
             : 0;
}

template <class R, class PT, class ColR, class Col64>
struct StagedIn {
  const double *s_up, *s_u;
  const PT *s_p;
  const R *s_f;
  int t, slot[3];
  ColR cr;
  Col64 c64;
  __device__ __forceinline__ StagedIn(ColR cr_, Col64 c64_) : cr(cr_), c64(c64_) {}
  __device__ __forceinline__ const ColR &table_r() const { return cr; }
  __device__ __forceinline__ const Col64 &table64() const { return c64; }
  // issue the three copy groups (primitives, face fluxes, up and u) of this thread's cell
  __device__ __forceinline__ void issue(const GridDev &G, const CellIndex &x, const int MODE, unsigned char *raw) {
    t = threadIdx.x;
    double *up = (double *)raw;
    double *u = up + NEQ * CELL_BS_STAGE;
    PT *p = (PT *)(u + NEQ * CELL_BS_STAGE);
    R *f = (R *)(p + NEQ * CELL_BS_STAGE);
    s_up = up; s_u = u; s_p = p; s_f = f;
    slot[0] = 0;
    slot[1] = 1;
    slot[2] = G.ny > 1 ? 2 : 1;
    const PT *Pg = (const PT *)G.P;
#pragma unroll
    for (int v = 0; v < NEQ; ++v) cp_async<sizeof(PT)>(&p[v * CELL_BS_STAGE + t], &Pg[v * G.pplane + x.c]);
    cp_async_commit();
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if ((d == 1 && G.ny == 1) || (d == 2 && G.nz == 1)) continue;
      const R *Fg = (const R *)G.F[d];
      const long long lo = face_lo(G, x, d), nf = face_n(G, d), off = face_up(G, d);
#pragma unroll
      for (int v = 0; v < NEQ; ++v) {
        cp_async<sizeof(R)>(&f[((2 * slot[d]) * NEQ + v) * CELL_BS_STAGE + t], &Fg[v * nf + lo]);
        cp_async<sizeof(R)>(&f[((2 * slot[d] + 1) * NEQ + v) * CELL_BS_STAGE + t], &Fg[v * nf + lo + off]);
      }
    }
    cp_async_commit();
    if (MODE != 0) {
#pragma unroll
      for (int v = 0; v < NEQ; ++v) cp_async<8>(&up[v * CELL_BS_STAGE + t], &G.UP[v * G.pplane + x.c]);
      if (MODE >= 2) {
#pragma unroll
        for (int v = 0; v < NEQ; ++v) cp_async<8>(&u[v * CELL_BS_STAGE + t], &G.U[v * G.pplane + x.c]);
      }
    }
    cp_async_commit();
  }
  __device__ __forceinline__ void wait_prims() const { cp_async_wait<2>(); }
  __device__ __forceinline__ void wait_fluxes() const { cp_async_wait<1>(); }
  __device__ __forceinline__ void wait_state() const { cp_async_wait<0>(); }
  __device__ __forceinline__ double prim(int v) const { return (double)s_p[v * CELL_BS_STAGE + t]; }
  __device__ __forceinline__ R flux(int d, int upper, int v) const {
    return s_f[((2 * slot[d] + upper) * NEQ + v) * CELL_BS_STAGE + t];
  }
  __device__ __forceinline__ double up(int v) const { return s_up[v * CELL_BS_STAGE + t]; }
  __device__ __forceinline__ double u(int v) const { return s_u[v * CELL_BS_STAGE + t]; }
};

// Dynamic shared memory: the table slice (slice_bytes<R>()), then for the mixed policy the
// staged inputs (cell_stage_bytes<R, PT>(dirs); dirs = the most active directions of any
// grid of the launch).
template <int MODE, class R, class PT>
__global__ void __launch_bounds__(CELL_BS_STAGE, cell_min_blocks<PT>())
    k_cell_update(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  extern __shared__ __align__(16) unsigned char cell_stage[];
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  unsigned ia, jb, kc;
  const bool valid = tile_item<7>(G.tiles[TILE_CELL], (unsigned)bm.first >> 7, threadIdx.x, (unsigned)G.nx,
                                  (unsigned)G.ny, (unsigned)G.nz, ia, jb, kc);
  double dt = 0.0;
  if (MODE != 0) {
    const GridClock ck = *G.clock;
    if (clock_skip(ck)) return;  // the same for the whole block (one grid)
    dt = clock_dt(ck);
  }
  const unsigned lane = threadIdx.x & 31u;
  const bool sliced = cell_tile_sliced(G);  // the same for the whole block
  R *slice = (R *)cell_stage;
  if (sliced) stage_slice<R>(slice, centre_table<R>(G), G, ia - lane, jb);
  const CellIndex x = cell_index_of(G, ia, jb, kc);
  const long long ij = (long long)ia + (long long)G.nx * jb;
  if (!cell_staged<PT>()) {  // FP64: direct loads of the streamed inputs
    if (sliced) {
      cp_async_wait<0>();
      __syncthreads();
    }
    if (!valid) return;
    if (sliced)
      cell_core<R, PT>(G, ia, jb, x, MODE, dt,
                       DirectIn<R, PT, SliceCol<R>, SliceCol<R>>{G, x, SliceCol<R>{slice, lane}, SliceCol<R>{slice, lane}});
    else
      cell_core<R, PT>(G, ia, jb, x, MODE, dt,
                       DirectIn<R, PT>{G, x, global_col(centre_table<R>(G), G, ij), global_col(G.centre, G, ij)});
    return;
  }
  // mixed policy: the FP32 table from the slice, the FP64 metric of con2prim from global
  // memory field by field
  unsigned char *inputs = cell_stage + slice_bytes<R>();
  if (sliced) {
    StagedIn<R, PT, SliceCol<R>, LazyCol<double>> in(SliceCol<R>{slice, lane}, LazyCol<double>{global_col(G.centre, G, ij)});
    if (valid) {
      in.issue(G, x, MODE, inputs);
      cp_async_wait<3>();  // the slice's group; the three input groups stay in flight
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (!valid) return;
    cell_core<R, PT>(G, ia, jb, x, MODE, dt, in);
  } else {
    if (!valid) return;
    StagedIn<R, PT, GlobalCol<R>, LazyCol<double>> in(global_col(centre_table<R>(G), G, ij),
                                                       LazyCol<double>{global_col(G.centre, G, ij)});
    in.issue(G, x, MODE, inputs);
    cell_core<R, PT>(G, ia, jb, x, MODE, dt, in);
  }
}

}  // namespace grhd
