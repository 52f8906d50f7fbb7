// flux.cuh -- face fluxes of one direction.
//
//   k_recon<DIR, REC>      one thread per face: selects the branch of reconstruct_1d_core
//                          (reconstruction.f90:318-645) from the density and pressure
//                          stencils, then per variable loads the stencil (boundary fill
//                          evaluated on load) and writes q_L, q_R with the positivity
//                          floors (reconstruction.f90:647-655).
//   k_recon_var<DIR, REC>  the same with one thread per (face, variable), for launches
//                          too small for one thread per face.
//   k_riemann<DIR, RS>     one thread per face: resolve_riemann_problem (fluxes.f90:56) on
//                          the reconstructed states, zero flux on degenerate faces
//                          (evolution.f90:69-71, :122-124).
//   k_flux<DIR, REC, RS>   both in one kernel, the interface states kept on chip.
//
// Splitting the per-face work keeps each kernel's code and register footprint small (the
// reconstruction holds ~75% of the divisions), and compile-time specialisation on the
// scheme and the Riemann solver removes the code of the schemes a run does not use; the
// autotuner picks among the split forms and the fused one per launch shape.
#pragma once

#include "common.cuh"

namespace grhd {

struct FaceIndex {
  int i, j, k, face;  // 1-based strip cell indices; face 0..n along DIR
  long long ft;       // face-table index (k-invariant)
};

// extents of the face index space of direction DIR (faces along DIR: n + 1)
template <int DIR>
__device__ __forceinline__ void face_space(const GridDev &G, unsigned &nI, unsigned &nJ, unsigned &nK) {
  nI = (unsigned)G.nx + (DIR == 1 ? 1u : 0u);
  nJ = (unsigned)G.ny + (DIR == 2 ? 1u : 0u);
  nK = (unsigned)G.nz + (DIR == 3 ? 1u : 0u);
}

// face (a, b, c) of the index space: strip cell indices, face number along DIR, table index
template <int DIR>
__device__ __forceinline__ FaceIndex face_at(const GridDev &G, unsigned a, unsigned b, unsigned c) {
  FaceIndex x;
  if (DIR == 1) {
    x.face = (int)a; x.i = (int)a; x.j = (int)b + 1; x.k = (int)c + 1;
    x.ft = (long long)a + (long long)(G.nx + 1) * b;
  } else if (DIR == 2) {
    x.i = (int)a + 1; x.face = (int)b; x.j = (int)b; x.k = (int)c + 1;
    x.ft = (long long)a + (long long)G.nx * b;
  } else {
    x.i = (int)a + 1; x.j = (int)b + 1; x.face = (int)c; x.k = (int)c;
    x.ft = (long long)a + (long long)G.nx * b;
  }
  return x;
}

template <int DIR>
__device__ __forceinline__ long long n_faces(const GridDev &G) {
  if (DIR == 1) return (long long)(G.nx + 1) * G.ny * G.nz;
  if (DIR == 2) return (long long)G.nx * (G.ny + 1) * G.nz;
  return (long long)G.nx * G.ny * (G.nz + 1);
}

// variable v of the cell c along DIR of the face's strip (boundary fill on load)
template <int DIR, class PT>
__device__ __forceinline__ double load_var(const PT *__restrict__ P, const GridDev &G, const FaceIndex &x, int c, int v) {
  const int n = DIR == 1 ? G.nx : (DIR == 2 ? G.ny : G.nz);
  int i = x.i, j = x.j, k = x.k;
  if (DIR == 1) i = c; else if (DIR == 2) j = c; else k = c;
  if (c >= 1 && c <= n) return ld_prim(P, G, v, i, j, k);
  double q[NEQ];
  load_cell<DIR>(P, G, i, j, k, q);
  double out = q[0];
#pragma unroll
  for (int w = 1; w < NEQ; ++w) if (w == v) out = q[w];
  return out;
}

// All five variables of the window cells m = lo..hi (0 elsewhere) of a face whose window
// leaves the grid, each cell's boundary fill evaluated once: w[v][m].  Out of line, with w
// in the caller's local memory, so the interior path keeps its registers and a warp that
// holds a few such faces among interior ones (two warps of each 401-face row along x)
// pays one short detour per face instead of one per (variable, cell).  Measured against
// boundary fill per (variable, cell): fused FP32 face kernel along x -27 % (mixed 2.5D
// torus batch +12 %, 3D torus +24 %); FP64 reconstruction along x -9 % (2.5D) and -37 %
// (3D torus, MP5 with the sensor).
template <int DIR, class R, class PT>
__device__ __noinline__ void edge_window(const PT *__restrict__ P, const GridDev &G, const FaceIndex &x, int lo, int hi,
                                         R (&w)[NEQ][6]) {
#pragma unroll 1
  for (int m = 0; m < 6; ++m) {
    double q[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (m >= lo && m <= hi) {
      const int c = x.face - 2 + m;
      load_cell<DIR>(P, G, DIR == 1 ? c : x.i, DIR == 2 ? c : x.j, DIR == 3 ? c : x.k, q);
    }
#pragma unroll
    for (int v = 0; v < NEQ; ++v) w[v][m] = (m >= lo && m <= hi) ? R(q[v]) : R(0);
  }
}

// branch selection of reconstruct_1d_core from the density and pressure stencils
// rho[m], p[m] = prim(., i-2+m), m = 0..4
template <int REC, class R>
__device__ __forceinline__ int branch_of(const Phys &P, const R (&rho)[5], const R (&p)[5], int i, int nodes, int dir) {
  if (REC == REC_GODUNOV) return BR_GODUNOV;
  R p_jump = R(0), rho_jump = R(0);
  if (P.sensor) {
    R pmax = p[0], pmin = p[0], rmx = rho[0], rmn = rho[0];
#pragma unroll
    for (int m = 1; m < 5; ++m) {
      pmax = rmax(pmax, p[m]); pmin = rmin(pmin, p[m]);
      rmx = rmax(rmx, rho[m]); rmn = rmin(rmn, rho[m]);
    }
    const R pf = R(P.p_floor), rf = R(P.rho_floor);
    p_jump = (pmax > R(1.0e3) * pf) ? (pmax - pmin) / rmax(pmin, pf) : R(0);
    rho_jump = (rmx > R(1.0e3) * rf) ? (rmx - rmn) / rmax(rmn, rf) : R(0);
  }
  const bool inner = P.nonmink && dir == 1 && i <= 0;
  const R atm = R(1.0e2) * R(P.rho_floor);
  const bool atmo = rho[2] <= atm || rho[3] <= atm;
  const bool cliff = p_jump >= R(10.0) || rho_jump >= R(10.0);
  const bool shock = p_jump >= R(0.80) || rho_jump >= R(0.50);
  const bool smooth_break = p_jump >= R(0.40) || rho_jump >= R(0.15);
  if (REC == REC_TVD) return (P.sensor && (inner || atmo || cliff)) ? BR_GODUNOV : BR_TVD;
  if (REC == REC_WENO3) {
    if (P.sensor) return (inner || atmo || cliff) ? BR_GODUNOV : (shock ? BR_TVD_MC : BR_WENO3);
    return inner ? BR_GODUNOV : BR_WENO3;
  }
  if (REC == REC_MP5) {
    if (P.sensor) {
      if (inner || atmo || cliff) return BR_GODUNOV;
      if (shock) return BR_TVD_MC;
      if (smooth_break || (P.nonmink && dir == 1 && i <= 3) || (P.nonmink && dir == 2 && (i <= 2 || i >= nodes - 2)))
        return BR_WENO3;
      return BR_MP5;
    }
    return inner ? BR_GODUNOV : BR_MP5;
  }
  if (P.sensor) {
    if (inner || atmo || cliff) return BR_GODUNOV;
    if (shock) return BR_TVD_MC;
    return smooth_break ? BR_WENO3 : BR_WENO5;
  }
  return inner ? BR_GODUNOV : BR_WENO5;
}

// interface states of one variable; only the branches a scheme can take are compiled
template <int REC, class R>
__device__ __forceinline__ void recon_one(int br, int lim, const R (&s)[6], R &qL, R &qR) {
  if (br == BR_GODUNOV) { qL = s[2]; qR = s[3]; return; }
  if (REC == REC_TVD) {
    qL = s[2] + R(0.5) * tvd_slope(s[2] - s[1], s[3] - s[2], lim);
    qR = s[3] - R(0.5) * tvd_slope(s[3] - s[2], s[4] - s[3], lim);
    return;
  }
  if (REC != REC_GODUNOV && br == BR_TVD_MC) {
    qL = s[2] + R(0.5) * tvd_slope(s[2] - s[1], s[3] - s[2], LIM_MC);
    qR = s[3] - R(0.5) * tvd_slope(s[3] - s[2], s[4] - s[3], LIM_MC);
    return;
  }
  if (REC != REC_GODUNOV && br == BR_WENO3) { qL = weno3(s[1], s[2], s[3]); qR = weno3(s[4], s[3], s[2]); return; }
  if (REC == REC_MP5) { qL = mp5(s[0], s[1], s[2], s[3], s[4]); qR = mp5(s[5], s[4], s[3], s[2], s[1]); return; }
  if (REC == REC_WENO5) { qL = weno5(s[0], s[1], s[2], s[3], s[4]); qR = weno5(s[5], s[4], s[3], s[2], s[1]); return; }
}

// Batched launches: block b works on grid map[b].grid, tile map[b].first / blockDim.x.
// Q layout per grid: Q[(side*5 + v) * nfaces + f], side 0 = q_L, 1 = q_R
// Resident blocks per SM the register allocation must allow (256-thread recon blocks,
// 128-thread Riemann blocks), measured on the batched 2.5D torus and the 3D torus: recon
// 4 (64 registers); Riemann 8 for HLLE (64 registers), HLLC 4 in FP64 (128 registers)
// and 6 in FP32 (80): HLLC's larger state spills at 64.
constexpr int RECON_MIN_BLOCKS = 4;
template <int RS, class R>
constexpr int riemann_min_blocks() { return RS == RS_HLLC ? (sizeof(R) == sizeof(double) ? 4 : 6) : 8; }
// One thread per face reconstructs all five variables (rolled variable loop): the set-up
// of a work item (block map, descriptor, tile decode, window check, the sensor's density
// and pressure windows and branch) is paid once per face.  Measured against one thread
// per (face, variable): FP64 2.5D torus batch +2 %, 3D torus (MP5 + sensor) +24 %.
template <int DIR, int REC, class R, class PT>
__global__ void __launch_bounds__(256, RECON_MIN_BLOCKS) k_recon(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  const Phys P = G.phys;
  const long long nf = n_faces<DIR>(G);
  unsigned nI, nJ, nK, a, b, c;
  face_space<DIR>(G, nI, nJ, nK);
  if (!tile_item<8>(G.tiles[TILE_RECON + DIR - 1], (unsigned)bm.first >> 8, threadIdx.x, nI, nJ, nK, a, b, c) ||
      clock_skip(*G.clock))
    return;
  const long long f = (long long)a + (long long)nI * ((long long)b + (long long)nJ * c);
  const PT *__restrict__ Pin = (const PT *)G.P;
  R *__restrict__ Q = (R *)G.Q;
  const FaceIndex x = face_at<DIR>(G, a, b, c);
  const int n = DIR == 1 ? G.nx : (DIR == 2 ? G.ny : G.nz);
  int lo, hi;
  stencil_range(REC, P.sensor, lo, hi);
  const bool inside = x.face - 2 + lo >= 1 && x.face - 2 + hi <= n;
  const long long stride = DIR == 1 ? 1LL : (DIR == 2 ? (long long)G.nx : (long long)G.nx * G.ny);
  long long base = 0;
  if (inside) {
    const int c0 = x.face - 2 + lo;
    base = (long long)cell_index(G, DIR == 1 ? c0 : x.i, DIR == 2 ? c0 : x.j, DIR == 3 ? c0 : x.k) - lo * stride;
  }
  R ew[NEQ][6];  // an edge face's window, boundary-filled (local memory)
  if (!inside) edge_window<DIR>(Pin, G, x, lo, hi, ew);
  auto ld = [&](int w, int m) -> R {
    return inside ? R(GRHD_LDP(&Pin[w * G.pplane + base + m * stride])) : ew[w][m];
  };
  int br = BR_GODUNOV;
  if (REC != REC_GODUNOV) {
    R rho[5], pr[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      rho[m] = P.sensor ? ld(EQ_DE, m) : R(0);
      pr[m] = P.sensor ? ld(EQ_PR, m) : R(0);
    }
    br = branch_of<REC>(P, rho, pr, x.face, n, DIR);
  }
  unsigned clamps = 0;
  // loop invariants in registers; a variable's stencil is read at 32-bit offsets from its
  // row pointer (hoisting these measured -8 % on the k-direction reconstruction)
  const long long pplane = G.pplane;
  const unsigned ustride = (unsigned)stride;
  const int lim = P.lim;
  const R rho_fl = R(P.rho_floor), p_fl = R(P.p_floor);
#pragma unroll 1
  for (int v = 0; v < NEQ; ++v) {
    R s[6];
    if (inside) {
      const PT *row = Pin + (base + (long long)v * pplane);
#pragma unroll
      for (int m = 0; m < 6; ++m) s[m] = (m >= lo && m <= hi) ? R(GRHD_LDP(row + m * ustride)) : R(0);
    } else {
#pragma unroll
      for (int m = 0; m < 6; ++m) s[m] = (m >= lo && m <= hi) ? ew[v][m] : R(0);
    }
    R qL, qR;
    recon_one<REC>(br, lim, s, qL, qR);
    if (v == EQ_DE || v == EQ_PR) {  // reconstruction.f90:647-655
      const R fl = v == EQ_DE ? rho_fl : p_fl;
      clamps += (unsigned)!(qL >= fl) + (unsigned)!(qR >= fl);
      qL = rmax(qL, fl);
      qR = rmax(qR, fl);
    }
    Q[(long long)v * nf + f] = qL;
    Q[(long long)(5 + v) * nf + f] = qR;
  }
  count_add(G.cnt, CNT_RECON_CLAMP, clamps);
}

// The same reconstruction with one thread per (face, variable), blockIdx.y = variable:
// five times the threads of k_recon, for launches too small to fill the GPU with one
// thread per face (a single 2.5D grid: 400x1x200 has 80k faces per direction).  Its
// launch bound (5 blocks, 48 registers) was measured on such launches.
template <int DIR, int REC, class R, class PT>
__global__ void __launch_bounds__(256, 5) k_recon_var(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  const Phys P = G.phys;
  const long long nf = n_faces<DIR>(G);
  const int v = blockIdx.y;
  unsigned nI, nJ, nK, a, b, c;
  face_space<DIR>(G, nI, nJ, nK);
  if (!tile_item<8>(G.tiles[TILE_RECON + DIR - 1], (unsigned)bm.first >> 8, threadIdx.x, nI, nJ, nK, a, b, c) ||
      clock_skip(*G.clock))
    return;
  const long long f = (long long)a + (long long)nI * ((long long)b + (long long)nJ * c);
  const PT *__restrict__ Pin = (const PT *)G.P;
  R *__restrict__ Q = (R *)G.Q;
  unsigned long long *cnt = G.cnt;
  const FaceIndex x = face_at<DIR>(G, a, b, c);
  const int n = DIR == 1 ? G.nx : (DIR == 2 ? G.ny : G.nz);
  int lo, hi;
  stencil_range(REC, P.sensor, lo, hi);
  // a stencil entirely inside the grid reads P directly at a fixed stride along DIR
  const bool inside = x.face - 2 + lo >= 1 && x.face - 2 + hi <= n;
  const long long stride = DIR == 1 ? 1LL : (DIR == 2 ? (long long)G.nx : (long long)G.nx * G.ny);
  long long base = 0;
  if (inside) {
    const int c0 = x.face - 2 + lo;
    base = (long long)cell_index(G, DIR == 1 ? c0 : x.i, DIR == 2 ? c0 : x.j, DIR == 3 ? c0 : x.k) - lo * stride;
  }
  const long long pplane = G.pplane;
  const unsigned ustride = (unsigned)stride;
  auto ld = [&](int w, int m) -> R {
    return inside ? R(GRHD_LDP(Pin + (base + (long long)w * pplane) + m * ustride))
                  : R(load_var<DIR>(Pin, G, x, x.face - 2 + m, w));
  };
  R s[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) s[m] = (m >= lo && m <= hi) ? ld(v, m) : R(0);
  int br = BR_GODUNOV;
  if (REC != REC_GODUNOV) {
    R rho[5], pr[5];
    if (P.sensor) {
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        rho[m] = v == EQ_DE ? s[m] : ld(EQ_DE, m);
        pr[m] = v == EQ_PR ? s[m] : ld(EQ_PR, m);
      }
    } else {
#pragma unroll
      for (int m = 0; m < 5; ++m) { rho[m] = R(0); pr[m] = R(0); }
    }
    br = branch_of<REC>(P, rho, pr, x.face, n, DIR);
  }
  R qL, qR;
  recon_one<REC>(br, P.lim, s, qL, qR);
  unsigned clamps = 0;
  if (v == EQ_DE || v == EQ_PR) {  // reconstruction.f90:647-655
    const R fl = v == EQ_DE ? R(P.rho_floor) : R(P.p_floor);
    clamps = (unsigned)!(qL >= fl) + (unsigned)!(qR >= fl);
    qL = rmax(qL, fl);
    qR = rmax(qR, fl);
  }
  Q[(long long)v * nf + f] = qL;
  Q[(long long)(5 + v) * nf + f] = qR;
  count_add(cnt, CNT_RECON_CLAMP, clamps);
}

// ------------------------------------------------------------------------------------
// Fused alternative: one thread per face reconstructs all five variables and solves the
// Riemann problem, so q_L, q_R never leave the SM.  Same arithmetic as k_recon + k_riemann
// (bit-identical results); the branch of the sensor cascade is evaluated once per face
// instead of once per (face, variable).  The variable loop is kept rolled (one copy of
// the reconstruction code) and the interface states are staged in shared memory.
// ------------------------------------------------------------------------------------
constexpr int FLUX_BS = 128;

// One face (a, b, c) of direction DIR: all five variables reconstructed, then the Riemann
// flux.  sq is this thread's column of a [2*NEQ][blockDim] shared array (the rolled
// variable loop indexes it at run time).
template <int DIR, int REC, int RS, class R, class PT>
__device__ __forceinline__ void flux_item(const GridDev &G, unsigned a, unsigned b, unsigned c, R (*sq)[FLUX_BS]) {
  if (clock_skip(*G.clock)) return;
  const Phys P = G.phys;
  const long long nf = n_faces<DIR>(G);
  unsigned nI, nJ, nK;
  face_space<DIR>(G, nI, nJ, nK);
  const long long f = (long long)a + (long long)nI * ((long long)b + (long long)nJ * c);
  const PT *__restrict__ Pin = (const PT *)G.P;
  const FaceIndex x = face_at<DIR>(G, a, b, c);
  const int n = DIR == 1 ? G.nx : (DIR == 2 ? G.ny : G.nz);
  int lo, hi;
  stencil_range(REC, P.sensor, lo, hi);
  // a stencil entirely inside the grid reads P directly at a fixed stride along DIR
  const bool inside = x.face - 2 + lo >= 1 && x.face - 2 + hi <= n;
  const long long stride = DIR == 1 ? 1LL : (DIR == 2 ? (long long)G.nx : (long long)G.nx * G.ny);
  long long base = 0;
  if (inside) {
    const int c0 = x.face - 2 + lo;
    base = (long long)cell_index(G, DIR == 1 ? c0 : x.i, DIR == 2 ? c0 : x.j, DIR == 3 ? c0 : x.k) - lo * stride;
  }
  // window m = a..b of variable w; the interior case reads P at 32-bit offsets from the
  // variable's row pointer, an edge face its window of boundary-filled cells
  const long long pplane = G.pplane;
  const unsigned ustride = (unsigned)stride;
  R ew[NEQ][6];
  if (!inside) edge_window<DIR>(Pin, G, x, lo, hi, ew);
  auto window = [&](int w, int a, int b, R(&out)[6]) {
    if (inside) {
      const PT *row = Pin + (base + (long long)w * pplane);
#pragma unroll
      for (int m = 0; m < 6; ++m) out[m] = (m >= a && m <= b) ? R(GRHD_LDP(row + m * ustride)) : R(0);
    } else {
#pragma unroll
      for (int m = 0; m < 6; ++m) out[m] = (m >= a && m <= b) ? ew[w][m] : R(0);
    }
  };
  int br = BR_GODUNOV;
  if (REC != REC_GODUNOV) {
    R rho[5], pr[5];
    if (P.sensor) {  // the sensor reads cells 0..4 of the window (inside [lo, hi] when it is on)
      R t[6];
      window(EQ_DE, 0, 4, t);
#pragma unroll
      for (int m = 0; m < 5; ++m) rho[m] = t[m];
      window(EQ_PR, 0, 4, t);
#pragma unroll
      for (int m = 0; m < 5; ++m) pr[m] = t[m];
    } else {
#pragma unroll
      for (int m = 0; m < 5; ++m) { rho[m] = R(0); pr[m] = R(0); }
    }
    br = branch_of<REC>(P, rho, pr, x.face, n, DIR);
  }
  unsigned clamps = 0;
#pragma unroll 1
  for (int v = 0; v < NEQ; ++v) {
    R s[6];
    window(v, lo, hi, s);
    R qL, qR;
    recon_one<REC>(br, P.lim, s, qL, qR);
    if (v == EQ_DE || v == EQ_PR) {  // reconstruction.f90:647-655
      const R fl = v == EQ_DE ? R(P.rho_floor) : R(P.p_floor);
      clamps += (unsigned)!(qL >= fl) + (unsigned)!(qR >= fl);
      qL = rmax(qL, fl);
      qR = rmax(qR, fl);
    }
    sq[v][threadIdx.x] = qL;
    sq[NEQ + v][threadIdx.x] = qR;
  }
  count_add(G.cnt, CNT_RECON_CLAMP, clamps);
  R qL[NEQ], qR[NEQ], flux[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) { qL[v] = sq[v][threadIdx.x]; qR[v] = sq[NEQ + v][threadIdx.x]; }
  R *__restrict__ F = (R *)G.F[DIR - 1];
  const R *T = face_table<R>(G, DIR - 1);
  const long long ntab = G.nface[DIR - 1];
  bool fb = false;
  if (__ldg(&T[FF_ZERO * ntab + x.ft]) != R(0)) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) flux[v] = R(0);
  } else {
    const FaceMetric<R> m = load_face_metric<R>(T, ntab, x.ft);
    if (RS == RS_HLLC) {
      const FaceFrame<R> fr = load_face_frame<R>(T, ntab, x.ft);
      fb = hllc_try(P, qL, qR, DIR, m, fr, flux);
    } else {
      fb = true;
    }
    if (fb) hlle(P, qL, qR, DIR, m, flux);
  }
#pragma unroll
  for (int v = 0; v < NEQ; ++v) F[(long long)v * nf + f] = flux[v];
  if (RS == RS_HLLC) count_add(G.cnt, CNT_HLLC_FALLBACK, fb ? 1u : 0u);
}


// Resident 128-thread blocks per SM for the fused kernel.  FP32 (mixed policy): 10 with
// HLLE (48 registers; 8 and 12 measured 2.5 % and 0-1 % slower on the batched 2.5D torus),
// 8 with HLLC, whose larger state spills at 48 (64 registers; 3D torus +2.8 %, its x faces
// -8 %).  FP64: 8 with HLLE (64 registers, a few spills; 32 tori 400x1x200: 7.90e8
// zone-updates/s against 7.36e8 for the split kernels and 6.61e8 with the 104 registers it
// takes unbounded; 6 and 10 blocks 7.47e8 and 7.87e8), 4 with HLLC (3D torus 4.05e8, 2 and
// 6-8 blocks slower -- the split kernels, 4.89e8, stay ahead there and the autotuner keeps
// them).
template <int RS, class R>
constexpr int flux_min_blocks() {
  return sizeof(R) == sizeof(float) ? (RS == RS_HLLC ? 8 : 10) : (RS == RS_HLLC ? 4 : 8);
}
template <int DIR, int REC, int RS, class R, class PT>
__global__ void __launch_bounds__(FLUX_BS, flux_min_blocks<RS, R>())
    k_flux(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  __shared__ R sq[2 * NEQ][FLUX_BS];
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  unsigned nI, nJ, nK, a, b, c;
  face_space<DIR>(G, nI, nJ, nK);
  if (!tile_item<7>(G.tiles[TILE_FACE + DIR - 1], (unsigned)bm.first >> 7, threadIdx.x, nI, nJ, nK, a, b, c)) return;
  flux_item<DIR, REC, RS, R, PT>(G, a, b, c, sq);
}

template <int DIR, int RS, class R>
__global__ void __launch_bounds__(128, riemann_min_blocks<RS, R>()) k_riemann(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map) {
  const BlockMap bm = map[blockIdx.x];
  const GridDev &G = grids[bm.grid];
  const Phys P = G.phys;
  const long long nf = n_faces<DIR>(G);
  unsigned nI, nJ, nK, a, b, c;
  face_space<DIR>(G, nI, nJ, nK);
  if (!tile_item<7>(G.tiles[TILE_FACE + DIR - 1], (unsigned)bm.first >> 7, threadIdx.x, nI, nJ, nK, a, b, c) ||
      clock_skip(*G.clock))
    return;
  const long long f = (long long)a + (long long)nI * ((long long)b + (long long)nJ * c);
  const R *__restrict__ Q = (const R *)G.Q;
  R *__restrict__ F = (R *)G.F[DIR - 1];
  unsigned long long *cnt = G.cnt;
  const FaceIndex x = face_at<DIR>(G, a, b, c);
  R qL[NEQ], qR[NEQ], flux[NEQ];
#pragma unroll
  for (int v = 0; v < NEQ; ++v) { qL[v] = Q[(long long)v * nf + f]; qR[v] = Q[(long long)(5 + v) * nf + f]; }
  const R *T = face_table<R>(G, DIR - 1);
  const long long ntab = G.nface[DIR - 1];
  bool fb = false;
  if (__ldg(&T[FF_ZERO * ntab + x.ft]) != R(0)) {
#pragma unroll
    for (int v = 0; v < NEQ; ++v) flux[v] = R(0);
  } else {
    const FaceMetric<R> m = load_face_metric<R>(T, ntab, x.ft);
    if (RS == RS_HLLC) {
      const FaceFrame<R> fr = load_face_frame<R>(T, ntab, x.ft);
      fb = hllc_try(P, qL, qR, DIR, m, fr, flux);
    } else {
      fb = true;
    }
    if (fb) hlle(P, qL, qR, DIR, m, flux);  // the single HLLE call site
  }
#pragma unroll
  for (int v = 0; v < NEQ; ++v) F[(long long)v * nf + f] = flux[v];
  if (RS == RS_HLLC) count_add(cnt, CNT_HLLC_FALLBACK, fb ? 1u : 0u);
}

}  // namespace grhd
