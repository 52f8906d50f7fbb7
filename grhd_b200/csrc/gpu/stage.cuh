// stage.cuh -- one whole SSP-RK3 stage of a 1D or 2D grid in one kernel.
//
// A block owns a tile of cells: 32 along i x 8 along the grid's second direction (y or z)
// for a 2D grid, 256 along i for a 1D grid.  It runs the stage in three phases, all
// through shared memory:
//   1. the tile's primitives with their stencil halo (the cross-shaped box of the cells the
//      tile's faces read, 3 deep; a cell outside the domain along one direction is its
//      boundary fill, evaluated once here -- set_boundary_conditions, conditions.f90:773)
//      and, for x-z tiles, the block's slice of the centre metric table;
//   2. every face of the tile, both directions: the reconstruction (reconstruct_1d_core,
//      reconstruction.f90:285-657) from the staged window and the Riemann flux
//      (resolve_riemann_problem, fluxes.f90:56), into shared memory;
//   3. every cell of the tile: the flux divergence and metric sources (calc_rhs,
//      evolution.f90:30-191), the RK stage combination (grhd2.f90:243-249) and con2prim
//      (equations.f90:94-205), written to up and to the next primitive buffer.
// The per-face and per-cell arithmetic is that of the split kernels (flux.cuh, cell.cuh),
// the same functions in the same order, so the FP64 results are the same to the bit.
// Interface states and face fluxes never reach global memory: a stage reads P (with the
// halo re-reads served by L2), u and up, and writes up and P, the stage's algorithmic
// bytes.
//
// Blocks read their neighbours' halo cells while other blocks write their new primitives,
// so a stage cannot update P in place: the primitives rotate through three buffers,
// P -> P2 (stage 1) -> P3 (stage 2) -> P (stage 3), and P is current again after every
// step.
//
// A face on a tile edge is computed by both tiles that touch it (the flux must be on chip
// for both); its counters (reconstruction floors, HLLC fallbacks) are counted by the tile
// that holds the face's upper cell (the domain's last face by the last tile), so every
// face counts once.
#pragma once

#include "flux.cuh"
#include "cell.cuh"

namespace grhd {

// A tile holds STAGE_CELLS cells; its block has STAGE_BS threads, enough that no thread
// computes more than two of the tile's 552 faces (2D) and no warp waits at the barrier for
// another's third.
constexpr int STAGE_CELLS = 256;
constexpr int STAGE_BS = 288;
constexpr int STAGE_H = 3;  // halo depth: the widest window (nghost = 3)

// tile geometry per second direction SD: 0 (1D grid), 2 (x-y grid), 3 (x-z grid)
template <int SD>
struct StageGeom {
  static constexpr int TX = SD == 0 ? STAGE_CELLS : 32;  // cells along i
  static constexpr int TR = SD == 0 ? 1 : STAGE_CELLS / 32;  // cells along the second direction
  static constexpr int BX = TX + 2 * STAGE_H;          // box extent along i
  static constexpr int BR = SD == 0 ? 1 : TR + 2 * STAGE_H;
  static constexpr int NBOX = BX * BR;
  static constexpr int NFX = (TX + 1) * TR;             // faces along x of a tile
  static constexpr int NFR = SD == 0 ? 0 : TX * (TR + 1);  // faces along the second direction
  static constexpr bool SLICE = SD == 3;                // the tile's rows share their (i,j) columns
};
static_assert(StageGeom<3>::TX == SLICE_COLS, "x-z tiles stage one table slice of SLICE_COLS columns");
static_assert(StageGeom<3>::NFX + StageGeom<3>::NFR <= 2 * STAGE_BS && StageGeom<0>::NFX <= STAGE_BS,
              "at most two faces per thread");

__host__ __device__ constexpr size_t stage_align(size_t b) { return (b + 15) / 16 * 16; }
template <int SD, class R>
__host__ __device__ constexpr size_t stage_smem_bytes() {
  using Gm = StageGeom<SD>;
  return stage_align((size_t)NEQ * Gm::NBOX * sizeof(R)) + stage_align((size_t)NEQ * Gm::NFX * sizeof(R)) +
         stage_align((size_t)NEQ * Gm::NFR * sizeof(R)) + (Gm::SLICE ? slice_bytes<R>() : 0);
}

// Resident blocks per SM the register allocation must allow: 3 (72 registers).  Measured on
// the 32-grid 2.5D torus batch: the variable loop unrolled (96 or 72 registers), 2 or 4
// blocks, and x-z tiles without the table slice (4 blocks fit) were 3-21 % slower in FP64
// and 0-26 % slower (4 blocks: equal) in the mixed policy.
template <class R>
constexpr int stage_min_blocks() { return 3; }

// One face of direction dir whose window cell m (m = 0..5, cells face-2 .. face+3 along
// dir) of variable v sits at w[v * vs + m * ms] in shared memory: the interface states
// with their floors (reconstruction.f90:647-655), then the Riemann flux into out[v * os].
// Returns the face's reconstruction floor clamps, plus STAGE_FB if HLLC fell back to HLLE.
// Out of line, with the variable loop rolled, so the kernel holds one copy of the face
// code for both directions: with the code of both directions inlined and the variable
// loop unrolled, the stage kernel stalled on instruction fetch more than on anything else.
constexpr unsigned STAGE_FB = 1u << 16;
template <int REC, int RS, class R>
__device__ __noinline__ unsigned stage_face(const GridDev &G, int dir, const R *w, int vs, int ms, int face, int n,
                                            long long ft, R *out, int os) {
  const Phys &P = G.phys;
  int lo, hi;
  stencil_range(REC, P.sensor, lo, hi);
  int br = BR_GODUNOV;
  if (REC != REC_GODUNOV) {
    R rho[5], pr[5];
    const bool sensor = P.sensor != 0;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      rho[m] = sensor ? w[EQ_DE * vs + m * ms] : R(0);
      pr[m] = sensor ? w[EQ_PR * vs + m * ms] : R(0);
    }
    br = branch_of<REC>(P, rho, pr, face, n, dir);
  }
  R qL[NEQ], qR[NEQ];
  unsigned cl = 0;
  const R rho_fl = R(P.rho_floor), p_fl = R(P.p_floor);
  const int lim = P.lim;
  auto one = [&](int v) {
    R s6[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) s6[m] = (m >= lo && m <= hi) ? w[v * vs + m * ms] : R(0);
    R l, r;
    recon_one<REC>(br, lim, s6, l, r);
    if (v == EQ_DE || v == EQ_PR) {  // reconstruction.f90:647-655
      const R fl = v == EQ_DE ? rho_fl : p_fl;
      cl += (unsigned)!(l >= fl) + (unsigned)!(r >= fl);
      l = rmax(l, fl);
      r = rmax(r, fl);
    }
    qL[v] = l;
    qR[v] = r;
  };
#pragma unroll 1
  for (int v = 0; v < NEQ; ++v) one(v);
  R flux[NEQ];
  const R *T = face_table<R>(G, dir - 1);
  const long long ntab = G.nface[dir - 1];
  bool fb = false;
  if (__ldg(&T[FF_ZERO * ntab + ft]) != R(0)) {  // evolution.f90:69-71, :122-124
#pragma unroll
    for (int v = 0; v < NEQ; ++v) flux[v] = R(0);
  } else {
    const FaceMetric<R> m = load_face_metric<R>(T, ntab, ft);
    if (RS == RS_HLLC) {
      const FaceFrame<R> fr = load_face_frame<R>(T, ntab, ft);
      fb = hllc_try(P, qL, qR, dir, m, fr, flux);
    } else {
      fb = true;
    }
    if (fb) hlle(P, qL, qR, dir, m, flux);
  }
#pragma unroll
  for (int v = 0; v < NEQ; ++v) out[v * os] = flux[v];
  return cl + ((RS == RS_HLLC && fb) ? STAGE_FB : 0u);
}

// cell_core's inputs for a cell of the tile: its primitives and face fluxes from shared
// memory, up and u from global memory
template <class R, class PT, int SD, class ColR, class Col64>
struct TileIn {
  const GridDev &G;
  const CellIndex &x;
  const R *sp;   // this cell's variable 0 in the box (variables NBOX apart)
  const R *sfx;  // this cell's lower x face (variables NFX apart, upper face +1)
  const R *sfr;  // this cell's lower face along the second direction (variables NFR apart, upper +TX)
  ColR cr;
  Col64 c64;
  using Gm = StageGeom<SD>;
  __device__ __forceinline__ void wait_prims() const {}
  __device__ __forceinline__ void wait_fluxes() const {}
  __device__ __forceinline__ void wait_state() const {}
  __device__ __forceinline__ const ColR &table_r() const { return cr; }
  __device__ __forceinline__ const Col64 &table64() const { return c64; }
  __device__ __forceinline__ double prim(int v) const { return (double)sp[v * Gm::NBOX]; }
  __device__ __forceinline__ R flux(int d, int upper, int v) const {
    if (d == 0) return sfx[v * Gm::NFX + upper];
    return sfr[v * Gm::NFR + upper * Gm::TX];  // d: the second direction (the only other active one)
  }
  __device__ __forceinline__ double up(int v) const { return G.UP[v * G.pplane + x.c]; }
  __device__ __forceinline__ double u(int v) const { return G.U[v * G.pplane + x.c]; }
};

// primitive buffers of a stage: read Pin, write Pout (P -> P2 -> P3 -> P)
template <class PT>
__device__ __forceinline__ void stage_buffers(const GridDev &G, int mode, const PT *&pin, PT *&pout) {
  pin = (const PT *)(mode == 1 ? G.P : G.Prot[mode - 2]);
  pout = (PT *)(mode == 3 ? G.P : G.Prot[mode - 1]);
}

// The work of one block on one tile, bm: grid bm.grid, tile bm.first / STAGE_BS (tiles
// numbered with i fastest); mode: the RK stage, 1..3.  The block's first STAGE_CELLS
// threads update the tile's cells.  k_stage runs one tile per block; the persistent stage
// kernel (persistent.cuh) loops over tiles.
template <int SD, int REC, int RS, class R, class PT>
__device__ __forceinline__ void stage_tile(const GridDev *__restrict__ grids, const BlockMap bm, int mode,
                                           unsigned char *stage_smem) {
  using Gm = StageGeom<SD>;
  constexpr int TX = Gm::TX, TR = Gm::TR, BX = Gm::BX, NBOX = Gm::NBOX, NFX = Gm::NFX, NFR = Gm::NFR;
  constexpr bool SLICE = Gm::SLICE;
  constexpr int RD = SD == 0 ? 1 : SD;  // the second direction (1D: none)
  R *s_p = (R *)stage_smem;
  R *s_fx = (R *)(stage_smem + stage_align((size_t)NEQ * NBOX * sizeof(R)));
  R *s_fr = (R *)((unsigned char *)s_fx + stage_align((size_t)NEQ * NFX * sizeof(R)));
  R *slice = (R *)((unsigned char *)s_fr + stage_align((size_t)NEQ * NFR * sizeof(R)));

  const GridDev &G = grids[bm.grid];
  const GridClock ck = *G.clock;
  if (clock_skip(ck)) return;  // the same for the whole block (one grid)
  const double dt = clock_dt(ck);
  const Phys P = G.phys;
  const unsigned tile = (unsigned)bm.first / STAGE_BS;
  const unsigned tr_ = fdiv(tile, G.stage_ntx);
  const int i0 = (int)(tile - tr_ * G.stage_ntx.d) * TX + 1;  // first cell of the tile (1-based)
  const int r0 = (int)tr_ * TR + 1;
  const int nx = G.nx, nr = SD == 2 ? G.ny : (SD == 3 ? G.nz : 1);
  const PT *Pin;
  PT *Pout;
  stage_buffers(G, mode, Pin, Pout);
  const unsigned t = threadIdx.x;

  // ---- 1. the primitive box (and the table slice) --------------------------------------
  if (SLICE) stage_slice<R>(slice, centre_table<R>(G), G, (unsigned)(i0 - 1), 0u);
  {
    int lo, hi;
    stencil_range(P.rec, P.sensor, lo, hi);
    const int ilast = min(i0 + TX - 1, nx), rlast = min(r0 + TR - 1, nr);
    const int ia = i0 - 3 + lo, ib = ilast - 2 + hi;  // cells the x faces read
    const int ra = r0 - 3 + lo, rb = rlast - 2 + hi;  // cells the faces of the second direction read
    for (int pos = (int)t; pos < NBOX; pos += STAGE_BS) {
      const int bx = pos % BX, brow = pos / BX;
      const int i = i0 - STAGE_H + bx, r = SD == 0 ? 1 : r0 - STAGE_H + brow;
      const bool row_ok = r >= r0 && r <= rlast && i >= ia && i <= ib;
      const bool col_ok = SD != 0 && i >= i0 && i <= ilast && r >= ra && r <= rb;
      if (!(row_ok || col_ok)) continue;
      const int j = SD == 2 ? r : 1, k = SD == 3 ? r : 1;
      double q[NEQ];
      if (i >= 1 && i <= nx && r >= 1 && r <= nr) {
        const unsigned c = cell_index(G, i, j, k);
#pragma unroll
        for (int v = 0; v < NEQ; ++v) q[v] = (double)GRHD_LDP(&Pin[v * G.pplane + c]);
      } else if (i < 1 || i > nx) {
        load_cell<1>(Pin, G, i, j, k, q);
      } else {
        load_cell<RD>(Pin, G, i, j, k, q);
      }
#pragma unroll
      for (int v = 0; v < NEQ; ++v) s_p[v * NBOX + pos] = R(q[v]);
    }
  }
  if (SLICE) cp_async_wait<0>();
  __syncthreads();

  // ---- 2. the faces of the tile: x faces, then those of the second direction ------------
  unsigned clamps = 0, fallbacks = 0;
  {
    const int afx = min(TX, nx - i0 + 1);  // last x face of the tile (local index)
    const int afr = min(TR, nr - r0 + 1);  // last face of the second direction (local index)
    for (int q = (int)t; q < NFX + NFR; q += STAGE_BS) {
      unsigned res;
      bool owned;
      if (q < NFX) {
        const int rr = q / (TX + 1), a = q - rr * (TX + 1);
        const int f = i0 - 1 + a, rc = r0 + rr;
        if (a > afx || rc > nr) continue;
        const int j = SD == 2 ? rc : 1;
        const long long ft = (long long)f + (long long)(nx + 1) * (j - 1);
        res = stage_face<REC, RS, R>(G, 1, s_p + (rr + (SD == 0 ? 0 : STAGE_H)) * BX + a, NBOX, 1, f, nx, ft, s_fx + q,
                                     NFX);
        owned = a < TX || f == nx;
      } else {
        const int qr = q - NFX, b = qr / TX, a = qr - b * TX;
        const int f = r0 - 1 + b, i = i0 + a;
        if (i > nx || b > afr) continue;
        const long long ft = SD == 3 ? (long long)(i - 1) : (long long)(i - 1) + (long long)nx * f;
        res = stage_face<REC, RS, R>(G, RD, s_p + b * BX + a + STAGE_H, NBOX, BX, f, nr, ft, s_fr + qr, NFR);
        owned = b < TR || f == nr;
      }
      if (owned) {
        clamps += res & (STAGE_FB - 1u);
        fallbacks += res >> 16;
      }
    }
  }
  count_add(G.cnt, CNT_RECON_CLAMP, clamps);
  if (RS == RS_HLLC) count_add(G.cnt, CNT_HLLC_FALLBACK, fallbacks);
  __syncthreads();

  // ---- 3. the cells of the tile ----------------------------------------------------------
  if (t >= (unsigned)STAGE_CELLS) return;
  const int a = (int)(t % TX), rr = (int)(t / TX);
  const int i = i0 + a, r = r0 + rr;
  if (i > nx || r > nr) return;
  const unsigned ia = (unsigned)(i - 1), jb = SD == 2 ? (unsigned)(r - 1) : 0u, kc = SD == 3 ? (unsigned)(r - 1) : 0u;
  const CellIndex x = cell_index_of(G, ia, jb, kc);
  const long long ij = (long long)ia + (long long)G.nx * jb;
  const R *sp = s_p + (rr + (SD == 0 ? 0 : STAGE_H)) * BX + a + STAGE_H;
  const R *sfx = s_fx + rr * (TX + 1) + a;
  const R *sfr = s_fr + rr * TX + a;
  if constexpr (SLICE) {
    if constexpr (sizeof(PT) == sizeof(float)) {  // mixed: FP32 slice for the sources, FP64 con2prim metric from global
      const TileIn<R, PT, SD, SliceCol<R>, LazyCol<double>> in{G, x, sp, sfx, sfr, SliceCol<R>{slice, (unsigned)a},
                                                             LazyCol<double>{global_col(G.centre, G, ij)}};
      cell_core<R, PT>(G, ia, jb, x, mode, dt, in, Pout);
    } else {
      const TileIn<R, PT, SD, SliceCol<R>, SliceCol<R>> in{G, x, sp, sfx, sfr, SliceCol<R>{slice, (unsigned)a},
                                                           SliceCol<R>{slice, (unsigned)a}};
      cell_core<R, PT>(G, ia, jb, x, mode, dt, in, Pout);
    }
  } else {
    if constexpr (sizeof(PT) == sizeof(float)) {
      const TileIn<R, PT, SD, GlobalCol<R>, LazyCol<double>> in{G, x, sp, sfx, sfr, global_col(centre_table<R>(G), G, ij),
                                                              LazyCol<double>{global_col(G.centre, G, ij)}};
      cell_core<R, PT>(G, ia, jb, x, mode, dt, in, Pout);
    } else {
      const TileIn<R, PT, SD, GlobalCol<R>, GlobalCol<double>> in{G, x, sp, sfx, sfr, global_col(centre_table<R>(G), G, ij),
                                                                  global_col(G.centre, G, ij)};
      cell_core<R, PT>(G, ia, jb, x, mode, dt, in, Pout);
    }
  }
}

// Batched: block b works on tile map[b] of the launch.
template <int SD, int REC, int RS, class R, class PT>
__global__ void __launch_bounds__(STAGE_BS, stage_min_blocks<R>())
    k_stage(const GridDev *__restrict__ grids, const BlockMap *__restrict__ map, int mode) {
  extern __shared__ __align__(16) unsigned char stage_smem[];
  stage_tile<SD, REC, RS, R, PT>(grids, map[blockIdx.x], mode, stage_smem);
}

}  // namespace grhd
