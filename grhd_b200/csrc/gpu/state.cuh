// state.cuh -- device layout of one grid and the boundary fill evaluated on load.
//
// Primitives are stored for interior cells only, structure-of-arrays: plane v holds
// p(v, 1:nx, 1:ny, 1:nz) with i fastest.  Ghost cells are never stored: a stencil load
// that leaves the domain along one direction returns the value set_boundary_conditions
// (conditions.f90:773-1066) would have written there.  calc_rhs reads only ghost cells
// that are outside the domain in exactly one direction (its strips, evolution.f90:60,
// :112, :164, run through interior cells), and each such ghost is a function of one
// interior cell plus static data, so evaluating it on load is exact.
//
// One ghost index is never written by the reference's boundary routines: -nghost (the
// loops fill 1-g for g = 1..nghost).  It keeps whatever the caller's array held when the
// state was uploaded (the jet case re-initialises it to the ambient state every call,
// conditions.f90:824-835).  Only the shock sensor of nghost = 2 schemes reads it
// (reconstruction.f90:334-341 at face 0); those values are kept in "frozen" slabs.
#pragma once

#include "physics.cuh"

namespace grhd {

// centre table fields (per (i,j); the metric cache is k-invariant)
enum CentreField {
  CF_ALPHA = 0, CF_B1, CF_B2, CF_B3,
  CF_G11, CF_G12, CF_G13, CF_G22, CF_G23, CF_G33,
  CF_I11, CF_I12, CF_I13, CF_I22, CF_I23, CF_I33,
  CF_SQG,
  CF_GM = 17,    // g^{mu nu}, 10 symmetric entries
  CF_CH0 = 27,   // Gamma^0_{mu nu}, 10 symmetric entries
  CF_DG = 37,    // d_d g_{mu nu}, d = 1..3, 10 symmetric entries each
  CF_DLNA = 67,  // d_mu ln(alpha), 4 entries
  CF_VA = 71,    // beta^i / alpha, i = 1..3 (the shift-aware outflow clamp, conditions.f90:926,
                 // and the four-velocity of the sources, metrics.f90:1251-1310): the quotient
                 // of the same operands the reference divides per cell, rounded once
  NCF = 74
};
// face table fields (per face of one direction)
enum FaceField {
  FF_ALPHA = 0, FF_BETA_N, FF_G11, FF_G12, FF_G13, FF_G22, FF_G23, FF_G33, FF_SQG, FF_GUP,
  FF_COF = 10,  // coframe(a,i) at FF_COF + 3a + i
  FF_FRAME_OK = 19, FF_ZERO = 20, NFF = 21
};

__host__ __device__ __forceinline__ int sym4(int mu, int nu) {
  if (mu > nu) { int t = mu; mu = nu; nu = t; }
  // 00 01 02 03 11 12 13 22 23 33
  return mu == 0 ? nu : (mu == 1 ? 3 + nu : (mu == 2 ? 5 + nu : 9));
}

// Per-grid time keeping on the device.  mode 0: the caller passes dt (grhd2_gpu_step);
// mode 1: the grid steps with its CFL dt clamped to its final time (grhd2.f90:180-184)
// and deactivates when it reaches it, so steps of a batch can be replayed as one graph
// without host involvement.
struct GridClock {
  double t, final_time, dt_cfl, dt_explicit;
  long long steps, max_steps;
  int mode, active;
};
__host__ __device__ __forceinline__ double clock_dt(const GridClock &c) {
  if (c.mode == 0) return c.dt_explicit;
  return (c.t + c.dt_cfl > c.final_time) ? c.final_time - c.t : c.dt_cfl;
}
__host__ __device__ __forceinline__ bool clock_skip(const GridClock &c) { return c.mode == 1 && !c.active; }
// end of a step: t = t + dt, steps += 1 (grhd2.f90:229-230); a grid that reached its final
// time or step limit deactivates
__device__ __forceinline__ void advance_clock(GridClock *c) {
  if (c->mode == 1) {
    if (!c->active) return;
    c->t = c->t + clock_dt(*c);
    c->steps += 1;
    c->active = c->t < c->final_time && (c->max_steps < 0 || c->steps < c->max_steps);
  } else {
    c->steps += 1;
  }
}

// Loads of the primitives.  Within one stage kernel they are read-only (the non-coherent
// read-only path is safe); the persistent step kernel writes them between its phases, so
// its translation units read them through L2 (ld.global.cg), coherent across blocks.
#ifdef GRHD_PERSISTENT_TU
#define GRHD_LDP(ptr) __ldcg(ptr)
#else
#define GRHD_LDP(ptr) __ldg(ptr)
#endif

// Division by a grid extent with a multiply-high and a shift (Granlund and Montgomery,
// "Division by invariant integers using multiplication", 1994): for d >= 1 with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1, n / d = (umulhi(n, m) + n) >> l
// for every n < 2^31 (the sum cannot overflow).  Face and cell counts per grid are below
// 2^31 (checked at create), so the index decode needs no integer division instruction.
struct FastDiv {
  unsigned d, m, l;
};
inline FastDiv make_fastdiv(unsigned d) {
  unsigned l = 0;
  while ((1ull << l) < d) ++l;
  const unsigned long long m = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
  return FastDiv{d, (unsigned)m, l};
}
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv &f) { return (__umulhi(n, f.m) + n) >> f.l; }

// Block tile of a stage kernel over its index space (nI, nJ, nK) -- cells, or the faces of
// one direction.  A block of BS = 2^lb threads covers tx = 2^lx consecutive items along i,
// ty = 2^ly along j and tz = BS / (tx ty) along k; a warp always spans consecutive i, so
// loads stay coalesced, while the block's rows along j/k reuse the k-invariant metric
// tables and the stencil values of their neighbours through L1.  Tiles are numbered with
// i fastest: t = ti + nti (tj + ntj tk).
struct Tile {
  unsigned lx, ly;   // log2 of the tile extent along i and j
  FastDiv nti, ntj;  // tiles along i and j
};
enum TileKind { TILE_CELL = 0, TILE_RECON = 1, TILE_FACE = 4, NTILE = 7 };  // + DIR - 1 for faces

template <int LB>  // log2 of the block size
__device__ __forceinline__ bool tile_item(const Tile &T, unsigned t, unsigned tid, unsigned nI, unsigned nJ,
                                          unsigned nK, unsigned &a, unsigned &b, unsigned &c) {
  const unsigned r = fdiv(t, T.nti);
  const unsigned ti = t - r * T.nti.d;
  const unsigned tk = fdiv(r, T.ntj);
  const unsigned tj = r - tk * T.ntj.d;
  a = (ti << T.lx) + (tid & ((1u << T.lx) - 1u));
  b = (tj << T.ly) + ((tid >> T.lx) & ((1u << T.ly) - 1u));
  c = (tk << (LB - T.lx - T.ly)) + (tid >> (T.lx + T.ly));
  return a < nI && b < nJ && c < nK;
}

// Everything a kernel needs about one grid.  The stage kernels read these descriptors from
// a device array, one entry per grid of a batch (a single grid is a batch of one).
struct GridDev {
  // sizes
  int nx, ny, nz, ng;
  int case_id;
  FastDiv div_nx, div_ny, div_nx1, div_ny1;  // nx, ny, nx + 1, ny + 1
  Tile tiles[NTILE];                         // block tiles: cells, recon per direction, faces per direction
  long long ncell;   // nx*ny*nz
  long long pplane;  // plane stride of the primitive / conserved arrays (elements)
  // metric tables
  const double *centre;  // [NCF][nij]
  long long nij;
  const double *face[3];  // [NFF][nface_d]
  long long nface[3];
  // FP32 copies of the tables for the mixed policy's FP32 arithmetic (sources, Riemann
  // solver): the same values rounded once at upload instead of at every load; NULL for FP64
  const float *centre_f;
  const float *face_f[3];
  // boundary data
  const double *inj;     // Michel injector [v][g][j][k]  (5*g*ny*nz)
  const double *dust;    // [v][g]
  const double *xc;      // x(-g:nx+g)
  const double *frozen[3];  // -nghost slabs [v][..] (nghost == 2 only)
  double jet[7];
  double rho_floor, p_floor;
  // physics of the grid (adiabatic index, floors, limiter, sensor, metric flags)
  Phys phys;
  double dx, dy, dz;
  // the grid's device state
  void *P;                      // primitives (double or float planes)
  void *Prot[2];                // the stage kernel's rotation buffers P2, P3 (1D and 2D grids; stage.cuh)
  FastDiv stage_ntx;            // stage-kernel tiles along i
  double *U, *UP, *RHS;         // conserved u, up; RHS scratch of grhd2_gpu_calc_rhs
  void *Uc, *UPc;               // carries of the compensated accumulation (u + Uc, up + UPc)
  int carry;                    // 0: none, 1: FP64 carries, 2: FP32 carries
  void *F[3];                   // face fluxes per direction
  void *Q;                      // interface states of the direction being processed
  unsigned long long *cnt;      // failure / floor counters
  GridClock *clock;             // device clock of the grid
};

// the table of the arithmetic type R (double: the FP64 tables; float: their FP32 copies)
template <class R> __device__ __forceinline__ const R *centre_table(const GridDev &G);
template <> __device__ __forceinline__ const double *centre_table<double>(const GridDev &G) { return G.centre; }
template <> __device__ __forceinline__ const float *centre_table<float>(const GridDev &G) { return G.centre_f; }
template <class R> __device__ __forceinline__ const R *face_table(const GridDev &G, int d);
template <> __device__ __forceinline__ const double *face_table<double>(const GridDev &G, int d) { return G.face[d]; }
template <> __device__ __forceinline__ const float *face_table<float>(const GridDev &G, int d) { return G.face_f[d]; }

// one block of a batched launch: the grid it works on and its first item (face or cell)
struct BlockMap {
  int grid, first;
};

// interior primitive read (1-based cell indices)
// (cell counts are below 2^31, so the linear cell index is computed in 32 bits)
__device__ __forceinline__ unsigned cell_index(const GridDev &G, int i, int j, int k) {
  return (unsigned)(i - 1) + (unsigned)G.nx * ((unsigned)(j - 1) + (unsigned)G.ny * (unsigned)(k - 1));
}
template <class PT>
__device__ __forceinline__ double ld_prim(const PT *__restrict__ P, const GridDev &G, int v, int i, int j, int k) {
  const unsigned c = cell_index(G, i, j, k);
  return (double)GRHD_LDP(&P[v * G.pplane + c]);
}
template <class PT>
__device__ __forceinline__ void ld_cell(const PT *__restrict__ P, const GridDev &G, int i, int j, int k, double (&q)[NEQ]) {
  const unsigned c = cell_index(G, i, j, k);
#pragma unroll
  for (int v = 0; v < NEQ; ++v) q[v] = (double)GRHD_LDP(&P[v * G.pplane + c]);
}
__device__ __forceinline__ int wrap(int i, int n) {  // periodic (whole-array statements per g) == modular
  int r = (i - 1) % n;
  if (r < 0) r += n;
  return r + 1;
}
__device__ __forceinline__ void jet_ambient(const GridDev &G, double (&q)[NEQ]) {
  q[EQ_DE] = G.jet[0]; q[EQ_PR] = G.jet[1]; q[EQ_VX] = 0.0; q[EQ_VY] = 0.0; q[EQ_VZ] = G.jet[2];
}

// Value of cell (i,j,k) where only the DIR index may lie outside [1, n_DIR].
template <int DIR, class PT>
__device__ __forceinline__ void load_cell(const PT *__restrict__ P, const GridDev &G, int i, int j, int k, double (&q)[NEQ]) {
  const int n = DIR == 1 ? G.nx : (DIR == 2 ? G.ny : G.nz);
  const int idx = DIR == 1 ? i : (DIR == 2 ? j : k);
  if (idx >= 1 && idx <= n) { ld_cell(P, G, i, j, k, q); return; }
  const int cs = G.case_id;
  if (idx == -G.ng) {  // never written by the boundary loops (see header)
    if (cs == 5) { jet_ambient(G, q); return; }
    const double *fz = G.frozen[DIR - 1];
    long long s, ns;
    if (DIR == 1) { s = (j - 1) + (long long)G.ny * (k - 1); ns = (long long)G.ny * G.nz; }
    else if (DIR == 2) { s = (i - 1) + (long long)G.nx * (k - 1); ns = (long long)G.nx * G.nz; }
    else { s = (i - 1) + (long long)G.nx * (j - 1); ns = (long long)G.nx * G.ny; }
#pragma unroll
    for (int v = 0; v < NEQ; ++v) q[v] = fz[v * ns + s];
    return;
  }
  const bool lo = idx < 1;
  const int g = lo ? 1 - idx : idx - n;
  if (DIR == 1) {
    switch (cs) {
      case 1: case 2: case 3:  // zero-gradient outflow, conditions.f90:795-798
        ld_cell(P, G, lo ? 1 : G.nx, j, k, q); return;
      case 4: case 6:  // periodic, conditions.f90:809-811
        ld_cell(P, G, wrap(i, G.nx), j, k, q); return;
      case 5:  // reflecting axis / ambient, conditions.f90:838-848
        if (lo) { ld_cell(P, G, g, j, k, q); q[EQ_VX] = -q[EQ_VX]; } else jet_ambient(G, q);
        return;
      case 7:  // copy inside, analytic injector outside, conditions.f90:872-883
        if (lo) ld_cell(P, G, 1, j, k, q);
        else {
#pragma unroll
          for (int v = 0; v < NEQ; ++v)
            q[v] = G.inj[(long long)v * G.ng * G.ny * G.nz + (g - 1) + (long long)G.ng * ((j - 1) + (long long)G.ny * (k - 1))];
        }
        return;
      case 8:  // dust, conditions.f90:896-907
        if (lo) {
          ld_cell(P, G, 1, j, k, q);
          q[EQ_DE] = rmax(q[EQ_DE], G.rho_floor);
          q[EQ_PR] = rmax(q[EQ_PR], G.p_floor);
          q[EQ_VX] = rmin(0.0, q[EQ_VX]);
        } else {
#pragma unroll
          for (int v = 0; v < NEQ; ++v) q[v] = G.dust[v * G.ng + (g - 1)];
        }
        return;
      default: {  // 9-12: shift-aware radial outflow, conditions.f90:916-938, :951-973, :1007-1026
        const int src = lo ? 1 : G.nx;
        ld_cell(P, G, src, j, k, q);
        const double d_in = q[EQ_DE];
        const double va = G.centre[(long long)CF_VA * G.nij + (src - 1) + (long long)G.nx * (j - 1)];
        q[EQ_DE] = rmax(q[EQ_DE], G.rho_floor);
        q[EQ_PR] = rmax(q[EQ_PR], G.p_floor);
        q[EQ_VX] = lo ? rmin(va, q[EQ_VX]) : rmax(va, q[EQ_VX]);
        if (lo && (cs == 9 || cs == 10) && d_in < 1.0e-6) { q[EQ_VY] = 0.0; q[EQ_VZ] = 0.0; }
        return;
      }
    }
  } else if (DIR == 2) {
    if (cs == 5) { jet_ambient(G, q); return; }  // reset to ambient, no y fill (conditions.f90:824-835)
    if (cs == 11) {  // reflecting poles, conditions.f90:977-988 (ny >= nghost enforced)
      ld_cell(P, G, i, lo ? g : G.ny + 1 - g, k, q);
      q[EQ_VY] = -q[EQ_VY];
      return;
    }
    if (cs == 12) {  // trans-polar, conditions.f90:1033-1050 (ny >= nghost, nz even enforced)
      int ks = k + G.nz / 2;
      if (ks > G.nz) ks -= G.nz;
      ld_cell(P, G, i, lo ? g : G.ny + 1 - g, ks, q);
      q[EQ_VY] = -q[EQ_VY];
      return;
    }
    ld_cell(P, G, i, wrap(j, G.ny), k, q);  // periodic
    return;
  } else {
    if (cs == 5) {  // nozzle inflow / reflecting wall below, outflow above, conditions.f90:851-869
      if (lo) {
        if (G.xc[i + G.ng] <= G.jet[3]) {
          q[EQ_DE] = G.jet[4]; q[EQ_PR] = G.jet[5]; q[EQ_VX] = 0.0; q[EQ_VY] = 0.0; q[EQ_VZ] = G.jet[6];
        } else {
          ld_cell(P, G, i, j, g, q);
          q[EQ_VZ] = -q[EQ_VZ];
        }
      } else {
        ld_cell(P, G, i, j, G.nz, q);
        q[EQ_VZ] = rmax(0.0, q[EQ_VZ]);
      }
      return;
    }
    ld_cell(P, G, i, j, wrap(k, G.nz), q);  // periodic
  }
}

}  // namespace grhd
