// persistent.cuh -- whole SSP-RK3 steps of every grid of a scheme group in one launch.
//
// For batches of small grids (the 1D Riemann and Michel solves of the serving workload)
// the stage kernels are launch-bound: each of the ~10 launches of a step finishes in a
// few microseconds.  k_persistent runs nsteps steps in one cooperative launch instead.
// Each stage has two phases over flattened item spaces that span every grid of the group:
//   A  fused face fluxes (recon + Riemann, flux.cuh flux_item) of every active direction,
//   B  the cell update of the stage (cell.cuh cell_item),
// and after the third stage every grid's clock advances.  Phases are separated by a grid
// barrier; the launch is cooperative, so all blocks are resident and the barrier
// completes.  The barrier still waits a bounded time: on a timeout the block sets the
// status word and returns, and every other block stops at its next barrier.
//
// Arithmetic is the stage kernels' (same device functions): FP64 results are bit-identical
// to the stage path; under the mixed policy the FP32 parts may round differently where the
// compiler contracts a different multiply-add pair.  Loads of state that other blocks write
// during the launch go through L2 (GRHD_LDP and -dlcm=cg in the persistent translation
// units).
#pragma once

#include "cell.cuh"
#include "flux.cuh"
#include "flux_launch.h"
#include "stage.cuh"

namespace grhd {

constexpr long long BARRIER_SPIN_LIMIT = 1LL << 24;  // x >= 64 ns sleeps: a second or more

// Grid-wide barrier over nblocks resident blocks.  bar[0] counts arrivals, bar[1] is the
// generation; status != 0 means some block gave up.  Returns false if this block gave up
// or saw another block give up.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned nblocks, unsigned *status) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned *gen = bar + 1;
    volatile unsigned *st = status;
    const unsigned g0 = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*gen == g0) {
        if (*st != 0u || ++spins > BARRIER_SPIN_LIMIT) {
          atomicOr(status, 1u);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (*st != 0u) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

// segment holding item it (segments sorted by first, it < total)
__device__ __forceinline__ int find_segment(const Segment *__restrict__ seg, int nseg, long long it) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid].first <= it) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int REC, int RS, class R, class PT>
__global__ void __launch_bounds__(FLUX_BS)
    k_persistent(const GridDev *__restrict__ grids, const int *__restrict__ members, int nmembers,
                 const Segment *__restrict__ seg_face, int nseg_face, long long n_face,
                 const Segment *__restrict__ seg_cell, int nseg_cell, long long n_cell, int nsteps, unsigned *bar,
                 unsigned *status) {
  __shared__ R sq[2 * NEQ][FLUX_BS];
  const unsigned nblk = gridDim.x;
  const long long stride = (long long)nblk * FLUX_BS;
  for (int step = 0; step < nsteps; ++step) {
    for (int stage = 1; stage <= 3; ++stage) {
      for (long long it = (long long)blockIdx.x * FLUX_BS + threadIdx.x; it < n_face; it += stride) {
        const Segment sg = seg_face[find_segment(seg_face, nseg_face, it)];
        const GridDev &G = grids[sg.grid];
        const unsigned f = (unsigned)(it - sg.first);
        if (sg.dir == 1) {
          const unsigned r = fdiv(f, G.div_nx1), k = fdiv(r, G.div_ny);
          flux_item<1, REC, RS, R, PT>(G, f - r * G.div_nx1.d, r - k * G.div_ny.d, k, sq);
        } else if (sg.dir == 2) {
          const unsigned r = fdiv(f, G.div_nx), k = fdiv(r, G.div_ny1);
          flux_item<2, REC, RS, R, PT>(G, f - r * G.div_nx.d, r - k * G.div_ny1.d, k, sq);
        } else {
          const unsigned r = fdiv(f, G.div_nx), k = fdiv(r, G.div_ny);
          flux_item<3, REC, RS, R, PT>(G, f - r * G.div_nx.d, r - k * G.div_ny.d, k, sq);
        }
      }
      if (!grid_barrier(bar, nblk, status)) return;
      for (long long it = (long long)blockIdx.x * FLUX_BS + threadIdx.x; it < n_cell; it += stride) {
        const Segment sg = seg_cell[find_segment(seg_cell, nseg_cell, it)];
        const GridDev &G = grids[sg.grid];
        const unsigned c = (unsigned)(it - sg.first);
        const unsigned r = fdiv(c, G.div_nx), k = fdiv(r, G.div_ny);
        cell_item<R, PT>(G, c - r * G.div_nx.d, r - k * G.div_ny.d, k, stage);
      }
      if (!grid_barrier(bar, nblk, status)) return;
    }
    for (long long it = (long long)blockIdx.x * FLUX_BS + threadIdx.x; it < nmembers; it += stride)
      advance_clock(grids[members[it]].clock);
    if (!grid_barrier(bar, nblk, status)) return;
  }
}

// Whole steps of a group of 1D grids in one cooperative launch, built on the stage kernel
// (stage.cuh): each stage is one pass of the group's tiles (the stage kernel's block map,
// ntiles entries) spread over the resident blocks, then one grid barrier; after the third
// stage every grid's clock advances, then a barrier.  Four barriers per step, against seven
// for k_persistent, and the stage kernel's tile work (faces and cells through shared
// memory).  The primitives rotate through P, P2, P3 as in the stage kernel, so a stage
// never reads what it writes; what another block wrote in an earlier stage is read through
// L2 (GRHD_LDP, -dlcm=cg in this translation unit).
template <int REC, int RS, class R, class PT>
__global__ void __launch_bounds__(STAGE_BS, stage_min_blocks<R>())
    k_persistent_stage(const GridDev *__restrict__ grids, const BlockMap *__restrict__ tiles, int ntiles,
                       const int *__restrict__ members, int nmembers, int nsteps, unsigned *bar, unsigned *status) {
  extern __shared__ __align__(16) unsigned char stage_smem[];
  const unsigned nblk = gridDim.x;
  for (int step = 0; step < nsteps; ++step) {
    for (int mode = 1; mode <= 3; ++mode) {
      for (int t = (int)blockIdx.x; t < ntiles; t += (int)nblk) {
        __syncthreads();  // the previous tile's cell phase is done with shared memory
        stage_tile<0, REC, RS, R, PT>(grids, tiles[t], mode, stage_smem);
      }
      if (!grid_barrier(bar, nblk, status)) return;
    }
    for (int it = (int)(blockIdx.x * STAGE_BS + threadIdx.x); it < nmembers; it += (int)(nblk * STAGE_BS))
      advance_clock(grids[members[it]].clock);
    if (!grid_barrier(bar, nblk, status)) return;
  }
}

template <int REC, int RS, class R, class PT>
inline cudaError_t persistent_stage_rs(bool query, int *max_blocks, const PersistentStageArgs &a, int nsteps,
                                       int nblocks, cudaStream_t s) {
  auto kern = k_persistent_stage<REC, RS, R, PT>;
  const size_t smem = stage_smem_bytes<0, R>();
  if (query) {
    int per_sm = 0, dev = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, STAGE_BS, smem);
    if (e != cudaSuccess) return e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    *max_blocks = per_sm * sms;
    return cudaSuccess;
  }
  const GridDev *g = a.grids;
  const BlockMap *tl = a.tiles;
  int nt = a.ntiles;
  const int *m = a.members;
  int nm = a.nmembers;
  unsigned *bar = a.bar, *st = a.status;
  void *args[] = {&g, &tl, &nt, &m, &nm, &nsteps, &bar, &st};
  return cudaLaunchCooperativeKernel((const void *)kern, dim3((unsigned)nblocks), dim3(STAGE_BS), args, smem, s);
}

template <class R, class PT>
cudaError_t run_persistent_stage(int rec, int rs, bool query, int *max_blocks, const PersistentStageArgs &a,
                                 int nsteps, int nblocks, cudaStream_t s) {
#define GRHD_PERSIST_REC(RC)                                                                                \
  return rs == RS_HLLC ? persistent_stage_rs<RC, RS_HLLC, R, PT>(query, max_blocks, a, nsteps, nblocks, s) \
                       : persistent_stage_rs<RC, RS_HLLE, R, PT>(query, max_blocks, a, nsteps, nblocks, s)
  switch (rec) {
    case REC_GODUNOV: GRHD_PERSIST_REC(REC_GODUNOV);
    case REC_TVD: GRHD_PERSIST_REC(REC_TVD);
    case REC_WENO3: GRHD_PERSIST_REC(REC_WENO3);
    case REC_MP5: GRHD_PERSIST_REC(REC_MP5);
    default: GRHD_PERSIST_REC(REC_WENO5);
  }
#undef GRHD_PERSIST_REC
}

// Host side: maximum resident blocks of the instantiation for (rec, rs), and the launch.
template <int REC, int RS, class R, class PT>
inline cudaError_t persistent_rs(bool query, int *max_blocks, const PersistentArgs &a, int nsteps, int nblocks,
                                 cudaStream_t s) {
  auto kern = k_persistent<REC, RS, R, PT>;
  if (query) {
    int per_sm = 0, dev = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FLUX_BS, 0);
    if (e != cudaSuccess) return e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    *max_blocks = per_sm * sms;
    return cudaSuccess;
  }
  const GridDev *g = a.grids;
  const int *m = a.members;
  int nm = a.nmembers;
  const Segment *sf = a.seg_face;
  int nsf = a.nseg_face;
  long long nf = a.n_face;
  const Segment *sc = a.seg_cell;
  int nsc = a.nseg_cell;
  long long nc = a.n_cell;
  unsigned *bar = a.bar, *st = a.status;
  void *args[] = {&g, &m, &nm, &sf, &nsf, &nf, &sc, &nsc, &nc, &nsteps, &bar, &st};
  return cudaLaunchCooperativeKernel((const void *)kern, dim3((unsigned)nblocks), dim3(FLUX_BS), args, 0, s);
}

template <class R, class PT>
cudaError_t run_persistent(int rec, int rs, bool query, int *max_blocks, const PersistentArgs &a, int nsteps,
                           int nblocks, cudaStream_t s) {
#define GRHD_PERSIST_REC(RC)                                                                        \
  return rs == RS_HLLC ? persistent_rs<RC, RS_HLLC, R, PT>(query, max_blocks, a, nsteps, nblocks, s) \
                       : persistent_rs<RC, RS_HLLE, R, PT>(query, max_blocks, a, nsteps, nblocks, s)
  switch (rec) {
    case REC_GODUNOV: GRHD_PERSIST_REC(REC_GODUNOV);
    case REC_TVD: GRHD_PERSIST_REC(REC_TVD);
    case REC_WENO3: GRHD_PERSIST_REC(REC_WENO3);
    case REC_MP5: GRHD_PERSIST_REC(REC_MP5);
    default: GRHD_PERSIST_REC(REC_WENO5);
  }
#undef GRHD_PERSIST_REC
}

}  // namespace grhd
