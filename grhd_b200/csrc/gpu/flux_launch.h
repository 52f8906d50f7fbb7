// flux_launch.h -- declarations of the batched face-flux launchers (defined in recon_*.cu
// and riemann_*.cu) for the API translation unit.
#pragma once

#include <cuda_runtime.h>

namespace grhd {

struct GridDev;
struct BlockMap;

// block sizes of the batched kernels (items per block: faces or cells)
constexpr int RECON_BS = 256;
constexpr int RIEMANN_BS = 128;
constexpr int CELL_BS = 128;
constexpr int FUSED_FLUX_BS = 128;  // k_flux (flux.cuh FLUX_BS)

template <class R, class PT>
void launch_recon(int dir, int rec, bool per_variable, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s);
template <class R>
void launch_riemann(int dir, int rs, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s);

template <int DIR, class R, class PT>
void launch_flux_dir(int rec, int rs, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s);

#define GRHD_FLUX_EXTERN(D, R, PT) \
  extern template void launch_flux_dir<D, R, PT>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
GRHD_FLUX_EXTERN(1, double, double)
GRHD_FLUX_EXTERN(2, double, double)
GRHD_FLUX_EXTERN(3, double, double)
GRHD_FLUX_EXTERN(1, float, float)
GRHD_FLUX_EXTERN(2, float, float)
GRHD_FLUX_EXTERN(3, float, float)
#undef GRHD_FLUX_EXTERN

// stage cell kernel (cell_fp64.cu / cell_fp32.cu): mode 0 RHS only, 1..3 RK stages
template <class R, class PT>
void launch_cell(int mode, const GridDev *grids, const BlockMap *map, int nblocks, int dirs, cudaStream_t s);
extern template void launch_cell<double, double>(int, const GridDev *, const BlockMap *, int, int, cudaStream_t);
extern template void launch_cell<float, float>(int, const GridDev *, const BlockMap *, int, int, cudaStream_t);

// stage kernel (stage.cuh): one whole RK stage (mode 1..3) of 1D grids (sd 0), x-y grids
// (sd 2) or x-z grids (sd 3); tiles of STAGE_TILE_CELLS cells (256 along i, or 32 x 8),
// one block of STAGE_BLOCK threads each
constexpr int STAGE_TILE_CELLS = 256;
constexpr int STAGE_BLOCK = 288;
template <int SD, class R, class PT>
cudaError_t stage_setup_sd(int rec, int rs);
template <int SD, class R, class PT>
void launch_stage_sd(int rec, int rs, int mode, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s);
#define GRHD_STAGE_EXTERN(SD, R)                                                                            \
  extern template cudaError_t stage_setup_sd<SD, R, R>(int, int);                                        \
  extern template void launch_stage_sd<SD, R, R>(int, int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
GRHD_STAGE_EXTERN(0, double)
GRHD_STAGE_EXTERN(2, double)
GRHD_STAGE_EXTERN(3, double)
GRHD_STAGE_EXTERN(0, float)
GRHD_STAGE_EXTERN(2, float)
GRHD_STAGE_EXTERN(3, float)
#undef GRHD_STAGE_EXTERN
// sets the kernel's dynamic shared-memory limit; call before the first launch (outside a
// stream capture)
template <class R, class PT>
inline cudaError_t stage_setup(int sd, int rec, int rs) {
  return sd == 0 ? stage_setup_sd<0, R, PT>(rec, rs) : (sd == 2 ? stage_setup_sd<2, R, PT>(rec, rs) : stage_setup_sd<3, R, PT>(rec, rs));
}
template <class R, class PT>
inline void launch_stage(int sd, int rec, int rs, int mode, const GridDev *grids, const BlockMap *map, int nblocks,
                         cudaStream_t s) {
  if (sd == 0) launch_stage_sd<0, R, PT>(rec, rs, mode, grids, map, nblocks, s);
  else if (sd == 2) launch_stage_sd<2, R, PT>(rec, rs, mode, grids, map, nblocks, s);
  else launch_stage_sd<3, R, PT>(rec, rs, mode, grids, map, nblocks, s);
}

// persistent step kernel (persistent.cuh): one contiguous range of items of a phase --
// the faces of one direction of one grid (dir 1..3) or the cells of one grid (dir 0)
struct Segment {
  int grid, dir;
  long long first, count;
};
struct PersistentArgs {
  const GridDev *grids;
  const int *members;
  int nmembers;
  const Segment *seg_face;
  int nseg_face;
  long long n_face;
  const Segment *seg_cell;
  int nseg_cell;
  long long n_cell;
  unsigned *bar;     // barrier words: arrivals, generation
  unsigned *status;  // nonzero: a barrier timed out
};
// query: *max_blocks = resident blocks of the (rec, rs) instantiation; else launch nsteps
// steps on nblocks blocks (cooperative launch)
template <class R, class PT>
cudaError_t run_persistent(int rec, int rs, bool query, int *max_blocks, const PersistentArgs &a, int nsteps,
                           int nblocks, cudaStream_t s);
extern template cudaError_t run_persistent<double, double>(int, int, bool, int *, const PersistentArgs &, int, int,
                                                           cudaStream_t);
extern template cudaError_t run_persistent<float, float>(int, int, bool, int *, const PersistentArgs &, int, int,
                                                         cudaStream_t);

// persistent stage kernel (persistent.cuh): whole steps of a group of 1D grids in one
// cooperative launch over the stage kernel's tiles (the group's K_STAGE block map)
struct PersistentStageArgs {
  const GridDev *grids;
  const BlockMap *tiles;
  int ntiles;
  const int *members;
  int nmembers;
  unsigned *bar;
  unsigned *status;
};
template <class R, class PT>
cudaError_t run_persistent_stage(int rec, int rs, bool query, int *max_blocks, const PersistentStageArgs &a,
                                 int nsteps, int nblocks, cudaStream_t s);
extern template cudaError_t run_persistent_stage<double, double>(int, int, bool, int *, const PersistentStageArgs &,
                                                                 int, int, cudaStream_t);
extern template cudaError_t run_persistent_stage<float, float>(int, int, bool, int *, const PersistentStageArgs &,
                                                               int, int, cudaStream_t);

// fused face fluxes of direction dir (recon + Riemann in one kernel)
template <class R, class PT>
inline void launch_flux(int dir, int rec, int rs, const GridDev *grids, const BlockMap *map, int nblocks,
                        cudaStream_t s) {
  if (dir == 1) launch_flux_dir<1, R, PT>(rec, rs, grids, map, nblocks, s);
  else if (dir == 2) launch_flux_dir<2, R, PT>(rec, rs, grids, map, nblocks, s);
  else launch_flux_dir<3, R, PT>(rec, rs, grids, map, nblocks, s);
}

extern template void launch_recon<double, double>(int, int, bool, const GridDev *, const BlockMap *, int, cudaStream_t);
extern template void launch_recon<float, float>(int, int, bool, const GridDev *, const BlockMap *, int, cudaStream_t);
extern template void launch_riemann<double>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
extern template void launch_riemann<float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);

}  // namespace grhd
