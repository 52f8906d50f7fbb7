// flux_launch.cuh -- host launchers of the face-flux kernels (compile-time dispatch on the
// reconstruction scheme and the Riemann solver).  Included by one translation unit per
// precision and kernel kind (recon_fp64.cu, riemann_fp64.cu, ...) so they compile in
// parallel.  Every launch is batched: `map` lists, per block, the grid and its first face.
#pragma once

#include "flux.cuh"
#include "flux_launch.h"

namespace grhd {

template <int DIR, class R, class PT>
inline void recon_dir(int rec, bool per_variable, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s) {
  const unsigned nb = (unsigned)nblocks;
  if (per_variable) {
    const dim3 grid(nb, 5);
    switch (rec) {
      case REC_GODUNOV: k_recon_var<DIR, REC_GODUNOV, R, PT><<<grid, RECON_BS, 0, s>>>(grids, map); break;
      case REC_TVD: k_recon_var<DIR, REC_TVD, R, PT><<<grid, RECON_BS, 0, s>>>(grids, map); break;
      case REC_WENO3: k_recon_var<DIR, REC_WENO3, R, PT><<<grid, RECON_BS, 0, s>>>(grids, map); break;
      case REC_MP5: k_recon_var<DIR, REC_MP5, R, PT><<<grid, RECON_BS, 0, s>>>(grids, map); break;
      default: k_recon_var<DIR, REC_WENO5, R, PT><<<grid, RECON_BS, 0, s>>>(grids, map); break;
    }
    return;
  }
  switch (rec) {
    case REC_GODUNOV: k_recon<DIR, REC_GODUNOV, R, PT><<<nb, RECON_BS, 0, s>>>(grids, map); break;
    case REC_TVD: k_recon<DIR, REC_TVD, R, PT><<<nb, RECON_BS, 0, s>>>(grids, map); break;
    case REC_WENO3: k_recon<DIR, REC_WENO3, R, PT><<<nb, RECON_BS, 0, s>>>(grids, map); break;
    case REC_MP5: k_recon<DIR, REC_MP5, R, PT><<<nb, RECON_BS, 0, s>>>(grids, map); break;
    default: k_recon<DIR, REC_WENO5, R, PT><<<nb, RECON_BS, 0, s>>>(grids, map); break;
  }
}

template <class R, class PT>
void launch_recon(int dir, int rec, bool per_variable, const GridDev *grids, const BlockMap *map, int nblocks,
                  cudaStream_t s) {
  if (nblocks <= 0) return;
  if (dir == 1) recon_dir<1, R, PT>(rec, per_variable, grids, map, nblocks, s);
  else if (dir == 2) recon_dir<2, R, PT>(rec, per_variable, grids, map, nblocks, s);
  else recon_dir<3, R, PT>(rec, per_variable, grids, map, nblocks, s);
}

template <class R>
void launch_riemann(int dir, int rs, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s) {
  if (nblocks <= 0) return;
  const unsigned nb = (unsigned)nblocks;
  if (rs == RS_HLLC) {
    if (dir == 1) k_riemann<1, RS_HLLC, R><<<nb, 128, 0, s>>>(grids, map);
    else if (dir == 2) k_riemann<2, RS_HLLC, R><<<nb, 128, 0, s>>>(grids, map);
    else k_riemann<3, RS_HLLC, R><<<nb, 128, 0, s>>>(grids, map);
  } else {
    if (dir == 1) k_riemann<1, RS_HLLE, R><<<nb, 128, 0, s>>>(grids, map);
    else if (dir == 2) k_riemann<2, RS_HLLE, R><<<nb, 128, 0, s>>>(grids, map);
    else k_riemann<3, RS_HLLE, R><<<nb, 128, 0, s>>>(grids, map);
  }
}

template <int DIR, int REC, class R, class PT>
inline void flux_rs(int rs, const GridDev *grids, const BlockMap *map, unsigned nb, cudaStream_t s) {
  if (rs == RS_HLLC) k_flux<DIR, REC, RS_HLLC, R, PT><<<nb, FLUX_BS, 0, s>>>(grids, map);
  else k_flux<DIR, REC, RS_HLLE, R, PT><<<nb, FLUX_BS, 0, s>>>(grids, map);
}

template <int DIR, class R, class PT>
void launch_flux_dir(int rec, int rs, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s) {
  if (nblocks <= 0) return;
  const unsigned nb = (unsigned)nblocks;
  switch (rec) {
    case REC_GODUNOV: flux_rs<DIR, REC_GODUNOV, R, PT>(rs, grids, map, nb, s); break;
    case REC_TVD: flux_rs<DIR, REC_TVD, R, PT>(rs, grids, map, nb, s); break;
    case REC_WENO3: flux_rs<DIR, REC_WENO3, R, PT>(rs, grids, map, nb, s); break;
    case REC_MP5: flux_rs<DIR, REC_MP5, R, PT>(rs, grids, map, nb, s); break;
    default: flux_rs<DIR, REC_WENO5, R, PT>(rs, grids, map, nb, s); break;
  }
}

}  // namespace grhd
