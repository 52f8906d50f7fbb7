// stage_launch.cuh -- host launchers of the stage kernel (stage.cuh), compile-time dispatch
// on the reconstruction scheme and the Riemann solver.  Included by one translation unit
// per precision and tile shape (stage_fp64_x.cu: 1D grids, _y: x-y grids, _z: x-z grids).
#pragma once

#include "stage.cuh"
#include "flux_launch.h"

namespace grhd {

static_assert(STAGE_BS == STAGE_BLOCK && STAGE_CELLS == STAGE_TILE_CELLS, "the host's tile geometry is the kernel's");

template <int SD, int REC, class R, class PT>
inline const void *stage_fn(int rs) {
  return rs == RS_HLLC ? (const void *)k_stage<SD, REC, RS_HLLC, R, PT> : (const void *)k_stage<SD, REC, RS_HLLE, R, PT>;
}
template <int SD, class R, class PT>
inline const void *stage_kernel(int rec, int rs) {
  switch (rec) {
    case REC_GODUNOV: return stage_fn<SD, REC_GODUNOV, R, PT>(rs);
    case REC_TVD: return stage_fn<SD, REC_TVD, R, PT>(rs);
    case REC_WENO3: return stage_fn<SD, REC_WENO3, R, PT>(rs);
    case REC_MP5: return stage_fn<SD, REC_MP5, R, PT>(rs);
    default: return stage_fn<SD, REC_WENO5, R, PT>(rs);
  }
}

template <int SD, class R, class PT>
cudaError_t stage_setup_sd(int rec, int rs) {
  return cudaFuncSetAttribute(stage_kernel<SD, R, PT>(rec, rs), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)stage_smem_bytes<SD, R>());
}

template <int SD, class R, class PT>
void launch_stage_sd(int rec, int rs, int mode, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s) {
  if (nblocks <= 0) return;
  const void *fn = stage_kernel<SD, R, PT>(rec, rs);
  void *args[] = {(void *)&grids, (void *)&map, (void *)&mode};
  cudaLaunchKernel(fn, dim3((unsigned)nblocks), dim3(STAGE_BS), args, stage_smem_bytes<SD, R>(), s);
}

}  // namespace grhd
