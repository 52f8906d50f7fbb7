// cell_launch.cuh -- host launcher of the stage cell kernel, instantiated per precision in
// cell_fp64.cu / cell_fp32.cu (each precision compiled with its own floating-point flags,
// the same as the face kernels and the persistent kernel of that precision).
#pragma once

#include "flux_launch.h"
#include "cell.cuh"

namespace grhd {

static_assert(CELL_BS == CELL_BS_STAGE, "the cell kernel's staging layout is per block thread");

// dirs: the most active directions of any grid in the launch (sizes the staging buffers)
template <class R, class PT>
void launch_cell(int mode, const GridDev *grids, const BlockMap *map, int nblocks, int dirs, cudaStream_t s) {
  if (nblocks <= 0) return;
  const unsigned nb = (unsigned)nblocks;
  const size_t smem = slice_bytes<R>() + cell_stage_bytes<R, PT>(dirs);
  switch (mode) {
    case 0: k_cell_update<0, R, PT><<<nb, CELL_BS, smem, s>>>(grids, map); break;
    case 1: k_cell_update<1, R, PT><<<nb, CELL_BS, smem, s>>>(grids, map); break;
    case 2: k_cell_update<2, R, PT><<<nb, CELL_BS, smem, s>>>(grids, map); break;
    default: k_cell_update<3, R, PT><<<nb, CELL_BS, smem, s>>>(grids, map); break;
  }
}

}  // namespace grhd
