// cell_launch.cuh -- host launcher of the stage cell kernel, instantiated per precision in
// cell_fp64.cu / cell_fp32.cu (each precision compiled with its own floating-point flags,
// the same as the face kernels and the persistent kernel of that precision).
#pragma once

#include "flux_launch.h"
#include "cell.cuh"

namespace grhd {

template <class R, class PT>
void launch_cell(int mode, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s) {
  if (nblocks <= 0) return;
  const unsigned nb = (unsigned)nblocks;
  switch (mode) {
    case 0: k_cell_update<0, R, PT><<<nb, CELL_BS, 0, s>>>(grids, map); break;
    case 1: k_cell_update<1, R, PT><<<nb, CELL_BS, 0, s>>>(grids, map); break;
    case 2: k_cell_update<2, R, PT><<<nb, CELL_BS, 0, s>>>(grids, map); break;
    default: k_cell_update<3, R, PT><<<nb, CELL_BS, 0, s>>>(grids, map); break;
  }
}

}  // namespace grhd
