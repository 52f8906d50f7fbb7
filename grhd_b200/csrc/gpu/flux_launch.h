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

template <class R, class PT>
void launch_recon(int dir, int rec, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s);
template <class R>
void launch_riemann(int dir, int rs, const GridDev *grids, const BlockMap *map, int nblocks, cudaStream_t s);

extern template void launch_recon<double, double>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
extern template void launch_recon<float, float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
extern template void launch_riemann<double>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
extern template void launch_riemann<float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);

}  // namespace grhd
