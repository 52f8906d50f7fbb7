// flux_fp64_x.cu -- fused face-flux kernels of direction x, double instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_flux_dir<1, double, double>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
