// flux_fp32_y.cu -- fused face-flux kernels of direction y, float instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_flux_dir<2, float, float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
