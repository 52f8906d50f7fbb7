// flux_fp32_x.cu -- fused face-flux kernels of direction x, float instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_flux_dir<1, float, float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
