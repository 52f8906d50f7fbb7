// flux_fp32_z.cu -- fused face-flux kernels of direction z, float instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_flux_dir<3, float, float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
