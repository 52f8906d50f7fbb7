// flux_fp64_z.cu -- fused face-flux kernels of direction z, double instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_flux_dir<3, double, double>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
