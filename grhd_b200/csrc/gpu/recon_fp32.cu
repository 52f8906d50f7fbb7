// recon_fp32.cu -- reconstruction kernels, float instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_recon<float, float>(int, int, bool, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
