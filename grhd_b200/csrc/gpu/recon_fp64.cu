// recon_fp64.cu -- reconstruction kernels, double instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_recon<double, double>(int, int, bool, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
