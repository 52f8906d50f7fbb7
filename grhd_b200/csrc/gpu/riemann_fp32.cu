// riemann_fp32.cu -- Riemann kernels, float instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_riemann<float>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
