// riemann_fp64.cu -- Riemann kernels, double instantiation (see flux.cuh).
#include "flux_launch.cuh"

namespace grhd {
template void launch_riemann<double>(int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
