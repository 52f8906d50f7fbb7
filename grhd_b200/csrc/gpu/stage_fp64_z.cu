// stage_fp64_z.cu -- stage kernels of x-z grids, double instantiation (see stage.cuh).
#include "stage_launch.cuh"

namespace grhd {
template cudaError_t stage_setup_sd<3, double, double>(int, int);
template void launch_stage_sd<3, double, double>(int, int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
