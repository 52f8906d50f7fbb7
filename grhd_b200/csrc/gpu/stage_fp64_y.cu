// stage_fp64_y.cu -- stage kernels of x-y grids, double instantiation (see stage.cuh).
#include "stage_launch.cuh"

namespace grhd {
template cudaError_t stage_setup_sd<2, double, double>(int, int);
template void launch_stage_sd<2, double, double>(int, int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
