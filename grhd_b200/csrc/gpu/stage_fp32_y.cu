// stage_fp32_y.cu -- stage kernels of x-y grids, float instantiation (see stage.cuh).
#include "stage_launch.cuh"

namespace grhd {
template cudaError_t stage_setup_sd<2, float, float>(int, int);
template void launch_stage_sd<2, float, float>(int, int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
