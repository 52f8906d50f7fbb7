// stage_fp32_z.cu -- stage kernels of x-z grids, float instantiation (see stage.cuh).
#include "stage_launch.cuh"

namespace grhd {
template cudaError_t stage_setup_sd<3, float, float>(int, int);
template void launch_stage_sd<3, float, float>(int, int, int, const GridDev *, const BlockMap *, int, cudaStream_t);
}  // namespace grhd
