// cell_fp32.cu -- stage cell kernel, float instantiation (see cell.cuh).
#include "cell_launch.cuh"

namespace grhd {
template void launch_cell<float, float>(int, const GridDev *, const BlockMap *, int, int, cudaStream_t);
}  // namespace grhd
