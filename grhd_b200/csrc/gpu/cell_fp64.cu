// cell_fp64.cu -- stage cell kernel, double instantiation (see cell.cuh).
#include "cell_launch.cuh"

namespace grhd {
template void launch_cell<double, double>(int, const GridDev *, const BlockMap *, int, int, cudaStream_t);
}  // namespace grhd
