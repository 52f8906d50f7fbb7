// persistent_fp64.cu -- persistent step kernels, double instantiation (see persistent.cuh).
// State written by other blocks of the same launch is read through L2 (GRHD_LDP here, and
// -dlcm=cg for the plain loads, set by the build for persistent_*.cu).
#define GRHD_PERSISTENT_TU
#include "persistent.cuh"

namespace grhd {
template cudaError_t run_persistent<double, double>(int, int, bool, int *, const PersistentArgs &, int, int, cudaStream_t);
template cudaError_t run_persistent_stage<double, double>(int, int, bool, int *, const PersistentStageArgs &, int, int,
                                                   cudaStream_t);
}  // namespace grhd
