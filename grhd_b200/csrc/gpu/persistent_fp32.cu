// persistent_fp32.cu -- persistent step kernels, float instantiation (see persistent.cuh).
// State written by other blocks of the same launch is read through L2 (GRHD_LDP here, and
// -dlcm=cg for the plain loads, set by the build for persistent_*.cu).
#define GRHD_PERSISTENT_TU
#include "persistent.cuh"

namespace grhd {
template cudaError_t run_persistent<float, float>(int, int, bool, int *, const PersistentArgs &, int, int, cudaStream_t);
template cudaError_t run_persistent_stage<float, float>(int, int, bool, int *, const PersistentStageArgs &, int, int,
                                                   cudaStream_t);
}  // namespace grhd
