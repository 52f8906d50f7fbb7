// Check program for grhd::rcp_mixed (physics.cuh): the mixed policy's FP64 reciprocal
// against the correctly rounded 1.0 / x that CUDA computes, on seeded random positive
// normal x.  Prints, per exponent range, the largest difference in units in the last place
// and the largest relative error.  Built and run by tests/test_gpu_rcp.py.
#include <cstdio>
#include <cstring>

#include "physics.cuh"

__device__ unsigned long long g_ulp[2], g_rel[2];

__global__ void check(long long n, unsigned long long seed, int range, int emax) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  unsigned long long h = (unsigned long long)t * 6364136223846793005ULL + seed;
  h ^= h >> 29;
  h *= 0xbf58476d1ce4e5b9ULL;
  h ^= h >> 32;
  const int ex = (int)(h % (unsigned long long)(2 * emax + 1)) - emax;
  const double m = 1.0 + (double)(h >> 11) * (1.0 / 9007199254740992.0);  // [1, 2)
  const double x = ldexp(m, ex);
  const double ref = 1.0 / x;
  const double r = grhd::rcp_mixed(x);
  long long d = __double_as_longlong(r) - __double_as_longlong(ref);
  if (d < 0) d = -d;
  atomicMax(&g_ulp[range], (unsigned long long)d);
  const double rel = fabs(r - ref) / ref;
  atomicMax(&g_rel[range], (unsigned long long)__double_as_longlong(rel));
}

int main() {
  const long long n = 1LL << 24;
  const int bs = 256;
  const unsigned nb = (unsigned)((n + bs - 1) / bs);
  const int emax[2] = {60, 1000};  // con2prim's range; almost all normal doubles
  for (int range = 0; range < 2; ++range)
    for (int s = 0; s < 4; ++s) check<<<nb, bs>>>(n, 0x9e3779b97f4a7c15ULL * (s + 1) + range, range, emax[range]);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    printf("error %s\n", cudaGetErrorString(e));
    return 1;
  }
  unsigned long long ulp[2], rel[2];
  cudaMemcpyFromSymbol(ulp, g_ulp, sizeof(ulp));
  cudaMemcpyFromSymbol(rel, g_rel, sizeof(rel));
  for (int range = 0; range < 2; ++range) {
    double r;
    memcpy(&r, &rel[range], sizeof(r));
    printf("range %d emax %d samples %lld max_ulp %llu max_rel %.3e\n", range, emax[range], 4 * n, ulp[range], r);
  }
  return 0;
}
