// common.cuh -- helpers shared by every kernel translation unit: failure/floor counters
// and the per-face table loads.
#pragma once

#include "state.cuh"

namespace grhd {

enum CounterIdx { CNT_FLOOR_PRE = 0, CNT_CAUSAL, CNT_BRENT, CNT_ROOT_FAIL, CNT_BAD_V, CNT_SANITISE,
                  CNT_RECON_CLAMP, CNT_HLLC_FALLBACK, NCNT };

// warp-aggregated counter increment (call from converged code)
// Warp-aggregated counter update: lanes are grouped by counter array (a warp of a
// persistent kernel can span two grids), one atomic per group.
__device__ __forceinline__ void count_add(unsigned long long *cnt, int idx, unsigned v) {
  const unsigned mask = __match_any_sync(__activemask(), (unsigned long long)cnt);
  const unsigned tot = __reduce_add_sync(mask, v);
  if (tot && (threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1)) atomicAdd(&cnt[idx], (unsigned long long)tot);
}

template <class R, class TT>
__device__ __forceinline__ FaceMetric<R> load_face_metric(const TT *__restrict__ T, long long nf, long long f) {
  FaceMetric<R> m;
  m.alpha = R(__ldg(&T[FF_ALPHA * nf + f]));
  m.beta_n = R(__ldg(&T[FF_BETA_N * nf + f]));
  m.g11 = R(__ldg(&T[FF_G11 * nf + f])); m.g12 = R(__ldg(&T[FF_G12 * nf + f])); m.g13 = R(__ldg(&T[FF_G13 * nf + f]));
  m.g22 = R(__ldg(&T[FF_G22 * nf + f])); m.g23 = R(__ldg(&T[FF_G23 * nf + f])); m.g33 = R(__ldg(&T[FF_G33 * nf + f]));
  m.sqg = R(__ldg(&T[FF_SQG * nf + f]));
  m.gup = R(__ldg(&T[FF_GUP * nf + f]));
  return m;
}
template <class R, class TT>
__device__ __forceinline__ FaceFrame<R> load_face_frame(const TT *__restrict__ T, long long nf, long long f) {
  FaceFrame<R> fr;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) fr.cof[a][i] = R(__ldg(&T[(FF_COF + 3 * a + i) * nf + f]));
  fr.gup = R(__ldg(&T[FF_GUP * nf + f]));
  fr.ok = __ldg(&T[FF_FRAME_OK * nf + f]) != TT(0);
  return fr;
}

}  // namespace grhd
