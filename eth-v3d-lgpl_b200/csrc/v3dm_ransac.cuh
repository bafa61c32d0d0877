// v3dm_ransac.cuh -- definitions shared by the RANSAC kernels (v3dm_ransac.cu) and the refining
// selection kernel (v3dm_ransac_refine.cu, built without fused multiply-adds).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace v3dm {

constexpr int kRsMaxSol = 10;        // solutions per sample
constexpr int kRsSlotDoubles = 18;   // E, F
constexpr int kRsRound = 128;        // samples per pair per round

// The loop's state per pair, carried from round to round.
struct RsState {
  double minError;  // best cost so far (1e30: none)
  int budget;       // nSamples, lowered by each accepted candidate
  int drawn;        // samples consumed
  int chosen;       // sample of the accepted candidate, -1: none
  int done;         // the loop has ended for this pair
};

// ransacNSamples(5, outlierRatio, 1 - 1e-9) (reconstruction_common.h:627-635).
__device__ __forceinline__ int rs_budget(double outlierRatio) {
  const double maxN = 1e8;
  if (outlierRatio >= 1.0) return (int)maxN;
  double N = log(1.0 - (1.0 - 10e-10)) / log(1.0 - pow(1.0 - outlierRatio, 5));
  N = fmax(0.0, fmin(maxN, N));
  return (int)N;
}

// The round's selection with mode.iterativeRefinement (v3dm_ransac_refine.cu): one warp per pair.
cudaError_t launch_rs_select_refine(const int32_t* offsets, int nPairs, int nDraw, int s0, int len, const int8_t* counts,
                                    const uint8_t* slotOk, const double* cost, const double* slots, RsState* st,
                                    double* bestEF, const float4* corrs, const double4* norm, const int32_t* samples,
                                    const double* invK, double thr, double thr2, double* bestRT, cudaStream_t stream);

}  // namespace v3dm
