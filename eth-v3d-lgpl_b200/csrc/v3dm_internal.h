// v3dm_internal.h -- host-side structures shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/v3dm.h"
#include "v3dm_common.cuh"

namespace v3dm {

// Device error flags (bitwise OR into MatchArgs::err).
constexpr int kErrWaitTimeout = 1;  // a bounded mbarrier wait in the tcgen05 kernel gave up
constexpr int kErrNotU8 = 2;        // a float descriptor was not u/512-valued
constexpr int kErrTmem = 4;         // TMEM allocation returned an unexpected address

// Layout of the small info block every matching call writes (int32 words).
constexpr int kInfoPairs = 0;     // number of mutual pairs
constexpr int kInfoErr = 1;       // device error flags
constexpr int kInfoMaxSeg = 2;    // largest candidate count of one list segment
constexpr int kInfoWords = 4;

struct MatchArgs {
  int nL, nR;
  int32_t T;                       // candidate threshold
  unsigned long long* lBest;       // per left: best key over rights
  unsigned int* lSec;              // per left: second value + 1
  unsigned long long* rBest;       // per right: best key over lefts
  unsigned int* rSec;              // per right: second value + 1
  unsigned long long* cand;        // candidate list, nSeg segments of segCap entries
  int* segCount;                   // per segment: number of candidates found
  long long segCap;
  int nSeg;
  int* err;
  int nGates;
  GateParams gates[V3DM_MAX_GATES];
};

// Kernel launchers (v3dm_match.cu, v3dm_match_tc.cu).
cudaError_t launch_match_simt(const uint8_t* dL, const uint8_t* dR, const MatchArgs& a, cudaStream_t s);
cudaError_t launch_seconds(const MatchArgs& a, cudaStream_t s);
cudaError_t launch_finalize(const MatchArgs& a, float minScore, float minRatio, int32_t* dScratch, int32_t* dPairs,
                            int32_t* dInfo, cudaStream_t s);
cudaError_t launch_gate_precompute(int type, const double* m, const float* dLPos, int nL, const float* dRPos,
                                   int nR, float4* lv, float4* rv, cudaStream_t s);
cudaError_t launch_f32_to_u8(const float* src, uint8_t* dst, int n, int* err, cudaStream_t s);

// tcgen05 path: per-matcher prepared operand maps (opaque, v3dm_match_tc.cu).
struct TcPlan;
cudaError_t tc_plan_create(TcPlan** p, int device);
void tc_plan_destroy(TcPlan* p);
// Rebuilds the operand tensor maps when the buffers or counts change.
cudaError_t tc_plan_bind(TcPlan* p, const uint8_t* dL, int nL, const uint8_t* dR, int nR);
// Number of candidate-list segments the tcgen05 kernel uses (one per CTA).
int tc_segments(TcPlan* p);
cudaError_t launch_match_tc(TcPlan* p, const MatchArgs& a, cudaStream_t s, int* launches);

// Candidate threshold (v3dm_api.cu).
int host_candidate_threshold(float minScore, float minRatio, bool gated, int32_t* T);

}  // namespace v3dm
