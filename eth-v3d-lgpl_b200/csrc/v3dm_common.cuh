// v3dm_common.cuh -- definitions shared by the matching kernels and the host code.
//
// Fused selection.  The reference materialises the nL x nR FP32 score matrix
// (v3d_cudamatching.cu:529-530) and scans it twice: per left over rights
// (_cuda_computeColumnMaximaWithRatioTest, .cu:133-162) and per right over lefts
// (_cuda_computeRowMaximaWithRatioTest, .cu:164-210).  Here no score leaves the SM.  A
// per-call integer threshold T (host_candidate_threshold) is chosen so that
//   (1) T <= the smallest S that can pass the min-score test, and
//   (2) the decision of every side does not change when its second-best value is replaced
//       by any value below T (or by a masked -1e20f, or by "none", -1e30f).
// Scores S >= T that survive the guided gates are "candidates".  For every feature the
// kernels keep
//   best key   max over its candidates of (S + 1) << 17 | (kIndexMask - other index),
//              an atomicMax without a returned value; the largest key is the largest score
//              with the first index on ties, the reference's argMax rule (.cu:145);
//   second     max over its candidates that are not the best of S + 1, filled by a pass
//              over the candidate list once all best keys are known: the second largest
//              value of the multiset, the reference's nextVal (.cu:146).
// The final decision therefore equals the reference's scan over all scores.
#pragma once
#include <stdint.h>
#include <cstring>

#ifdef __CUDACC__
#define V3DM_HD __host__ __device__ __forceinline__
#else
#define V3DM_HD inline
#endif

namespace v3dm {

constexpr int kDescBytes = 128;
constexpr int32_t kMaxScore = 255 * 255 * 128;  // 8,323,200 < 2^23
constexpr int kIndexBits = 17;                  // feature index field: n <= 131072
constexpr uint32_t kIndexMask = (1u << kIndexBits) - 1u;
constexpr float kNone = -1e30f;    // initial maxVal / nextVal (v3d_cudamatching.cu:138-139)
constexpr float kMasked = -1e20f;  // gated score (v3d_cudamatching.cu:308, :340)

// Best key of a candidate with score S against the feature with index idx on the other
// side: larger key = larger score, then lower index.  0 means "no candidate".
V3DM_HD uint64_t best_key(int32_t S, int32_t idx) {
  return ((uint64_t)(uint32_t)(S + 1) << kIndexBits) | (uint64_t)(kIndexMask - (uint32_t)idx);
}

// Candidate list entry: left index, right index and score in one 64-bit word.
V3DM_HD uint64_t cand_pack(int32_t l, int32_t r, int32_t S) {
  return (uint64_t)(uint32_t)l | ((uint64_t)(uint32_t)r << kIndexBits) | ((uint64_t)(uint32_t)S << (2 * kIndexBits));
}
V3DM_HD void cand_unpack(uint64_t e, int32_t& l, int32_t& r, int32_t& S) {
  l = (int32_t)(e & kIndexMask);
  r = (int32_t)((e >> kIndexBits) & kIndexMask);
  S = (int32_t)(e >> (2 * kIndexBits));
}

V3DM_HD float score_of(int32_t S) { return (float)S * 0x1p-18f; }

// The reference's per-side decision (v3d_cudamatching.cu:150-161 and :199-209; the
// no-ratio kernels' test at .cu:48 and :84 when minRatio < 0), with IEEE round-to-nearest
// and no contraction:
//   bestDist = 2 - 2*s1;  nextDist = (float)max(0.001, (double)(2 - 2*s2));
//   accept   = s1 > minScore && bestDist / nextDist < minRatio.
V3DM_HD bool accept_scores(float s1, float s2, float minScore, float minRatio) {
  if (minRatio < 0.0f) return s1 > minScore;
#ifdef __CUDA_ARCH__
  float t = __fsub_rn(2.0f, __fmul_rn(2.0f, s2));
  float nextDist = (float)fmax(0.001, (double)t);
  float bestDist = __fsub_rn(2.0f, __fmul_rn(2.0f, s1));
  float ratio = __fdiv_rn(bestDist, nextDist);
#else
  // host code is compiled with -ffp-contract=off
  float t = 2.0f - 2.0f * s2;
  float nextDist = (float)(0.001 > (double)t ? 0.001 : (double)t);
  float bestDist = 2.0f - 2.0f * s1;
  float ratio = bestDist / nextDist;
#endif
  return s1 > minScore && ratio < minRatio;
}

// Decision of one feature: the accepted index or -1.  A missing second value is
// equivalent to any value below T by construction of T, so "none" (-1e30f) stands for it.
V3DM_HD int32_t decide(uint64_t bestKey, uint32_t secondP1, float minScore, float minRatio) {
  if (bestKey == 0) return -1;
  int32_t S1 = (int32_t)(bestKey >> kIndexBits) - 1;
  int32_t idx = (int32_t)(kIndexMask - (uint32_t)(bestKey & kIndexMask));
  float s2 = secondP1 ? score_of((int32_t)secondP1 - 1) : kNone;
  return accept_scores(score_of(S1), s2, minScore, minRatio) ? idx : -1;
}

// ---- float scores (BF16 hi/lo path) ------------------------------------------------------
// Order-preserving map of a float to a 32-bit key (larger float -> larger key, every real value
// -> key >= 1, so 0 can mean "none").
V3DM_HD uint32_t f32_order(float f) {
#ifdef __CUDA_ARCH__
  const uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  std::memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
V3DM_HD float f32_unorder(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}
// Best key of a float score: larger score, then lower index.
V3DM_HD uint64_t best_key_f(float s, int32_t idx) {
  return ((uint64_t)f32_order(s) << kIndexBits) | (uint64_t)(kIndexMask - (uint32_t)idx);
}
// Decision of one feature from a float best key and the ordered second score (0: none).
V3DM_HD int32_t decide_f(uint64_t bestKey, uint32_t secondOrd, float minScore, float minRatio) {
  if (bestKey == 0) return -1;
  const float s1 = f32_unorder((uint32_t)(bestKey >> kIndexBits));
  const int32_t idx = (int32_t)(kIndexMask - (uint32_t)(bestKey & kIndexMask));
  const float s2 = secondOrd ? f32_unorder(secondOrd) : kNone;
  return accept_scores(s1, s2, minScore, minRatio) ? idx : -1;
}

// Guided gate, one per guided call since the last putative call (the reference masks the
// stored score matrix in place, so gates compound).  Per-left and per-right terms are
// precomputed once per call with the reference's expressions; see gate_rejects.
struct GateParams {
  int type;        // 1 epipolar (F), 2 homography (H)
  float sqrThr;    // thr*thr in float (.cu:591, :662)
  const float4* lv;  // per left: epipolar (Fp.x, Fp.y, Fp.z, 0); homography (Hp.x/Hp.z, Hp.y/Hp.z, Hp.z, 0)
  const float4* rv;  // per right: epipolar (q.x, q.y, Ftq.x, Ftq.y); homography (q.x, q.y, 0, 0)
};

}  // namespace v3dm
