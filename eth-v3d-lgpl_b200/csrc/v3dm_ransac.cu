// v3dm_ransac.cu -- batched RANSAC for the essential matrix of many image pairs.
//
// The apps run computeRobustOrientationMLE(corrs, K1, K2, inlierThreshold, nSamples, ...)
// (V3D/Apps/SfM/reconstruction_common.cpp:139-340) on one pair at a time between putative and
// guided matching (match_sequence.cpp:260-268).  Per pair, that loop draws 5-correspondence
// samples, solves each for up to 10 essential matrices (computeEssentialsFromFiveCorrs), scores
// every candidate with the truncated Sampson cost sum_i min(d_i, thr^2) over all correspondences
// (sampsonEpipolarError of F = K2^-T E K1^-1), and keeps a candidate whose cost is strictly below
// the best so far and whose pose is consistent (relativePoseFromEssential on the sample); each
// accepted candidate lowers the sample budget to ransacNSamples(5, outlier fraction, 1 - 1e-9).
//
// Here all pairs and all samples run at once:
//   k_rs_normalize  correspondences normalised by K^-1 (the solver's input);
//   k_rs_draw       (optional) 5 distinct correspondences per sample from a counter-based hash;
// then rounds of 128 samples per pair (pairs whose loop has ended are skipped):
//   k_rs_hyp        one thread per sample: five-point solver, F, pose consistency -> slots;
//   k_rs_compact    one CTA per pair: the round's candidates in loop order, densely;
//   k_rs_score      a CTA per (pair, 128 candidates): the pair's correspondences staged in
//                   shared memory, one candidate per thread, cost and inlier count in double;
//   k_rs_select     one warp per pair: the round's candidates staged in shared memory, then the
//                   loop's sequential rule (strictly lower cost, pose consistent, adaptive sample
//                   budget) over them in loop order, its state carried to the next round;
// and at the end
//   k_rs_finish     pose, error and inlier flags of the chosen candidate.
// With the loop's iterative refinement (mode.iterativeRefinement, v3dm_ransac_set_refinement),
// k_rs_select refines each accepted pose as reconstruction_common.cpp:255-314 does: the pose of the
// accepted sample is refined by refineRelativePose (v3d_poseutilities.cpp:1063-1101: Levenberg-
// Marquardt on the weighted Sampson residuals of the candidate's inliers; ess::refine_pose restates
// it, here with its sums over the inliers split across the warp), the refined F is scored over all
// correspondences in the loop's order, and the loop keeps min(cost, refined cost), the refined
// model and the refined inlier count for its sample budget.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <new>
#include <numeric>
#include <vector>

#include "v3dm_essential.cuh"
#include "v3dm_internal.h"
#include "v3dm_ransac.cuh"

using namespace v3dm;

namespace {

constexpr int kRsScoreThreads = 128;
constexpr int kRsStage = 1024;       // correspondences staged at a time in k_rs_score

struct RsDeviceGuard {
  int prev = -1;
  explicit RsDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~RsDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

__device__ __forceinline__ int rs_pair_of(const int32_t* __restrict__ offsets, int nPairs, int c) {
  int lo = 0, hi = nPairs - 1;  // the pair p with offsets[p] <= c < offsets[p + 1]
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (offsets[mid] <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// (A [x y 1]^T) projected, summed as multiply_A_v_projective (v3d_linearbase.h:1031-1048):
// the last column first.
__device__ __forceinline__ void rs_project(const double* A, double x, double y, double& u, double& v) {
  using ess::dadd;
  using ess::dmul;
  const double w = dadd(dadd(A[8], dmul(A[6], x)), dmul(A[7], y));
  u = ess::ddiv(dadd(dadd(A[2], dmul(A[0], x)), dmul(A[1], y)), w);
  v = ess::ddiv(dadd(dadd(A[5], dmul(A[3], x)), dmul(A[4], y)), w);
}

// invK: per pair invK1 (9), invK2 (9), row-major.
__global__ void k_rs_normalize(const int32_t* __restrict__ offsets, int nPairs, int nCorrs,
                               const float4* __restrict__ corrs, const double* __restrict__ invK,
                               double4* __restrict__ norm) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nCorrs; c += gridDim.x * blockDim.x) {
    const int p = rs_pair_of(offsets, nPairs, c);
    const float4 k = corrs[c];
    double4 o;
    rs_project(invK + 18 * p, k.x, k.y, o.x, o.y);
    rs_project(invK + 18 * p + 9, k.z, k.w, o.z, o.w);
    norm[c] = o;
  }
}

__device__ __forceinline__ uint64_t rs_mix(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// 5 distinct indices in [0, n) per (pair, sample); pairs with n < 5 get -1.
__global__ void k_rs_draw(const int32_t* __restrict__ offsets, int nPairs, int nDraw, uint64_t seed,
                          int32_t* __restrict__ samples) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nPairs * nDraw) return;
  const int p = (int)(t / nDraw);
  const int n = offsets[p + 1] - offsets[p];
  int32_t* s = samples + t * 5;
  if (n < 5) {
    for (int k = 0; k < 5; ++k) s[k] = -1;
    return;
  }
  uint64_t state = rs_mix(seed ^ rs_mix((uint64_t)t));
  int got = 0;
  for (int tries = 0; got < 5 && tries < 64; ++tries) {
    state = rs_mix(state);
    const int cand = (int)((state >> 11) % (uint64_t)n);
    bool dup = false;
    for (int k = 0; k < got; ++k) dup |= s[k] == cand;
    if (!dup) s[got++] = cand;
  }
  for (int k = got; k < 5; ++k) s[k] = (s[k - 1] + 1) % n;  // unreachable in practice (n >= 5)
}

__global__ void k_rs_init(const int32_t* __restrict__ offsets, int nPairs, int nSamples, RsState* __restrict__ st) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nPairs) return;
  RsState s;
  s.minError = 1e30;
  s.budget = nSamples;
  s.drawn = 0;
  s.chosen = -1;
  s.done = offsets[p + 1] - offsets[p] < 5;
  st[p] = s;
}

// One thread per (pair, sample of this round): candidates into the round's slots (pair, j, r),
// their count and pose flag.  Pairs whose loop has ended are skipped.
__global__ void __launch_bounds__(64)
k_rs_hyp(const int32_t* __restrict__ offsets, int nPairs, int nDraw, int s0, int len,
         const int32_t* __restrict__ samples, const double4* __restrict__ norm, const double* __restrict__ invK,
         const RsState* __restrict__ st, double* __restrict__ slots, uint8_t* __restrict__ slotOk,
         int8_t* __restrict__ counts) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // p * kRsRound + j
  const int p = (int)(t / kRsRound), j = (int)(t % kRsRound);
  if (p >= nPairs) return;
  if (j >= len || st[p].done) {
    counts[t] = 0;
    return;
  }
  const int b = offsets[p], n = offsets[p + 1] - b;
  const int32_t* s = samples + ((long long)p * nDraw + s0 + j) * 5;
  bool valid = n >= 5;
  for (int k = 0; k < 5 && valid; ++k) valid = s[k] >= 0 && s[k] < n;
  if (!valid) {
    counts[t] = 0;
    return;
  }
  double x1[5], y1[5], x2[5], y2[5];
  for (int k = 0; k < 5; ++k) {
    const double4 o = norm[b + s[k]];
    x1[k] = o.x;
    y1[k] = o.y;
    x2[k] = o.z;
    y2[k] = o.w;
  }
  double Es[kRsMaxSol][9];
  const int ns = ess::five_point(x1, y1, x2, y2, Es);
  const double* iK1 = invK + 18 * p;
  const double* iK2 = invK + 18 * p + 9;
  double iK2t[9];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c) iK2t[3 * a + c] = iK2[3 * c + a];
  for (int r = 0; r < ns; ++r) {
    double* slot = slots + (t * kRsMaxSol + r) * kRsSlotDoubles;
    double tmp[9], F[9], R[9], T[3];
    ess::mat3_mul(iK2t, Es[r], tmp);  // F = K2^-T E K1^-1
    ess::mat3_mul(tmp, iK1, F);
    for (int k = 0; k < 9; ++k) {
      slot[k] = Es[r][k];
      slot[9 + k] = F[k];
    }
    slotOk[t * kRsMaxSol + r] = ess::essential_pose(Es[r], 5, x1, y1, x2, y2, R, T) ? 1 : 0;
  }
  counts[t] = (int8_t)ns;
}

// Diagnostic: the five-point solutions of n samples (x1[5] y1[5] x2[5] y2[5] per sample).
__global__ void k_rs_five_point(int n, const double* __restrict__ pts, double* __restrict__ Es,
                                int32_t* __restrict__ counts) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double* q = pts + 20 * t;
  double E[kRsMaxSol][9];
  const int ns = ess::five_point(q, q + 5, q + 10, q + 15, E);
  for (int r = 0; r < ns; ++r)
    for (int k = 0; k < 9; ++k) Es[(size_t)t * 90 + 9 * r + k] = E[r][k];
  counts[t] = ns;
}

// One CTA per pair: the round's candidate slots (j * 10 + r) in loop order; work counters.
__global__ void k_rs_compact(const int32_t* __restrict__ offsets, const int8_t* __restrict__ counts,
                             int32_t* __restrict__ list, int32_t* __restrict__ listN,
                             unsigned long long* __restrict__ work) {
  static_assert(kRsRound <= 1024, "one thread per sample of the round");
  const int p = blockIdx.x;
  __shared__ int warpSum[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int j = threadIdx.x;
  const int c = j < kRsRound ? counts[(long long)p * kRsRound + j] : 0;
  int inc = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) warpSum[wid] = inc;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < wid; ++w) before += warpSum[w];
  int32_t* out = list + (long long)p * kRsRound * kRsMaxSol;
  for (int r = 0; r < c; ++r) out[before + inc - c + r] = j * kRsMaxSol + r;
  if (threadIdx.x == 0) {
    int total = 0;
    for (int w = 0; w < nw; ++w) total += warpSum[w];
    listN[p] = total;
    if (total) {
      atomicAdd(&work[0], (unsigned long long)total);
      atomicAdd(&work[1], (unsigned long long)total * (unsigned long long)(offsets[p + 1] - offsets[p]));
    }
  }
}

// CTA (pair, chunk): cost = sum_i min(d_i, thr2) and the count of d_i < thr2 for 128 candidates.
__global__ void __launch_bounds__(kRsScoreThreads)
k_rs_score(const int32_t* __restrict__ offsets, const float4* __restrict__ corrs, const int32_t* __restrict__ list,
           const int32_t* __restrict__ listN, const double* __restrict__ slots, double thr2,
           double* __restrict__ cost, int32_t* __restrict__ inl) {
  const int p = blockIdx.x;
  const int h = blockIdx.y * kRsScoreThreads + threadIdx.x;
  const int H = listN[p];
  if (blockIdx.y * kRsScoreThreads >= H) return;  // uniform over the CTA
  __shared__ double4 st[kRsStage];  // the positions converted once per CTA
  const int b = offsets[p], n = offsets[p + 1] - b;
  const bool mine = h < H;
  long long slot = 0;
  double F[9];
  if (mine) {
    slot = (long long)p * kRsRound * kRsMaxSol + list[(long long)p * kRsRound * kRsMaxSol + h];
    for (int k = 0; k < 9; ++k) F[k] = slots[slot * kRsSlotDoubles + 9 + k];
  }
  double sum = 0.0;
  int cnt = 0;
  for (int c0 = 0; c0 < n; c0 += kRsStage) {
    const int m = min(kRsStage, n - c0);
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const float4 c = corrs[b + c0 + k];
      st[k] = make_double4(c.x, c.y, c.z, c.w);
    }
    __syncthreads();
    if (mine)
      for (int k = 0; k < m; ++k) {
        const double4 c = st[k];
        bool in;
        sum = ess::dadd(sum, ess::sampson_truncated(F, c.x, c.y, c.z, c.w, thr2, in));
        cnt += in;
      }
  }
  if (mine) {
    cost[slot] = sum;
    inl[slot] = cnt;
  }
}

// One warp per pair: the round's costs, pose flags and inlier counts staged in shared memory by
// the warp (coalesced), then lane 0 walks the loop over the round's samples in order (the rule of
// reconstruction_common.cpp:177-335 without refinement); the last accepted candidate's E and F are
// kept (the warp copies them).  With refinement the selection is k_rs_select_refine
// (v3dm_ransac_refine.cu).
__global__ void __launch_bounds__(32)
k_rs_select(const int32_t* __restrict__ offsets, int nPairs, int nDraw, int s0, int len,
            const int8_t* __restrict__ counts, const uint8_t* __restrict__ slotOk, const double* __restrict__ cost,
            const int32_t* __restrict__ inl, const double* __restrict__ slots, RsState* __restrict__ st,
            double* __restrict__ bestEF) {
  const int p = blockIdx.x;
  const int lane = threadIdx.x;
  __shared__ double sCost[kRsRound * kRsMaxSol];
  __shared__ int32_t sInl[kRsRound * kRsMaxSol];
  __shared__ uint8_t sOk[kRsRound * kRsMaxSol];
  __shared__ int8_t sCnt[kRsRound];
  __shared__ int sAccepted;
  RsState s = st[p];
  if (s.done) return;  // uniform over the warp
  const long long base = (long long)p * kRsRound;
  for (int j = lane; j < len; j += 32) sCnt[j] = counts[base + j];
  __syncwarp();
  for (int idx = lane; idx < len * kRsMaxSol; idx += 32) {
    const int j = idx / kRsMaxSol, r = idx - j * kRsMaxSol;
    if (r < sCnt[j]) {
      sCost[idx] = cost[base * kRsMaxSol + idx];
      sInl[idx] = inl[base * kRsMaxSol + idx];
      sOk[idx] = slotOk[base * kRsMaxSol + idx];
    }
  }
  __syncwarp();
  if (lane == 0) {
    const int n = offsets[p + 1] - offsets[p];
    int accepted = -1;
    for (int j = 0; j < len; ++j) {
      if (s.drawn > s.budget) break;
      ++s.drawn;
      const int ns = sCnt[j];
      for (int r = 0; r < ns; ++r) {
        const int idx = j * kRsMaxSol + r;
        if (!(sCost[idx] < s.minError)) continue;
        if (!sOk[idx]) continue;
        s.minError = sCost[idx];
        s.chosen = s0 + j;
        accepted = idx;
        const float frac = (float)(sInl[idx] - 5) / (float)(n - 5);
        s.budget = min(s.budget, rs_budget(1.0 - (double)frac));
      }
    }
    if (s.drawn > s.budget || s0 + len >= nDraw) s.done = 1;  // the next sample would end the loop
    st[p] = s;
    sAccepted = accepted;
  }
  __syncwarp();
  const int accepted = sAccepted;
  if (accepted >= 0 && lane < kRsSlotDoubles)
    bestEF[(size_t)p * kRsSlotDoubles + lane] = slots[(base * kRsMaxSol + accepted) * kRsSlotDoubles + lane];
}

// One thread per pair: E, F, R, T and error of the choice.
__global__ void k_rs_finish(const int32_t* __restrict__ offsets, int nPairs, int nDraw,
                            const int32_t* __restrict__ samples, const double4* __restrict__ norm,
                            const RsState* __restrict__ st, const double* __restrict__ bestEF,
                            double* __restrict__ out, int refine, const double* __restrict__ bestRT) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nPairs) return;
  double* o = out + (size_t)p * 31;  // E 9, F 9, R 9, T 3, error 1
  const RsState s = st[p];
  if (s.chosen < 0) {
    for (int k = 0; k < 30; ++k) o[k] = 0.0;
    o[30] = -1.0;
    return;
  }
  const int b = offsets[p], n = offsets[p + 1] - b;
  const int32_t* smp = samples + ((long long)p * nDraw + s.chosen) * 5;
  double x1[5], y1[5], x2[5], y2[5];
  for (int k = 0; k < 5; ++k) {
    const double4 v = norm[b + smp[k]];
    x1[k] = v.x;
    y1[k] = v.y;
    x2[k] = v.z;
    y2[k] = v.w;
  }
  const double* ef = bestEF + (size_t)p * kRsSlotDoubles;
  for (int k = 0; k < 18; ++k) o[k] = ef[k];
  if (refine) {  // the refined pose (reconstruction_common.cpp:321-322)
    for (int k = 0; k < 12; ++k) o[18 + k] = bestRT[(size_t)p * 12 + k];
  } else {
    ess::essential_pose(ef, 5, x1, y1, x2, y2, o + 18, o + 27);
  }
  o[30] = s.minError / n;
}

// nIn = -1 for the pairs without a model.
__global__ void k_rs_nomodel(int nPairs, const double* __restrict__ out, int32_t* __restrict__ nIn) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nPairs && out[(size_t)p * 31 + 30] < 0.0) nIn[p] = -1;
}

// Inlier flags (Sampson distance of the chosen F below thr2) and counts.
__global__ void k_rs_inliers(const int32_t* __restrict__ offsets, int nPairs, int nCorrs,
                             const float4* __restrict__ corrs, const double* __restrict__ out, double thr2,
                             uint8_t* __restrict__ flags, int32_t* __restrict__ nIn) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nCorrs; c += gridDim.x * blockDim.x) {
    const int p = rs_pair_of(offsets, nPairs, c);
    const double* o = out + (size_t)p * 31;
    uint8_t f = 0;
    if (o[30] >= 0.0) {
      const float4 k = corrs[c];
      f = ess::sampson(o + 9, k.x, k.y, k.z, k.w) < thr2;
    }
    flags[c] = f;
    if (f) atomicAdd(&nIn[p], 1);
  }
}

bool rs_invert3(const double* A, double* inv) {
  const double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
  const double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
  if (!(det != 0.0) || !std::isfinite(det)) return false;
  const double id = 1.0 / det;
  inv[0] = c00 * id;
  inv[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  inv[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  inv[3] = c01 * id;
  inv[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  inv[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  inv[6] = c02 * id;
  inv[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  inv[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return true;
}

template <class T>
cudaError_t rs_grow(T*& p, size_t& cap, size_t n) {
  if (n <= cap) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) cap = n;
  return e;
}

#define V3DM_RS_TRY(expr)                               \
  do {                                                  \
    cudaError_t e_ = (expr);                            \
    if (e_ != cudaSuccess) {                            \
      record_cuda_error(e_, __FILE__, __LINE__, #expr); \
      return V3DM_ERR_CUDA;                             \
    }                                                   \
  } while (0)

}  // namespace

struct v3dm_ransac {
  int device = 0;
  cudaStream_t stream = nullptr;
  int32_t* dOffsets = nullptr;
  size_t offCap = 0;
  float4* dCorrs = nullptr;
  size_t corrCap = 0;
  double4* dNorm = nullptr;
  size_t normCap = 0;
  double* dInvK = nullptr;
  size_t invKCap = 0;
  int32_t* dSamples = nullptr;
  size_t sampleCap = 0;
  double* dSlots = nullptr;
  size_t slotCap = 0;
  uint8_t* dSlotOk = nullptr;
  size_t okCap = 0;
  int8_t* dCounts = nullptr;
  size_t countCap = 0;
  int32_t* dList = nullptr;
  size_t listCap = 0;
  int32_t* dListN = nullptr;
  size_t listNCap = 0;
  double* dCost = nullptr;
  size_t costCap = 0;
  int32_t* dInl = nullptr;
  size_t inlCap = 0;
  void* dState = nullptr;  // RsState per pair
  size_t stateCap = 0;
  double* dBestEF = nullptr;
  size_t bestEFCap = 0;
  double* dBestRT = nullptr;   // refined R, T per pair (iterative refinement)
  size_t bestRTCap = 0;
  bool refine = false;         // RobustOrientationMode::iterativeRefinement
  double thr = 0.0;            // inlier threshold of the call (pixels)
  unsigned long long* dWork = nullptr;  // candidates, Sampson evaluations of the last call
  size_t workCap = 0;
  double* dOut = nullptr;
  size_t outCap = 0;
  uint8_t* dFlags = nullptr;
  size_t flagCap = 0;
  int32_t* dNIn = nullptr;
  size_t nInCap = 0;
  int lastLaunches = 0;
  std::vector<int32_t> hOffsets;  // the last call's offsets
  // CUDA-event timing of k_rs_hyp (0) and k_rs_score (1): pending event pairs
  bool profile = false;
  std::vector<cudaEvent_t> prof[2];
  double profMs[2] = {0.0, 0.0};
  int profLaunches[2] = {0, 0};
};

namespace {

cudaError_t rs_mark(v3dm_ransac* r, int k) {
  if (!r->profile) return cudaSuccess;
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreate(&ev);
  if (e != cudaSuccess) return e;
  r->prof[k].push_back(ev);
  return cudaEventRecord(ev, r->stream);
}

// Everything from normalisation to inlier flags, on r's stream; inputs already on the device.
int rs_enqueue(v3dm_ransac* r, int nPairs, int nCorrs, int nDraw, int nSamples, bool draw, uint64_t seed,
               double thr2, const float4* dCorrs, int32_t* dSamples, double* dOut, int32_t* dNIn, uint8_t* dFlags) {
  const size_t nR = (size_t)nPairs * kRsRound;  // sample slots of one round
  V3DM_RS_TRY(rs_grow(r->dNorm, r->normCap, (size_t)nCorrs));
  V3DM_RS_TRY(rs_grow(r->dSlots, r->slotCap, nR * kRsMaxSol * kRsSlotDoubles));
  V3DM_RS_TRY(rs_grow(r->dSlotOk, r->okCap, nR * kRsMaxSol));
  V3DM_RS_TRY(rs_grow(r->dCounts, r->countCap, nR));
  V3DM_RS_TRY(rs_grow(r->dList, r->listCap, nR * kRsMaxSol));
  V3DM_RS_TRY(rs_grow(r->dListN, r->listNCap, (size_t)nPairs));
  V3DM_RS_TRY(rs_grow(r->dCost, r->costCap, nR * kRsMaxSol));
  V3DM_RS_TRY(rs_grow(r->dInl, r->inlCap, nR * kRsMaxSol));
  {
    char* st = static_cast<char*>(r->dState);
    V3DM_RS_TRY(rs_grow(st, r->stateCap, (size_t)nPairs * sizeof(RsState)));
    r->dState = st;
  }
  V3DM_RS_TRY(rs_grow(r->dBestEF, r->bestEFCap, (size_t)nPairs * kRsSlotDoubles));
  V3DM_RS_TRY(rs_grow(r->dBestRT, r->bestRTCap, (size_t)nPairs * 12));
  V3DM_RS_TRY(rs_grow(r->dWork, r->workCap, (size_t)2));
  RsState* state = static_cast<RsState*>(r->dState);
  int launches = 0;
  V3DM_RS_TRY(cudaMemsetAsync(r->dWork, 0, 2 * sizeof(unsigned long long), r->stream));
  if (nCorrs > 0) {
    k_rs_normalize<<<std::min((nCorrs + 255) / 256, 148 * 16), 256, 0, r->stream>>>(r->dOffsets, nPairs, nCorrs,
                                                                                  dCorrs, r->dInvK, r->dNorm);
    ++launches;
  }
  const size_t nT = (size_t)nPairs * nDraw;
  if (draw) {
    k_rs_draw<<<(unsigned)((nT + 255) / 256), 256, 0, r->stream>>>(r->dOffsets, nPairs, nDraw, seed, dSamples);
    ++launches;
  }
  k_rs_init<<<(nPairs + 127) / 128, 128, 0, r->stream>>>(r->dOffsets, nPairs, nSamples, state);
  ++launches;
  // rounds of kRsRound samples per pair; pairs whose loop has ended are skipped
  for (int s0 = 0; s0 < nDraw; s0 += kRsRound) {
    const int len = std::min(kRsRound, nDraw - s0);
    V3DM_RS_TRY(rs_mark(r, 0));
    k_rs_hyp<<<(unsigned)((nR + 63) / 64), 64, 0, r->stream>>>(r->dOffsets, nPairs, nDraw, s0, len, dSamples,
                                                                r->dNorm, r->dInvK, state, r->dSlots, r->dSlotOk,
                                                                r->dCounts);
    V3DM_RS_TRY(rs_mark(r, 0));
    k_rs_compact<<<nPairs, kRsRound, 0, r->stream>>>(r->dOffsets, r->dCounts, r->dList, r->dListN, r->dWork);
    const unsigned chunks = (unsigned)((kRsRound * kRsMaxSol + kRsScoreThreads - 1) / kRsScoreThreads);
    V3DM_RS_TRY(rs_mark(r, 1));
    k_rs_score<<<dim3(nPairs, chunks), kRsScoreThreads, 0, r->stream>>>(r->dOffsets, dCorrs, r->dList, r->dListN,
                                                                       r->dSlots, thr2, r->dCost, r->dInl);
    V3DM_RS_TRY(rs_mark(r, 1));
    if (r->refine)
      V3DM_RS_TRY(launch_rs_select_refine(r->dOffsets, nPairs, nDraw, s0, len, r->dCounts, r->dSlotOk, r->dCost,
                                          r->dSlots, state, r->dBestEF, dCorrs, r->dNorm, dSamples, r->dInvK, r->thr,
                                          thr2, r->dBestRT, r->stream));
    else
      k_rs_select<<<nPairs, 32, 0, r->stream>>>(r->dOffsets, nPairs, nDraw, s0, len, r->dCounts, r->dSlotOk,
                                                 r->dCost, r->dInl, r->dSlots, state, r->dBestEF);
    launches += 4;
  }
  k_rs_finish<<<(nPairs + 127) / 128, 128, 0, r->stream>>>(r->dOffsets, nPairs, nDraw, dSamples, r->dNorm, state,
                                                           r->dBestEF, dOut, r->refine ? 1 : 0, r->dBestRT);
  V3DM_RS_TRY(cudaMemsetAsync(dNIn, 0, (size_t)nPairs * sizeof(int32_t), r->stream));
  launches += 1;
  if (nCorrs > 0) {
    k_rs_inliers<<<std::min((nCorrs + 255) / 256, 148 * 16), 256, 0, r->stream>>>(
        r->dOffsets, nPairs, nCorrs, dCorrs, dOut, thr2, dFlags, dNIn);
    ++launches;
  }
  k_rs_nomodel<<<(nPairs + 127) / 128, 128, 0, r->stream>>>(nPairs, dOut, dNIn);
  ++launches;
  V3DM_RS_TRY(cudaGetLastError());
  r->lastLaunches = launches;
  return V3DM_OK;
}

}  // namespace

extern "C" {

int v3dm_ransac_create(v3dm_ransac** out, int device) {
  if (!out) return V3DM_ERR_ARG;
  *out = nullptr;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return V3DM_ERR_CUDA;
  if (prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_ransac* r = new (std::nothrow) v3dm_ransac();
  if (!r) return V3DM_ERR_ARG;
  r->device = device;
  RsDeviceGuard g(device);
  if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete r;
    return V3DM_ERR_CUDA;
  }
  *out = r;
  return V3DM_OK;
}

int v3dm_ransac_destroy(v3dm_ransac* r) {
  if (!r) return V3DM_OK;
  RsDeviceGuard g(r->device);
  cudaStreamSynchronize(r->stream);
  void* bufs[] = {r->dOffsets, r->dCorrs, r->dNorm, r->dInvK, r->dSamples, r->dSlots, r->dSlotOk, r->dCounts,
                  r->dList,    r->dListN, r->dCost, r->dInl,  r->dState,   r->dBestEF, r->dWork,  r->dOut,
                  r->dFlags,   r->dNIn,   r->dBestRT};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (int k = 0; k < 2; ++k)
    for (cudaEvent_t ev : r->prof[k]) cudaEventDestroy(ev);
  cudaStreamDestroy(r->stream);
  delete r;
  return V3DM_OK;
}

int v3dm_ransac_stream(v3dm_ransac* r, void** stream) {
  if (!r || !stream) return V3DM_ERR_ARG;
  *stream = r->stream;
  return V3DM_OK;
}

int v3dm_ransac_last_launches(v3dm_ransac* r, int* n) {
  if (!r || !n) return V3DM_ERR_ARG;
  *n = r->lastLaunches;
  return V3DM_OK;
}

static int rs_check(int nPairs, const int32_t* offsets, const double* K, double inlierThreshold, int nSamples,
                    int nDraw) {
  if (nPairs < 0 || (nPairs > 0 && (!offsets || !K)) || nSamples < 0 || nDraw < 1 || nDraw > V3DM_RANSAC_MAX_DRAW ||
      !(inlierThreshold >= 0.0))
    return V3DM_ERR_ARG;
  if (nPairs == 0) return V3DM_OK;
  if (offsets[0] != 0) return V3DM_ERR_ARG;
  for (int p = 0; p < nPairs; ++p)
    if (offsets[p + 1] < offsets[p]) return V3DM_ERR_ARG;
  if ((size_t)nPairs * (size_t)nDraw > (size_t)V3DM_RANSAC_MAX_SAMPLES) return V3DM_ERR_SIZE;
  if (nPairs > V3DM_RANSAC_MAX_PAIRS) return V3DM_ERR_SIZE;  // a round's buffers: ~184 KB per pair
  return V3DM_OK;
}

// Offsets and K^-1 to the device and every buffer sized; r's stream is idle on entry.
static int rs_stage(v3dm_ransac* r, int nPairs, const int32_t* offsets, const double* K, int nDraw) {
  std::vector<double> invK((size_t)nPairs * 18);
  for (int p = 0; p < nPairs; ++p)
    if (!rs_invert3(K + 18 * p, invK.data() + 18 * p) || !rs_invert3(K + 18 * p + 9, invK.data() + 18 * p + 9))
      return V3DM_ERR_ARG;
  const int nCorrs = offsets[nPairs];
  r->hOffsets.assign(offsets, offsets + nPairs + 1);
  V3DM_RS_TRY(rs_grow(r->dOffsets, r->offCap, (size_t)nPairs + 1));
  V3DM_RS_TRY(rs_grow(r->dInvK, r->invKCap, (size_t)nPairs * 18));
  V3DM_RS_TRY(rs_grow(r->dSamples, r->sampleCap, (size_t)nPairs * nDraw * 5));
  V3DM_RS_TRY(rs_grow(r->dOut, r->outCap, (size_t)nPairs * 31));
  V3DM_RS_TRY(rs_grow(r->dFlags, r->flagCap, (size_t)nCorrs));
  V3DM_RS_TRY(rs_grow(r->dNIn, r->nInCap, (size_t)nPairs));
  V3DM_RS_TRY(cudaMemcpyAsync(r->dOffsets, offsets, ((size_t)nPairs + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                              r->stream));
  V3DM_RS_TRY(cudaMemcpyAsync(r->dInvK, invK.data(), invK.size() * sizeof(double), cudaMemcpyHostToDevice, r->stream));
  // the copies above read pageable host memory that is freed on return
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  return V3DM_OK;
}

int v3dm_ransac_essential(v3dm_ransac* r, int nPairs, const int32_t* offsets, const float* corrs, const double* K,
                          double inlierThreshold, int nSamples, int nDraw, const int32_t* samples, uint64_t seed,
                          double* models, int32_t* nInliers, uint8_t* inlierFlags) {
  if (!r) return V3DM_ERR_ARG;
  int st = rs_check(nPairs, offsets, K, inlierThreshold, nSamples, nDraw);
  if (st != V3DM_OK || nPairs == 0) return st;
  if (!models || !nInliers) return V3DM_ERR_ARG;
  const int nCorrs = offsets[nPairs];
  if (nCorrs > 0 && !corrs) return V3DM_ERR_ARG;
  if (samples)
    for (size_t k = 0; k < (size_t)nPairs * nDraw * 5; ++k) {
      const int p = (int)(k / ((size_t)nDraw * 5));
      if (samples[k] < 0 || samples[k] >= offsets[p + 1] - offsets[p]) return V3DM_ERR_ARG;
    }
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  st = rs_stage(r, nPairs, offsets, K, nDraw);
  if (st != V3DM_OK) return st;
  V3DM_RS_TRY(rs_grow(r->dCorrs, r->corrCap, (size_t)nCorrs));
  if (nCorrs > 0)
    V3DM_RS_TRY(cudaMemcpyAsync(r->dCorrs, corrs, (size_t)nCorrs * sizeof(float4), cudaMemcpyHostToDevice, r->stream));
  if (samples)
    V3DM_RS_TRY(cudaMemcpyAsync(r->dSamples, samples, (size_t)nPairs * nDraw * 5 * sizeof(int32_t),
                                cudaMemcpyHostToDevice, r->stream));
  r->thr = inlierThreshold;
  st = rs_enqueue(r, nPairs, nCorrs, nDraw, nSamples, samples == nullptr, seed, inlierThreshold * inlierThreshold,
                  r->dCorrs, r->dSamples, r->dOut, r->dNIn, r->dFlags);
  if (st != V3DM_OK) return st;
  V3DM_RS_TRY(cudaMemcpyAsync(models, r->dOut, (size_t)nPairs * 31 * sizeof(double), cudaMemcpyDeviceToHost,
                              r->stream));
  V3DM_RS_TRY(cudaMemcpyAsync(nInliers, r->dNIn, (size_t)nPairs * sizeof(int32_t), cudaMemcpyDeviceToHost, r->stream));
  if (inlierFlags && nCorrs > 0)
    V3DM_RS_TRY(cudaMemcpyAsync(inlierFlags, r->dFlags, (size_t)nCorrs, cudaMemcpyDeviceToHost, r->stream));
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  return V3DM_OK;
}

int v3dm_ransac_essential_device(v3dm_ransac* r, int nPairs, const int32_t* offsets, const float* d_corrs,
                                 const double* K, double inlierThreshold, int nSamples, int nDraw,
                                 const int32_t* d_samples, uint64_t seed, double* d_models, int32_t* d_nInliers,
                                 uint8_t* d_inlierFlags) {
  if (!r) return V3DM_ERR_ARG;
  int st = rs_check(nPairs, offsets, K, inlierThreshold, nSamples, nDraw);
  if (st != V3DM_OK || nPairs == 0) return st;
  const int nCorrs = offsets[nPairs];
  if ((nCorrs > 0 && (!d_corrs || !d_inlierFlags)) || !d_models || !d_nInliers ||
      (reinterpret_cast<uintptr_t>(d_corrs) & 15))
    return V3DM_ERR_ARG;
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  st = rs_stage(r, nPairs, offsets, K, nDraw);
  if (st != V3DM_OK) return st;
  int32_t* dS = d_samples ? const_cast<int32_t*>(d_samples) : r->dSamples;
  r->thr = inlierThreshold;
  return rs_enqueue(r, nPairs, nCorrs, nDraw, nSamples, d_samples == nullptr, seed, inlierThreshold * inlierThreshold,
                    reinterpret_cast<const float4*>(d_corrs), dS, d_models, d_nInliers, d_inlierFlags);
}

int v3dm_ransac_set_refinement(v3dm_ransac* r, int enable) {
  if (!r) return V3DM_ERR_ARG;
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  r->refine = enable != 0;
  return V3DM_OK;
}

int v3dm_ransac_candidates(v3dm_ransac* r, long long* nCandidates, long long* nEvaluations) {
  if (!r || !nCandidates || !nEvaluations) return V3DM_ERR_ARG;
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  unsigned long long w[2] = {0, 0};
  if (r->dWork) V3DM_RS_TRY(cudaMemcpy(w, r->dWork, sizeof(w), cudaMemcpyDeviceToHost));
  *nCandidates = (long long)w[0];
  *nEvaluations = (long long)w[1];
  return V3DM_OK;
}

int v3dm_ransac_profile(v3dm_ransac* r, int enable) {
  if (!r) return V3DM_ERR_ARG;
  r->profile = enable != 0;
  return V3DM_OK;
}

int v3dm_ransac_profile_read(v3dm_ransac* r, int kernel, double* msTotal, int* launches) {
  if (!r || kernel < 0 || kernel > 1 || !msTotal || !launches) return V3DM_ERR_ARG;
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  for (int k = 0; k < 2; ++k) {
    std::vector<cudaEvent_t>& v = r->prof[k];
    for (size_t a = 0; a + 1 < v.size(); a += 2) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, v[a], v[a + 1]) == cudaSuccess) r->profMs[k] += ms;
      ++r->profLaunches[k];
    }
    for (cudaEvent_t ev : v) cudaEventDestroy(ev);
    v.clear();
  }
  *msTotal = r->profMs[kernel];
  *launches = r->profLaunches[kernel];
  r->profMs[kernel] = 0.0;
  r->profLaunches[kernel] = 0;
  return V3DM_OK;
}

int v3dm_ransac_wait(v3dm_ransac* r) {
  if (!r) return V3DM_ERR_ARG;
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  return V3DM_OK;
}

int v3dm_essential_five_point(v3dm_ransac* r, int n, const double* pts, double* Es, int32_t* counts) {
  if (!r || n < 0 || (n > 0 && (!pts || !Es || !counts)) || n > V3DM_RANSAC_MAX_SAMPLES) return V3DM_ERR_ARG;
  if (n == 0) return V3DM_OK;
  RsDeviceGuard g(r->device);
  V3DM_RS_TRY(cudaStreamSynchronize(r->stream));
  double* dPts = nullptr;
  double* dEs = nullptr;
  int32_t* dCnt = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&dPts), (size_t)n * 20 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&dEs), (size_t)n * 90 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&dCnt), (size_t)n * sizeof(int32_t));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dPts, pts, (size_t)n * 20 * sizeof(double), cudaMemcpyHostToDevice, r->stream);
  if (e == cudaSuccess) {
    k_rs_five_point<<<(n + 63) / 64, 64, 0, r->stream>>>(n, dPts, dEs, dCnt);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(Es, dEs, (size_t)n * 90 * sizeof(double), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(counts, dCnt, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, r->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
  cudaFree(dPts);
  cudaFree(dEs);
  cudaFree(dCnt);
  if (e != cudaSuccess) {
    record_cuda_error(e, __FILE__, __LINE__, "v3dm_essential_five_point");
    return V3DM_ERR_CUDA;
  }
  return V3DM_OK;
}

int v3dm_ransac_shuffle_samples(int N, int nSamples, unsigned seed, int cap, int32_t* samples, int* nDraw) {
  if (N < 0 || nSamples < 0 || cap < 0 || (cap > 0 && !samples) || !nDraw) return V3DM_ERR_ARG;
  *nDraw = 0;
  if (N < 5) return V3DM_OK;
  // getShuffleCount (reconstruction_common.cpp:110-114)
  const int nShuffles = std::max(1, (int)((float)nSamples * (float)5 / (float)N + 0.5));
  std::vector<int32_t> idx((size_t)N);
  std::iota(idx.begin(), idx.end(), 0);
  srand(seed);
  int drawn = 0;
  for (int s = 0; s < nShuffles && drawn <= nSamples; ++s) {
    // random_shuffle over rand(): element i swaps with element rand() % (i + 1)
    for (int i = 1; i < N; ++i) {
      const int j = rand() % (i + 1);
      if (i != j) std::swap(idx[(size_t)i], idx[(size_t)j]);
    }
    for (int j = 0; j < N - 5 && drawn <= nSamples; j += 5) {
      if (drawn < cap)
        for (int k = 0; k < 5; ++k) samples[(size_t)drawn * 5 + k] = idx[(size_t)j + k];
      ++drawn;
    }
  }
  *nDraw = std::min(drawn, cap);
  return drawn > cap ? V3DM_ERR_CAPACITY : V3DM_OK;
}

}  // extern "C"
