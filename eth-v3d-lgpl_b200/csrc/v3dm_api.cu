// v3dm_api.cu -- host side of the C ABI (include/v3dm.h) for the matcher.
//
// Mirrors V3D_CUDA::SIFT_Matching (V3D/CUDA/v3d_cudamatching.h:15-67,
// v3d_cudamatching.cu:437-696): the handle keeps device buffers sized at allocate(), the
// current left/right descriptors, and the guided gates applied since the last putative
// call.  The reference recomputes nothing in runGuidedMatching: it masks the score
// matrix that the last findPutativeMatches left behind (.cu:597), so gates of successive
// guided calls compound.  Here no score matrix exists; a guided call re-runs the fused
// kernel with every gate recorded since the last putative call, which yields the same
// masked matrix and therefore the same matches.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "v3dm_internal.h"

using namespace v3dm;

struct v3dm_matcher {
  int device = 0;
  unsigned kernel = V3DM_KERNEL_TCGEN05;
  cudaStream_t stream = nullptr;
  bool allocated = false;
  bool guidedAlloc = false;
  int nMaxL = 0, nMaxR = 0;
  int nL = 0, nR = 0;
  uint8_t* dL = nullptr;
  uint8_t* dR = nullptr;
  float* dStage = nullptr;        // float upload staging, max(nMaxL, nMaxR) x 128
  unsigned long long* dLBest = nullptr;  // per left: best key
  unsigned int* dLSec = nullptr;         // per left: second value + 1
  unsigned long long* dRBest = nullptr;  // per right: best key
  unsigned int* dRSec = nullptr;         // per right: second value + 1
  unsigned long long* dCand = nullptr;   // candidate list (SIMT) / chunk-record entries (tcgen05): nSeg x segCap
  uint4* dRecords = nullptr;             // tcgen05 chunk records: nSeg x segCap x kRecordQuads
  // Pass-A cache (tcgen05): the side kernel applies no gates, so the chunk records and per-left
  // bounds of a pass A serve every later call on the same features with the same Smin (the
  // guided calls after a putative call, as the reference masks its stored score matrix).
  uint4* dRecordsA = nullptr;            // pass-A chunk records: nSeg x segCap x kRecordQuads
  int32_t* dPassA = nullptr;             // nSeg record counts, then nMaxL + 1 per-left bounds
  bool passAValid = false;
  long long testWaitLimit = 0;  // failure-path test hooks of pass A (v3dm_matcher_test_wait_fault)
  int testSkipLoad = 0;
  int32_t passASmin = 0, passATsec = 0;
  int* dSegCount = nullptr;              // nSeg counts
  long long segCap = 0;
  int nSeg = 0;
  int32_t* dScratch = nullptr;    // nMaxR + nMaxL ints of finalize scratch
  int32_t* dPairs = nullptr;      // 2 * min(nMaxL, nMaxR)
  int32_t* dInfo = nullptr;       // kInfoWords: pair count, error flags, largest segment
  int32_t* hInfo = nullptr;       // pinned mirror of dInfo
  bool pendingCheck = false;      // a device-only call whose info block was not read yet
  float* dLPos = nullptr;         // positions upload (interleaved x, y)
  float* dRPos = nullptr;
  float4* dGateL = nullptr;       // V3DM_MAX_GATES x nMaxL
  float4* dGateR = nullptr;       // V3DM_MAX_GATES x nMaxR
  GateParams* dGates = nullptr;   // device copy of gates[]
  int nGates = 0;
  GateParams gates[V3DM_MAX_GATES];
  TcPlan* tc = nullptr;
  bool tcBound = false;
  TcMaps mapsA, mapsB;            // tensor maps of the two side passes
  uint8_t* dRc = nullptr;         // descriptors of the chosen rights (second side pass)
  int32_t* dLeftDec = nullptr;    // per left: accepted right or -1
  int32_t* dRightDec = nullptr;   // per right: accepted left or -1
  int* dChosenFlag = nullptr;     // per right: chosen by some left (cleared after each call)
  int* dChosenList = nullptr;
  int* dFlagA = nullptr;          // lefts to re-score exactly
  int* dFlagB = nullptr;          // rights to re-score exactly
  int* dCounters = nullptr;       // [0] chosen rights, [1] flagged lefts, [2] flagged rights
                                  // (the 4 words after the info block, cleared with it)
  int32_t* countOut = nullptr;    // device-only calls: where the pair count also goes
  bool countWritten = false;      // the last enqueue wrote *countOut itself
  int lastLaunches = 0;
  // Float descriptors that are not u/512 (tcgen05 kernel): BF16 hi/lo operand layouts
  // (v3dm_match_f.cu), 6 planes of cap rows x 128 bytes each.
  bool floatL = false, floatR = false;  // the side's current descriptors are float
  int capFL = 0, capFR = 0;
  uint8_t* dLfA = nullptr;  // lefts, A layout (pass A operand)
  uint8_t* dLfB = nullptr;  // lefts, B layout (pass B operand)
  uint8_t* dRfA = nullptr;  // rights, A layout (gathered into dRcf)
  uint8_t* dRfB = nullptr;  // rights, B layout (pass A operand)
  uint8_t* dRcf = nullptr;  // chosen rights, A layout (pass B operand)
  bool fBound = false;
  CUtensorMap fmA_A, fmA_B, fmB_A, fmB_B;
  int numSMs = 148;
  // Optional CUDA-event timing of the fused matching kernel (v3dm_matcher_profile).
  bool profile = false;
  std::vector<cudaEvent_t> evPool;
  std::vector<int> evTag;         // per event pair: 0 = main kernel (SIMT, or tcgen05 pass A), 1 = pass B
  int evUsed = 0;
};

namespace {

thread_local char g_lastError[256] = "";

int cuda_fail(cudaError_t e, const char* what, int line) {
  record_cuda_error(e, "v3dm_api.cu", line, what);
  return V3DM_ERR_CUDA;
}

#define V3DM_CUDA_TRY(expr)                                      \
  do {                                                           \
    cudaError_t e_ = (expr);                                     \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr, __LINE__); \
  } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void free_buffers(v3dm_matcher* h) {
  dfree(h->dL);
  dfree(h->dR);
  dfree(h->dStage);
  dfree(h->dLBest);
  dfree(h->dLSec);
  dfree(h->dRBest);
  dfree(h->dRSec);
  dfree(h->dCand);
  dfree(h->dSegCount);
  dfree(h->dRecords);
  dfree(h->dRecordsA);
  dfree(h->dPassA);
  dfree(h->dScratch);
  dfree(h->dPairs);
  dfree(h->dInfo);
  dfree(h->dLPos);
  dfree(h->dRPos);
  dfree(h->dGateL);
  dfree(h->dGateR);
  dfree(h->dGates);
  dfree(h->dRc);
  dfree(h->dLeftDec);
  dfree(h->dRightDec);
  dfree(h->dChosenFlag);
  dfree(h->dChosenList);
  dfree(h->dFlagA);
  dfree(h->dFlagB);
  h->dCounters = nullptr;  // points into dInfo
  dfree(h->dLfA);
  dfree(h->dLfB);
  dfree(h->dRfA);
  dfree(h->dRfB);
  dfree(h->dRcf);
  h->floatL = h->floatR = false;
  h->capFL = h->capFR = 0;
  h->fBound = false;
  if (h->hInfo) cudaFreeHost(h->hInfo);
  h->hInfo = nullptr;
  h->allocated = false;
  h->tcBound = false;
  h->passAValid = false;
  h->nL = h->nR = 0;
  h->nGates = 0;
  h->segCap = 0;
  h->nSeg = 0;
  h->pendingCheck = false;
}

// (Re)allocates the candidate list for nSeg segments of segCap entries each.
cudaError_t alloc_candidates(v3dm_matcher* h, int nSeg, long long segCap) {
  dfree(h->dCand);
  dfree(h->dSegCount);
  dfree(h->dRecords);
  dfree(h->dRecordsA);
  h->segCap = 0;
  h->nSeg = 0;
  h->passAValid = false;
  cudaError_t e = dalloc(&h->dCand, (size_t)nSeg * (size_t)segCap);
  if (e == cudaSuccess && h->kernel != V3DM_KERNEL_SIMT)
    e = dalloc(&h->dRecords, (size_t)nSeg * (size_t)segCap * kRecordQuads);
  if (e == cudaSuccess && h->kernel != V3DM_KERNEL_SIMT)
    e = dalloc(&h->dRecordsA, (size_t)nSeg * (size_t)segCap * kRecordQuads);
  if (e == cudaSuccess) e = dalloc(&h->dSegCount, (size_t)nSeg);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dSegCount, 0, (size_t)nSeg * sizeof(int), h->stream);
  if (e != cudaSuccess) return e;
  h->segCap = segCap;
  h->nSeg = nSeg;
  return cudaSuccess;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// ---- candidate threshold ------------------------------------------------------------
// The decision of one side is accept(s1, s2) with s1 the best and s2 the second best score
// of that side.  For fixed s1 it is monotone in s2: nextDist = max(0.001, 2 - 2*s2) is
// non-increasing in s2 (each rounding is monotone) and bestDist / nextDist is monotone in
// nextDist with the sign of bestDist.  Hence, if accept(s1, hi) == accept(s1, -1e30f) for
// the largest value hi below T, every value below T gives the same decision.  For
// s1 > 1 (S1 > 2^18) bestDist < 0 and ratio < 0 for every s2: the decision is the same
// for all s2 whenever minRatio >= 0, so only S1 in [Smin, 2^18] needs checking.

bool invariant_below(int32_t T, int32_t Smin, float minScore, float minRatio, bool gated) {
  float hi = T > 0 ? score_of(T - 1) : (gated ? kMasked : kNone);
  int32_t top = kMaxScore < (1 << 18) ? kMaxScore : (1 << 18);
  for (int32_t S1 = Smin; S1 <= top; ++S1) {
    float s1 = score_of(S1);
    if (accept_scores(s1, hi, minScore, minRatio) != accept_scores(s1, kNone, minScore, minRatio)) return false;
  }
  return true;
}

struct ThrKey {
  uint32_t ms, mr;
  bool gated;
  bool operator==(const ThrKey& o) const { return ms == o.ms && mr == o.mr && gated == o.gated; }
};

std::mutex g_thrMutex;
ThrKey g_thrKeys[16];
int32_t g_thrVals[16];
int g_thrN = 0, g_thrNext = 0;

// Smallest S with score(S) > minScore: no best below it can pass the min-score test
// (kMaxScore + 1 when none can).
int32_t smallest_passing_score(float minScore) {
  int32_t Smin;
  if (!(minScore == minScore)) {
    Smin = kMaxScore + 1;  // NaN: 's1 > minScore' is never true
  } else if (minScore < 0.0f) {
    Smin = 0;
  } else {
    double g = std::floor((double)minScore * 262144.0);
    Smin = g > (double)kMaxScore ? kMaxScore + 1 : (int32_t)g;
    while (Smin > 0 && score_of(Smin - 1) > minScore) --Smin;
    while (Smin <= kMaxScore && !(score_of(Smin) > minScore)) ++Smin;
  }
  return Smin;
}

int compute_threshold(float minScore, float minRatio, bool gated, int32_t* Tout) {
  const int32_t Smin = smallest_passing_score(minScore);
  if (Smin > kMaxScore || minRatio < 0.0f || !(minRatio == minRatio)) {
    // Nothing can pass, or no ratio test, or a NaN ratio (never accepted): only the best
    // value matters and it cannot pass below Smin.
    *Tout = Smin;
    return V3DM_OK;
  }
  if (!invariant_below(0, Smin, minScore, minRatio, gated)) return V3DM_ERR_UNSUPPORTED;
  // Largest valid T in [0, Smin]; validity is monotone (a smaller T is valid when T is).
  // Start from the analytic cut-off c = 1 - (1 - minScore)/minRatio of s2, then gallop up.
  int32_t lo = 0;
  if (minRatio > 0.0f) {
    double c = 1.0 - (1.0 - (double)minScore) / (double)minRatio;
    double gS = std::floor(c * 262144.0) - 4.0;
    if (gS > 0) {
      int32_t g = gS < (double)Smin ? (int32_t)gS : Smin;
      while (g > 0 && !invariant_below(g, Smin, minScore, minRatio, gated)) g /= 2;
      lo = g;
    }
  }
  int32_t step = 1;
  while (lo + step <= Smin && invariant_below(lo + step, Smin, minScore, minRatio, gated)) {
    lo += step;
    step *= 2;
  }
  int32_t hi = lo + step - 1 < Smin ? lo + step - 1 : Smin;  // lo valid; lo + step invalid or > Smin
  while (lo < hi) {
    int32_t mid = lo + (hi - lo + 1) / 2;
    if (invariant_below(mid, Smin, minScore, minRatio, gated)) lo = mid;
    else hi = mid - 1;
  }
  *Tout = lo;
  return V3DM_OK;
}

}  // namespace

int32_t v3dm::host_smallest_passing_score(float minScore) { return smallest_passing_score(minScore); }

void v3dm::record_cuda_error(cudaError_t e, const char* file, int line, const char* what) {
  std::snprintf(g_lastError, sizeof(g_lastError), "%s (%s) at %s:%d: %s", cudaGetErrorName(e), cudaGetErrorString(e),
                file, line, what);
}

int v3dm::host_candidate_threshold(float minScore, float minRatio, bool gated, int32_t* T) {
  ThrKey k;
  std::memcpy(&k.ms, &minScore, 4);
  std::memcpy(&k.mr, &minRatio, 4);
  k.gated = gated;
  {
    std::lock_guard<std::mutex> lock(g_thrMutex);
    for (int i = 0; i < g_thrN; ++i)
      if (g_thrKeys[i] == k) {
        *T = g_thrVals[i];
        return V3DM_OK;
      }
  }
  int32_t t = 0;
  int st = compute_threshold(minScore, minRatio, gated, &t);
  if (st != V3DM_OK) return st;
  std::lock_guard<std::mutex> lock(g_thrMutex);
  g_thrKeys[g_thrNext] = k;
  g_thrVals[g_thrNext] = t;
  g_thrNext = (g_thrNext + 1) % 16;
  if (g_thrN < 16) ++g_thrN;
  *T = t;
  return V3DM_OK;
}

extern "C" {

const char* v3dm_status_string(int s) {
  switch (s) {
    case V3DM_OK: return "ok";
    case V3DM_ERR_ARG: return "invalid argument";
    case V3DM_ERR_CUDA: return "CUDA error";
    case V3DM_ERR_NOT_ALLOCATED: return "not allocated";
    case V3DM_ERR_SIZE: return "feature count above the allocated maximum";
    case V3DM_ERR_CAPACITY: return "output buffer too small";
    case V3DM_ERR_NOT_U8: return "float descriptor is not u/512 with u in 0..255";
    case V3DM_ERR_UNSUPPORTED: return "parameters outside the exact domain";
    case V3DM_ERR_TIMEOUT: return "device wait timed out";
    case V3DM_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case V3DM_ERR_CANDIDATES: return "candidate list overflow (list grown; repeat the call)";
    case V3DM_ERR_IO: return "feature file missing, not a feature archive, malformed or truncated";
    default: return "unknown status";
  }
}

const char* v3dm_last_error(void) { return g_lastError; }

int v3dm_candidate_threshold(float minScore, float minRatio, int gated, int32_t* T) {
  if (!T) return V3DM_ERR_ARG;
  return host_candidate_threshold(minScore, minRatio, gated != 0, T);
}

int v3dm_matcher_create(v3dm_matcher** out, int device, unsigned kernel) {
  if (!out || kernel > V3DM_KERNEL_SIMT) return V3DM_ERR_ARG;
  *out = nullptr;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return V3DM_ERR_CUDA;
  if (prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_matcher* h = new (std::nothrow) v3dm_matcher();
  if (!h) return V3DM_ERR_ARG;
  h->device = device;
  h->kernel = kernel;
  DeviceGuard g(device);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return V3DM_ERR_CUDA;
  }
  h->numSMs = prop.multiProcessorCount;
  if (kernel == V3DM_KERNEL_TCGEN05 && tc_plan_create(&h->tc, device) != cudaSuccess) {
    cudaStreamDestroy(h->stream);
    delete h;
    return V3DM_ERR_CUDA;
  }
  *out = h;
  return V3DM_OK;
}

int v3dm_matcher_destroy(v3dm_matcher* h) {
  if (!h) return V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  free_buffers(h);
  if (h->tc) tc_plan_destroy(h->tc);
  for (cudaEvent_t e : h->evPool) cudaEventDestroy(e);
  cudaStreamDestroy(h->stream);
  delete h;
  return V3DM_OK;
}

int v3dm_allocate(v3dm_matcher* h, int nMaxL, int nMaxR, int useGuided) {
  if (!h || nMaxL < 0 || nMaxR < 0) return V3DM_ERR_ARG;
  if (nMaxL > V3DM_MAX_FEATURES || nMaxR > V3DM_MAX_FEATURES) return V3DM_ERR_SIZE;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  free_buffers(h);
  h->nMaxL = nMaxL;
  h->nMaxR = nMaxR;
  h->guidedAlloc = useGuided != 0;
  int nMax = nMaxL > nMaxR ? nMaxL : nMaxR;
  int nMin = nMaxL < nMaxR ? nMaxL : nMaxR;
  // Operand rows are padded to whole 256-row tiles so TMA boxes never leave the buffer.
  size_t rowsL = ((size_t)nMaxL + 255) / 256 * 256, rowsR = ((size_t)nMaxR + 255) / 256 * 256;
  bool ok = dalloc(&h->dL, rowsL * kDescBytes) == cudaSuccess && dalloc(&h->dR, rowsR * kDescBytes) == cudaSuccess &&
            dalloc(&h->dStage, (size_t)nMax * kDescBytes) == cudaSuccess &&
            dalloc(&h->dLBest, (size_t)nMaxL + 1) == cudaSuccess && dalloc(&h->dLSec, (size_t)nMaxL + 1) == cudaSuccess &&
            dalloc(&h->dRBest, (size_t)nMaxR + 1) == cudaSuccess && dalloc(&h->dRSec, (size_t)nMaxR + 1) == cudaSuccess &&
            dalloc(&h->dScratch, (size_t)nMaxL + nMaxR + 1) == cudaSuccess &&
            dalloc(&h->dPairs, 2 * (size_t)nMin + 2) == cudaSuccess && dalloc(&h->dInfo, kInfoWords + 4) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&h->hInfo), kInfoWords * sizeof(int32_t)) == cudaSuccess;
  if (ok && h->guidedAlloc)
    ok = dalloc(&h->dLPos, 2 * (size_t)nMaxL + 2) == cudaSuccess && dalloc(&h->dRPos, 2 * (size_t)nMaxR + 2) == cudaSuccess &&
         dalloc(&h->dGateL, (size_t)V3DM_MAX_GATES * nMaxL + 1) == cudaSuccess &&
         dalloc(&h->dGateR, (size_t)V3DM_MAX_GATES * nMaxR + 1) == cudaSuccess &&
         dalloc(&h->dGates, (size_t)V3DM_MAX_GATES) == cudaSuccess;
  if (ok && h->kernel == V3DM_KERNEL_SIMT) {
    // SIMT path: one candidate list; about 1e-3 of all scores exceed T on SIFT-like data.
    // Start with room for 1/256 of them and grow when a call reports an overflow.
    long long segCap = (long long)nMaxL * (long long)nMaxR / 256 + 1;
    if (segCap < 4096) segCap = 4096;
    ok = alloc_candidates(h, 1, segCap) == cudaSuccess;
  } else if (ok) {
    // tcgen05 path: one list segment per epilogue warp, holding that warp's unit bests.
    ok = alloc_candidates(h, tc_segments(h->tc), 64) == cudaSuccess &&
         dalloc(&h->dPassA, (size_t)tc_segments(h->tc) + nMaxL + 1) == cudaSuccess &&
         dalloc(&h->dRc, rowsR * kDescBytes) == cudaSuccess && dalloc(&h->dLeftDec, (size_t)nMaxL + 1) == cudaSuccess &&
         dalloc(&h->dRightDec, (size_t)nMaxR + 1) == cudaSuccess &&
         dalloc(&h->dChosenFlag, (size_t)nMaxR + 1) == cudaSuccess &&
         dalloc(&h->dChosenList, (size_t)nMaxR + 1) == cudaSuccess && dalloc(&h->dFlagA, (size_t)nMaxL + 1) == cudaSuccess &&
         dalloc(&h->dFlagB, (size_t)nMaxR + 1) == cudaSuccess;
    if (ok) h->dCounters = h->dInfo + kInfoWords;
    if (ok)
      ok = cudaMemsetAsync(h->dChosenFlag, 0, ((size_t)nMaxR + 1) * sizeof(int), h->stream) == cudaSuccess &&
           cudaMemsetAsync(h->dRc, 0, rowsR * kDescBytes, h->stream) == cudaSuccess;
  }
  if (ok) {
    ok = cudaMemsetAsync(h->dLBest, 0, ((size_t)nMaxL + 1) * 8, h->stream) == cudaSuccess &&
         cudaMemsetAsync(h->dLSec, 0, ((size_t)nMaxL + 1) * 4, h->stream) == cudaSuccess &&
         cudaMemsetAsync(h->dRBest, 0, ((size_t)nMaxR + 1) * 8, h->stream) == cudaSuccess &&
         cudaMemsetAsync(h->dRSec, 0, ((size_t)nMaxR + 1) * 4, h->stream) == cudaSuccess &&
         cudaMemsetAsync(h->dL, 0, rowsL * kDescBytes, h->stream) == cudaSuccess &&
         cudaMemsetAsync(h->dR, 0, rowsR * kDescBytes, h->stream) == cudaSuccess &&
         cudaMemsetAsync(h->dInfo, 0, kInfoWords * sizeof(int32_t), h->stream) == cudaSuccess &&
         cudaStreamSynchronize(h->stream) == cudaSuccess;
  }
  if (!ok) {
    free_buffers(h);
    return V3DM_ERR_CUDA;
  }
  h->allocated = true;
  return V3DM_OK;
}

int v3dm_deallocate(v3dm_matcher* h) {
  if (!h) return V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  free_buffers(h);
  return V3DM_OK;
}

}  // extern "C"

namespace {

int set_features_u8(v3dm_matcher* h, bool left, int n, const uint8_t* desc, bool onDevice) {
  if (!h || n < 0 || (n > 0 && !desc)) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  if (n > (left ? h->nMaxL : h->nMaxR)) return V3DM_ERR_SIZE;
  DeviceGuard g(h->device);
  uint8_t* dst = left ? h->dL : h->dR;
  if (n > 0)
    V3DM_CUDA_TRY(cudaMemcpyAsync(dst, desc, (size_t)n * kDescBytes,
                                  onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
  (left ? h->nL : h->nR) = n;
  (left ? h->floatL : h->floatR) = false;
  h->tcBound = false;
  h->passAValid = false;
  return V3DM_OK;
}

// Float operand layouts of both sides (allocated on first use, kept until deallocate).
cudaError_t alloc_float(v3dm_matcher* h) {
  if (h->dLfA) return cudaSuccess;
  const int capL = std::max(256, (h->nMaxL + 255) / 256 * 256), capR = std::max(256, (h->nMaxR + 255) / 256 * 256);
  cudaError_t e = dalloc(&h->dLfA, (size_t)capL * kFloatRowBytes);
  if (e == cudaSuccess) e = dalloc(&h->dLfB, (size_t)capL * kFloatRowBytes);
  if (e == cudaSuccess) e = dalloc(&h->dRfA, (size_t)capR * kFloatRowBytes);
  if (e == cudaSuccess) e = dalloc(&h->dRfB, (size_t)capR * kFloatRowBytes);
  if (e == cudaSuccess) e = dalloc(&h->dRcf, (size_t)capR * kFloatRowBytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dLfA, 0, (size_t)capL * kFloatRowBytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dLfB, 0, (size_t)capL * kFloatRowBytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dRfA, 0, (size_t)capR * kFloatRowBytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dRfB, 0, (size_t)capR * kFloatRowBytes, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->dRcf, 0, (size_t)capR * kFloatRowBytes, h->stream);
  if (e != cudaSuccess) {
    dfree(h->dLfA);
    dfree(h->dLfB);
    dfree(h->dRfA);
    dfree(h->dRfB);
    dfree(h->dRcf);
    return e;
  }
  h->capFL = capL;
  h->capFR = capR;
  h->fBound = false;
  return cudaSuccess;
}

// The staged floats (h->dStage, n descriptors) into the side's BF16 hi/lo layouts.
int stage_to_float(v3dm_matcher* h, bool left, int n) {
  V3DM_CUDA_TRY(alloc_float(h));
  V3DM_CUDA_TRY(cudaMemsetAsync(h->dInfo + kInfoErr, 0, sizeof(int32_t), h->stream));
  V3DM_CUDA_TRY(launch_hilo(h->dStage, nullptr, n, left ? h->capFL : h->capFR, left ? h->dLfA : h->dRfA,
                            left ? h->dLfB : h->dRfB, h->dInfo + kInfoErr, h->stream));
  V3DM_CUDA_TRY(cudaMemcpyAsync(h->hInfo + kInfoErr, h->dInfo + kInfoErr, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                h->stream));
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->hInfo[kInfoErr]) {  // a value that is not finite
    (left ? h->nL : h->nR) = 0;
    cudaMemsetAsync(h->dInfo + kInfoErr, 0, sizeof(int32_t), h->stream);
    return V3DM_ERR_ARG;
  }
  (left ? h->nL : h->nR) = n;
  (left ? h->floatL : h->floatR) = true;
  h->tcBound = false;
  h->passAValid = false;
  return V3DM_OK;
}

// Float descriptors scored with the BF16 hi/lo split whatever their values.
int set_features_bf16x3(v3dm_matcher* h, bool left, int n, const float* desc) {
  if (!h || n < 0 || (n > 0 && !desc)) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  if (h->kernel == V3DM_KERNEL_SIMT) return V3DM_ERR_UNSUPPORTED;
  if (n > (left ? h->nMaxL : h->nMaxR)) return V3DM_ERR_SIZE;
  DeviceGuard g(h->device);
  if (n > 0)
    V3DM_CUDA_TRY(cudaMemcpyAsync(h->dStage, desc, (size_t)n * kDescBytes * sizeof(float), cudaMemcpyHostToDevice,
                                  h->stream));
  return stage_to_float(h, left, n);
}

int set_features_f32(v3dm_matcher* h, bool left, int n, const float* desc, bool onDevice = false) {
  if (!h || n < 0 || (n > 0 && !desc)) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  if (n > (left ? h->nMaxL : h->nMaxR)) return V3DM_ERR_SIZE;
  DeviceGuard g(h->device);
  uint8_t* dst = left ? h->dL : h->dR;
  if (n > 0) {
    V3DM_CUDA_TRY(cudaMemsetAsync(h->dInfo + kInfoErr, 0, sizeof(int32_t), h->stream));
    V3DM_CUDA_TRY(cudaMemcpyAsync(h->dStage, desc, (size_t)n * kDescBytes * sizeof(float),
                                  onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
    V3DM_CUDA_TRY(launch_f32_to_u8(h->dStage, dst, n, h->dInfo + kInfoErr, h->stream));
    V3DM_CUDA_TRY(cudaMemcpyAsync(h->hInfo + kInfoErr, h->dInfo + kInfoErr, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->hInfo[kInfoErr] & kErrNotU8) {
      cudaMemsetAsync(h->dInfo + kInfoErr, 0, sizeof(int32_t), h->stream);
      if (h->kernel == V3DM_KERNEL_SIMT) {
        (left ? h->nL : h->nR) = 0;
        return V3DM_ERR_NOT_U8;
      }
      // not of the form u/512: the tcgen05 handle scores these with the BF16 hi/lo split
      return stage_to_float(h, left, n);
    }
  }
  (left ? h->nL : h->nR) = n;
  (left ? h->floatL : h->floatR) = false;
  h->tcBound = false;
  h->passAValid = false;
  return V3DM_OK;
}

// Next pair of timing events (created on first use) tagged 'tag'.
int event_pair(v3dm_matcher* h, int tag, cudaEvent_t* ev) {
  for (int i = 0; i < 2; ++i) {
    if (h->evUsed == (int)h->evPool.size()) {
      cudaEvent_t e;
      V3DM_CUDA_TRY(cudaEventCreate(&e));
      h->evPool.push_back(e);
      h->evTag.push_back(0);
    }
    h->evTag[h->evUsed] = tag;
    ev[i] = h->evPool[h->evUsed++];
  }
  return V3DM_OK;
}

// SIMT path: candidate kernel, seconds pass, finalize.
int enqueue_match_simt(v3dm_matcher* h, float minScore, float minRatio, int32_t* dPairs) {
  int32_t T = 0;
  int st = host_candidate_threshold(minScore, minRatio, h->nGates > 0, &T);
  if (st != V3DM_OK) return st;
  MatchArgs a;
  std::memset(&a, 0, sizeof(a));
  a.nL = h->nL;
  a.nR = h->nR;
  a.T = T;
  a.lBest = h->dLBest;
  a.lSec = h->dLSec;
  a.rBest = h->dRBest;
  a.rSec = h->dRSec;
  a.cand = h->dCand;
  a.segCount = h->dSegCount;
  a.segCap = h->segCap;
  a.nSeg = h->nSeg;
  a.err = h->dInfo + kInfoErr;
  a.nGates = h->nGates;
  for (int i = 0; i < h->nGates; ++i) a.gates[i] = h->gates[i];
  a.gatesDev = h->dGates;
  if (h->nL > 0 && h->nR > 0 && T <= kMaxScore) {
    cudaEvent_t ev[2];
    if (h->profile) {
      int e = event_pair(h, 0, ev);
      if (e != V3DM_OK) return e;
      V3DM_CUDA_TRY(cudaEventRecord(ev[0], h->stream));
    }
    V3DM_CUDA_TRY(launch_match_simt(h->dL, h->dR, a, h->stream));
    if (h->profile) V3DM_CUDA_TRY(cudaEventRecord(ev[1], h->stream));
    V3DM_CUDA_TRY(launch_seconds(a, h->stream));
    h->lastLaunches += 2;
  }
  V3DM_CUDA_TRY(launch_finalize(a, minScore, minRatio, h->dScratch, dPairs, h->dInfo, h->stream));
  h->lastLaunches += 1;
  return V3DM_OK;
}

// tcgen05 path: side pass lefts x rights, decisions of the lefts, the chosen rights, side
// pass chosen rights x lefts, their decisions, mutual filter.
int enqueue_match_tc(v3dm_matcher* h, float minScore, float minRatio, int32_t* dPairs) {
  const int32_t Smin = smallest_passing_score(minScore);
  const bool gated = h->nGates > 0;
  const int cfg = tc_get_config(h->tc);
  if (!h->tcBound || h->mapsA.cfg != cfg) {
    V3DM_CUDA_TRY(tc_side_maps(h->tc, &h->mapsA, h->dL, h->nL, h->dR, h->nR));
    V3DM_CUDA_TRY(tc_side_maps(h->tc, &h->mapsB, h->dRc, h->nR, h->dL, h->nL));
    h->tcBound = true;
  }
  SideArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.Smin = Smin;
  if (host_candidate_threshold(minScore, minRatio, gated, &sa.Tsec) != V3DM_OK) sa.Tsec = 0;
  sa.records = h->dRecords;
  sa.segCount = h->dSegCount;
  sa.segCap = h->segCap;
  sa.nSeg = h->nSeg;
  sa.err = h->dInfo + kInfoErr;
  sa.nGates = h->nGates;
  sa.gatesDev = h->dGates;
  PostArgs pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.records = h->dRecords;
  pa.segCount = h->dSegCount;
  pa.Smin = Smin;
  pa.nGates = h->nGates;
  pa.gatesDev = h->dGates;
  pa.segCap = h->segCap;
  pa.nSeg = h->nSeg;
  pa.minScore = minScore;
  pa.minRatio = minRatio;
  pa.gated = gated;
  pa.err = h->dInfo + kInfoErr;
  RescoreArgs ra;
  std::memset(&ra, 0, sizeof(ra));
  if (gated) {
    int st = host_candidate_threshold(minScore, minRatio, true, &ra.T);
    if (st != V3DM_OK) return st;
  }
  ra.nGates = h->nGates;
  ra.gatesDev = h->dGates;
  ra.minScore = minScore;
  ra.minRatio = minRatio;
  cudaEvent_t evA[2], evB[2];
  // pass A: every left against every right, into the pass-A cache (records and per-left
  // bounds).  A guided call uses the cache instead when it holds this pass: same features,
  // same Smin, and bounds kept down to a threshold no higher than this call's -- as the
  // reference's guided calls mask the score matrix its putative call stored.  A putative
  // call always computes the pass (and refreshes the cache).
  int32_t* segCountA = h->dPassA;
  unsigned int* boundA = reinterpret_cast<unsigned int*>(h->dPassA + h->nSeg);
  int32_t tNeed = 0;
  if (host_candidate_threshold(minScore, minRatio, gated, &tNeed) != V3DM_OK) tNeed = 0;
  const bool reuseA = gated && h->passAValid && h->passASmin == Smin && h->passATsec <= tNeed;
  sa.nA = h->nL;
  sa.nB = h->nR;
  sa.aIsLeft = 1;
  sa.best = h->dLBest;
  if (!reuseA) {
    // bounds below the smaller of the ungated and gated thresholds of these parameters are
    // dropped, so the guided calls that follow can use this pass
    int32_t tu = 0, tg = 0;
    if (host_candidate_threshold(minScore, minRatio, false, &tu) != V3DM_OK) tu = 0;
    if (host_candidate_threshold(minScore, minRatio, true, &tg) != V3DM_OK) tg = 0;
    sa.Tsec = std::min(std::min(tu, tg), tNeed);
    sa.sec = boundA;
    sa.records = h->dRecordsA;
    sa.segCount = segCountA;
    V3DM_CUDA_TRY(cudaMemsetAsync(h->dPassA, 0, ((size_t)h->nSeg + h->nL) * sizeof(int32_t), h->stream));
    if (h->profile) {
      int e = event_pair(h, 0, evA);
      if (e != V3DM_OK) return e;
      V3DM_CUDA_TRY(cudaEventRecord(evA[0], h->stream));
    }
    sa.waitLimit = h->testWaitLimit;
    sa.skipLoad = h->testSkipLoad;
    V3DM_CUDA_TRY(launch_side(h->tc, h->mapsA, sa, h->stream));
    sa.waitLimit = 0;
    sa.skipLoad = 0;
    if (h->profile) V3DM_CUDA_TRY(cudaEventRecord(evA[1], h->stream));
    h->passAValid = true;
    h->passASmin = Smin;
    h->passATsec = sa.Tsec;
    h->lastLaunches += 1;
  }
  sa.sec = h->dLSec;
  sa.records = h->dRecords;
  sa.segCount = h->dSegCount;
  sa.Tsec = tNeed;
  pa.records = h->dRecordsA;
  pa.segCount = segCountA;
  pa.keepSegments = 1;
  pa.secBound = boundA;
  pa.nRows = h->nL;
  pa.nB = h->nR;
  pa.aIsLeft = 1;
  pa.best = h->dLBest;
  pa.sec = h->dLSec;
  pa.decision = h->dLeftDec;
  pa.flagged = h->dFlagA;
  pa.flaggedCount = h->dCounters + 1;
  if (!gated) {  // choose the accepted rights while deciding (no re-score can change a decision)
    pa.chooseFlag = h->dChosenFlag;
    pa.chooseList = h->dChosenList;
    pa.chooseCount = h->dCounters;
    pa.chooseSrc = h->dR;
    pa.chooseDst = h->dRc;
  }
  V3DM_CUDA_TRY(launch_post(pa, h->stream));
  pa.chooseFlag = nullptr;
  pa.records = h->dRecords;
  pa.segCount = h->dSegCount;
  pa.keepSegments = 0;
  pa.secBound = nullptr;
  h->lastLaunches += 2;
  if (gated) {
    ra.descA = h->dL;
    ra.descB = h->dR;
    ra.nB = h->nR;
    ra.aIsLeft = 1;
    ra.flagged = h->dFlagA;
    ra.flaggedCount = h->dCounters + 1;
    ra.best = h->dLBest;
    ra.sec = h->dLSec;
    ra.decision = h->dLeftDec;
    V3DM_CUDA_TRY(launch_rescore(ra, 64, h->stream));
    h->lastLaunches += 2;
  }
  if (gated) {
    V3DM_CUDA_TRY(launch_choose(h->dLeftDec, h->nL, h->dChosenFlag, h->dChosenList, h->dCounters, h->dR, h->dRc,
                                h->stream));
    h->lastLaunches += 1;
  }
  // pass B: the chosen rights against every left
  sa.nAptr = h->dCounters;
  sa.nA = h->nR;
  sa.nB = h->nL;
  sa.amap = h->dChosenList;
  sa.aIsLeft = 0;
  sa.best = h->dRBest;
  sa.sec = h->dRSec;
  if (h->profile) {
    int e = event_pair(h, 1, evB);
    if (e != V3DM_OK) return e;
    V3DM_CUDA_TRY(cudaEventRecord(evB[0], h->stream));
  }
  V3DM_CUDA_TRY(launch_side(h->tc, h->mapsB, sa, h->stream));
  if (h->profile) V3DM_CUDA_TRY(cudaEventRecord(evB[1], h->stream));
  pa.nRows = h->nR;
  pa.nB = h->nL;
  pa.aIsLeft = 0;
  pa.rowsPtr = h->dCounters;
  pa.amap = h->dChosenList;
  pa.best = h->dRBest;
  pa.sec = h->dRSec;
  pa.decision = h->dRightDec;
  pa.flagged = h->dFlagB;
  pa.flaggedCount = h->dCounters + 2;
  V3DM_CUDA_TRY(launch_post(pa, h->stream));
  h->lastLaunches += 3;
  if (gated) {
    ra.descA = h->dR;
    ra.descB = h->dL;
    ra.nB = h->nL;
    ra.aIsLeft = 0;
    ra.flagged = h->dFlagB;
    ra.flaggedCount = h->dCounters + 2;
    ra.best = h->dRBest;
    ra.sec = h->dRSec;
    ra.decision = h->dRightDec;
    V3DM_CUDA_TRY(launch_rescore(ra, 64, h->stream));
    h->lastLaunches += 2;
  }
  V3DM_CUDA_TRY(launch_mutual(h->dLeftDec, h->nL, h->dRightDec, h->dChosenFlag, h->dScratch,
                              reinterpret_cast<int2*>(dPairs), h->dInfo, h->countOut, h->stream));
  h->countWritten = h->countOut != nullptr;
  h->lastLaunches += 2;
  return V3DM_OK;
}

// Float path (either side holds float descriptors): the same two side passes and decisions with
// BF16 hi/lo scores (v3dm_match_f.cu).  A side holding u/512 descriptors gets its float layouts
// from its uint8 values, which is exact.
int enqueue_match_f(v3dm_matcher* h, float minScore, float minRatio, int32_t* dPairs) {
  const float Tf = host_float_threshold(minScore, minRatio);
  V3DM_CUDA_TRY(alloc_float(h));
  if (!h->floatL)
    V3DM_CUDA_TRY(launch_hilo(nullptr, h->dL, h->nL, h->capFL, h->dLfA, h->dLfB, h->dInfo + kInfoErr, h->stream));
  if (!h->floatR)
    V3DM_CUDA_TRY(launch_hilo(nullptr, h->dR, h->nR, h->capFR, h->dRfA, h->dRfB, h->dInfo + kInfoErr, h->stream));
  if (!h->fBound) {
    V3DM_CUDA_TRY(f_maps(&h->fmA_A, h->dLfA, h->capFL, &h->fmA_B, h->dRfB, h->capFR));
    V3DM_CUDA_TRY(f_maps(&h->fmB_A, h->dRcf, h->capFR, &h->fmB_B, h->dLfB, h->capFL));
    h->fBound = true;
  }
  SideArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.records = h->dRecords;
  sa.segCount = h->dSegCount;
  sa.segCap = h->segCap;
  sa.nSeg = h->nSeg;
  sa.err = h->dInfo + kInfoErr;
  PostArgs pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.records = h->dRecords;
  pa.segCount = h->dSegCount;
  pa.segCap = h->segCap;
  pa.nSeg = f_segments(h->numSMs);
  pa.nGates = h->nGates;
  pa.gatesDev = h->dGates;
  pa.minScore = minScore;
  pa.minRatio = minRatio;
  pa.err = h->dInfo + kInfoErr;
  cudaEvent_t evA[2], evB[2];
  // pass A: every left against every right
  sa.nA = h->nL;
  sa.nB = h->nR;
  sa.aIsLeft = 1;
  sa.best = h->dLBest;
  sa.sec = h->dLSec;
  if (h->profile) {
    int e = event_pair(h, 0, evA);
    if (e != V3DM_OK) return e;
    V3DM_CUDA_TRY(cudaEventRecord(evA[0], h->stream));
  }
  // Each CTA scores whole rows (128 lefts against every right) and decides them from the exact
  // best and second it keeps in registers, the call's gates applied where a score could enter
  // them; no chunk records for pass A.
  sa.rows = nullptr;
  sa.nGates = h->nGates;
  sa.gatesDev = h->dGates;
  sa.decision = h->dLeftDec;
  sa.minScore = minScore;
  sa.minRatio = minRatio;
  V3DM_CUDA_TRY(launch_side_f_batch(h->fmA_A, h->fmA_B, sa, Tf, h->numSMs, h->stream));
  sa.decision = nullptr;
  if (h->profile) V3DM_CUDA_TRY(cudaEventRecord(evA[1], h->stream));
  // the accepted rights, once each, gathered (six planes) for pass B
  V3DM_CUDA_TRY(launch_choose_planes(h->dLeftDec, h->nL, h->dChosenFlag, h->dChosenList, h->dCounters, h->dRfA,
                                     h->dRcf, kFloatRowBytes / kDescBytes, h->capFR, h->capFR, h->stream));
  // pass B: the chosen rights against every left
  sa.nAptr = h->dCounters;
  sa.nA = h->nR;
  sa.nB = h->nL;
  sa.amap = h->dChosenList;
  sa.aIsLeft = 0;
  sa.best = h->dRBest;
  sa.sec = h->dRSec;
  if (h->profile) {
    int e = event_pair(h, 1, evB);
    if (e != V3DM_OK) return e;
    V3DM_CUDA_TRY(cudaEventRecord(evB[0], h->stream));
  }
  V3DM_CUDA_TRY(launch_side_f(h->fmB_A, h->fmB_B, sa, Tf, nullptr, h->numSMs, h->stream));
  if (h->profile) V3DM_CUDA_TRY(cudaEventRecord(evB[1], h->stream));
  pa.nRows = h->nR;
  pa.rowsPtr = h->dCounters;
  pa.amap = h->dChosenList;
  pa.aIsLeft = 0;
  pa.best = h->dRBest;
  pa.sec = h->dRSec;
  pa.decision = h->dRightDec;
  V3DM_CUDA_TRY(launch_post_f(pa, Tf, h->stream));
  V3DM_CUDA_TRY(launch_mutual(h->dLeftDec, h->nL, h->dRightDec, h->dChosenFlag, h->dScratch,
                              reinterpret_cast<int2*>(dPairs), h->dInfo, h->countOut, h->stream));
  h->countWritten = h->countOut != nullptr;
  h->lastLaunches = (h->floatL ? 0 : 1) + (h->floatR ? 0 : 1) + 7;
  return V3DM_OK;
}

// Enqueues one matching call for the current gates; the result lands in dPairs / dInfo on
// the handle's stream.
int enqueue_match(v3dm_matcher* h, float minScore, float minRatio, int32_t* dPairs) {
  h->lastLaunches = 0;
  h->countWritten = false;
  // the info block and, right after it on the tcgen05 path, the call's counters
  V3DM_CUDA_TRY(cudaMemsetAsync(h->dInfo, 0, (h->dCounters ? kInfoWords + 4 : kInfoWords) * sizeof(int32_t),
                                h->stream));
  if (h->nGates > 0)
    V3DM_CUDA_TRY(cudaMemcpyAsync(h->dGates, h->gates, sizeof(GateParams) * h->nGates, cudaMemcpyHostToDevice,
                                  h->stream));
  int st;
  if (h->nL == 0 || h->nR == 0) {
    st = V3DM_OK;  // no pairs: the info block already says so
  } else if (h->kernel == V3DM_KERNEL_SIMT) {
    st = enqueue_match_simt(h, minScore, minRatio, dPairs);
  } else if (h->floatL || h->floatR) {
    st = enqueue_match_f(h, minScore, minRatio, dPairs);
  } else {
    st = enqueue_match_tc(h, minScore, minRatio, dPairs);
  }
  if (st == V3DM_OK) h->pendingCheck = true;
  return st;
}

// Reads the info block of the last call.  Returns V3DM_OK, an error, or -1 when the
// candidate list overflowed (the list has been grown and the call must be repeated).
int read_info(v3dm_matcher* h) {
  V3DM_CUDA_TRY(cudaMemcpyAsync(h->hInfo, h->dInfo, kInfoWords * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->pendingCheck = false;
  int err = h->hInfo[kInfoErr];
  if (err & kErrWaitTimeout) {
    h->passAValid = false;  // the pass stopped early: its records are incomplete
    return V3DM_ERR_TIMEOUT;
  }
  if (err) return V3DM_ERR_CUDA;
  long long need = h->hInfo[kInfoMaxSeg];
  if (need > h->segCap) {
    V3DM_CUDA_TRY(alloc_candidates(h, h->nSeg, need + need / 4 + 1024));
    return -1;
  }
  return V3DM_OK;
}

// Runs one matching call with host output, repeating it once the candidate list has grown.
int run_host(v3dm_matcher* h, float minScore, float minRatio, int32_t* pairs, int cap, int* nOut) {
  for (int attempt = 0; attempt < 4; ++attempt) {
    int st = enqueue_match(h, minScore, minRatio, h->dPairs);
    if (st != V3DM_OK) return st;
    st = read_info(h);
    if (st == -1) continue;
    if (st != V3DM_OK) return st;
    int n = h->hInfo[kInfoPairs];
    if (nOut) *nOut = n;
    int ncopy = n < cap ? n : cap;
    if (ncopy > 0) {
      V3DM_CUDA_TRY(cudaMemcpyAsync(pairs, h->dPairs, (size_t)ncopy * 2 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                    h->stream));
      V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    return n > cap ? V3DM_ERR_CAPACITY : V3DM_OK;
  }
  return V3DM_ERR_CUDA;
}

int add_gate(v3dm_matcher* h, int type, const double* M, float thr, const float* lpos, const float* rpos,
             bool onDevice) {
  if (!h->guidedAlloc) return V3DM_ERR_NOT_ALLOCATED;
  if (h->nGates >= V3DM_MAX_GATES) return V3DM_ERR_SIZE;
  int gi = h->nGates;
  const float* dl = lpos;
  const float* dr = rpos;
  if (!onDevice) {
    if (h->nL > 0)
      V3DM_CUDA_TRY(cudaMemcpyAsync(h->dLPos, lpos, (size_t)h->nL * 2 * sizeof(float), cudaMemcpyHostToDevice,
                                    h->stream));
    if (h->nR > 0)
      V3DM_CUDA_TRY(cudaMemcpyAsync(h->dRPos, rpos, (size_t)h->nR * 2 * sizeof(float), cudaMemcpyHostToDevice,
                                    h->stream));
    dl = h->dLPos;
    dr = h->dRPos;
  }
  float4* lv = h->dGateL + (size_t)gi * h->nMaxL;
  float4* rv = h->dGateR + (size_t)gi * h->nMaxR;
  V3DM_CUDA_TRY(launch_gate_precompute(type, M, dl, h->nL, dr, h->nR, lv, rv, h->stream));
  GateParams& gp = h->gates[gi];
  gp.type = type;
  gp.sqrThr = thr * thr;  // float product, as the reference (.cu:591)
  gp.lv = lv;
  gp.rv = rv;
  h->nGates = gi + 1;
  return V3DM_OK;
}

int guided_common(v3dm_matcher* h, int type, const double* M, float thr, const float* lpos, const float* rpos,
                  float minScore, float minRatio, int32_t* pairs, int cap, int* nOut) {
  if (!h || !M || (cap > 0 && !pairs) || cap < 0) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  if ((h->nL > 0 && !lpos) || (h->nR > 0 && !rpos)) return V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  int st = add_gate(h, type, M, thr, lpos, rpos, false);
  if (st != V3DM_OK) return st;
  return run_host(h, minScore, minRatio, pairs, cap, nOut);
}

}  // namespace

extern "C" {

int v3dm_set_left_u8(v3dm_matcher* h, int n, const uint8_t* d) { return set_features_u8(h, true, n, d, false); }
int v3dm_set_right_u8(v3dm_matcher* h, int n, const uint8_t* d) { return set_features_u8(h, false, n, d, false); }
int v3dm_set_left_u8_device(v3dm_matcher* h, int n, const uint8_t* d) { return set_features_u8(h, true, n, d, true); }
int v3dm_set_right_u8_device(v3dm_matcher* h, int n, const uint8_t* d) { return set_features_u8(h, false, n, d, true); }
int v3dm_set_left_f32(v3dm_matcher* h, int n, const float* d) { return set_features_f32(h, true, n, d); }
int v3dm_set_right_f32(v3dm_matcher* h, int n, const float* d) { return set_features_f32(h, false, n, d); }
int v3dm_set_left_f32_device(v3dm_matcher* h, int n, const float* d) { return set_features_f32(h, true, n, d, true); }
int v3dm_set_right_f32_device(v3dm_matcher* h, int n, const float* d) {
  return set_features_f32(h, false, n, d, true);
}
int v3dm_set_left_f32_bf16x3(v3dm_matcher* h, int n, const float* d) { return set_features_bf16x3(h, true, n, d); }
int v3dm_set_right_f32_bf16x3(v3dm_matcher* h, int n, const float* d) { return set_features_bf16x3(h, false, n, d); }

int v3dm_matcher_test_wait_fault(v3dm_matcher* h, long long waitCycles, int skipLoad) {
  if (!h || waitCycles < 0 || skipLoad < 0) return V3DM_ERR_ARG;
  if (skipLoad > 0 && waitCycles == 0) return V3DM_ERR_ARG;  // a skipped load needs a short wait limit
  DeviceGuard g(h->device);
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->testWaitLimit = waitCycles;
  h->testSkipLoad = skipLoad;
  h->passAValid = false;
  return V3DM_OK;
}

int v3dm_float_threshold(float minScore, float minRatio, float* T) {
  if (!T) return V3DM_ERR_ARG;
  *T = host_float_threshold(minScore, minRatio);
  return V3DM_OK;
}

int v3dm_scores_f32(v3dm_matcher* h, float* scores) {
  if (!h || !scores) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  if (h->kernel == V3DM_KERNEL_SIMT) return V3DM_ERR_UNSUPPORTED;
  const long long n = (long long)h->nL * h->nR;
  if (n > (1LL << 26)) return V3DM_ERR_SIZE;
  if (n == 0) return V3DM_OK;
  DeviceGuard g(h->device);
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  V3DM_CUDA_TRY(alloc_float(h));
  if (!h->floatL)
    V3DM_CUDA_TRY(launch_hilo(nullptr, h->dL, h->nL, h->capFL, h->dLfA, h->dLfB, h->dInfo + kInfoErr, h->stream));
  if (!h->floatR)
    V3DM_CUDA_TRY(launch_hilo(nullptr, h->dR, h->nR, h->capFR, h->dRfA, h->dRfB, h->dInfo + kInfoErr, h->stream));
  if (!h->fBound) {
    V3DM_CUDA_TRY(f_maps(&h->fmA_A, h->dLfA, h->capFL, &h->fmA_B, h->dRfB, h->capFR));
    V3DM_CUDA_TRY(f_maps(&h->fmB_A, h->dRcf, h->capFR, &h->fmB_B, h->dLfB, h->capFL));
    h->fBound = true;
  }
  float* dS = nullptr;
  V3DM_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&dS), (size_t)n * sizeof(float)));
  SideArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.records = h->dRecords;
  sa.segCount = h->dSegCount;
  sa.segCap = h->segCap;
  sa.nSeg = h->nSeg;
  sa.err = h->dInfo + kInfoErr;
  sa.nA = h->nL;
  sa.nB = h->nR;
  sa.aIsLeft = 1;
  // Tf = +inf: no chunk is handed over, only the dump is written
  cudaError_t e = launch_side_f(h->fmA_A, h->fmA_B, sa, INFINITY, dS, h->numSMs, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(scores, dS, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dS);
  if (e != cudaSuccess) return cuda_fail(e, "scores_f32", __LINE__);
  return V3DM_OK;
}

int v3dm_putative(v3dm_matcher* h, float minScore, float minRatio, int32_t* pairs, int cap, int* nOut) {
  if (!h || (cap > 0 && !pairs) || cap < 0) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuard g(h->device);
  h->nGates = 0;
  return run_host(h, minScore, minRatio, pairs, cap, nOut);
}

int v3dm_guided_F(v3dm_matcher* h, const double* F, float thr, const float* lpos, const float* rpos, float minScore,
                  float minRatio, int32_t* pairs, int cap, int* nOut) {
  return guided_common(h, 1, F, thr, lpos, rpos, minScore, minRatio, pairs, cap, nOut);
}

int v3dm_guided_H(v3dm_matcher* h, const double* H, float thr, const float* lpos, const float* rpos, float minScore,
                  float minRatio, int32_t* pairs, int cap, int* nOut) {
  return guided_common(h, 2, H, thr, lpos, rpos, minScore, minRatio, pairs, cap, nOut);
}

int v3dm_putative_device(v3dm_matcher* h, float minScore, float minRatio, int32_t* d_pairs, int32_t* d_count) {
  if (!h || !d_pairs || !d_count) return V3DM_ERR_ARG;
  if (!dev_aligned(d_pairs, 8) || !dev_aligned(d_count, 4)) return V3DM_ERR_ARG;  // pairs are written as int2
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuard g(h->device);
  h->nGates = 0;
  h->countOut = d_count;
  int st = enqueue_match(h, minScore, minRatio, d_pairs);
  h->countOut = nullptr;
  if (st != V3DM_OK) return st;
  if (!h->countWritten)
    V3DM_CUDA_TRY(cudaMemcpyAsync(d_count, h->dInfo, sizeof(int32_t), cudaMemcpyDeviceToDevice, h->stream));
  return V3DM_OK;
}

int v3dm_guided_F_device(v3dm_matcher* h, const double* F, float thr, const float* d_lpos, const float* d_rpos,
                         float minScore, float minRatio, int32_t* d_pairs, int32_t* d_count) {
  if (!h || !F || !d_pairs || !d_count) return V3DM_ERR_ARG;
  // pairs are written as int2, positions read as float2
  if (!dev_aligned(d_pairs, 8) || !dev_aligned(d_count, 4) || !dev_aligned(d_lpos, 8) || !dev_aligned(d_rpos, 8))
    return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuard g(h->device);
  int st = add_gate(h, 1, F, thr, d_lpos, d_rpos, true);
  if (st != V3DM_OK) return st;
  h->countOut = d_count;
  st = enqueue_match(h, minScore, minRatio, d_pairs);
  h->countOut = nullptr;
  if (st != V3DM_OK) return st;
  if (!h->countWritten)
    V3DM_CUDA_TRY(cudaMemcpyAsync(d_count, h->dInfo, sizeof(int32_t), cudaMemcpyDeviceToDevice, h->stream));
  return V3DM_OK;
}

int v3dm_matcher_stream(v3dm_matcher* h, void** s) {
  if (!h || !s) return V3DM_ERR_ARG;
  *s = (void*)h->stream;
  return V3DM_OK;
}

int v3dm_matcher_wait(v3dm_matcher* h) {
  if (!h) return V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  if (!h->pendingCheck) {
    V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return V3DM_OK;
  }
  int st = read_info(h);
  return st == -1 ? V3DM_ERR_CANDIDATES : st;
}

int v3dm_matcher_profile(v3dm_matcher* h, int enable) {
  if (!h) return V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->profile = enable != 0;
  h->evUsed = 0;
  return V3DM_OK;
}

int v3dm_matcher_profile_read(v3dm_matcher* h, double* msTotal, int* launches) {
  return v3dm_matcher_profile_read_pass(h, 0, msTotal, launches);
}

int v3dm_matcher_profile_read_pass(v3dm_matcher* h, int pass, double* msTotal, int* launches) {
  if (!h || !msTotal || !launches || pass < 0 || pass > 1) return V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  double total = 0.0;
  int n = 0;
  for (int i = 0; i + 1 < h->evUsed; i += 2) {
    if (h->evTag[i] != pass) continue;
    float ms = 0.f;
    V3DM_CUDA_TRY(cudaEventElapsedTime(&ms, h->evPool[i], h->evPool[i + 1]));
    total += ms;
    ++n;
  }
  *msTotal = total;
  *launches = n;
  if (pass == 1 || !h->profile) h->evUsed = 0;
  return V3DM_OK;
}

int v3dm_matcher_num_configs(v3dm_matcher* h, int* n) {
  if (!h || !n) return V3DM_ERR_ARG;
  *n = h->kernel == V3DM_KERNEL_SIMT ? 1 : tc_num_configs();
  return V3DM_OK;
}

int v3dm_matcher_get_config(v3dm_matcher* h, int* cfg, int* rowsPerGroup, int* colsPerTile) {
  if (!h || !cfg) return V3DM_ERR_ARG;
  if (h->kernel == V3DM_KERNEL_SIMT) {
    *cfg = 0;
    if (rowsPerGroup) *rowsPerGroup = 64;
    if (colsPerTile) *colsPerTile = 64;
    return V3DM_OK;
  }
  *cfg = tc_get_config(h->tc);
  int r = 0, c = 0;
  tc_config_shape(*cfg, &r, &c);
  if (rowsPerGroup) *rowsPerGroup = r;
  if (colsPerTile) *colsPerTile = c;
  return V3DM_OK;
}

int v3dm_matcher_set_config(v3dm_matcher* h, int cfg) {
  if (!h) return V3DM_ERR_ARG;
  if (h->kernel == V3DM_KERNEL_SIMT) return cfg == 0 ? V3DM_OK : V3DM_ERR_ARG;
  DeviceGuard g(h->device);
  V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (tc_set_config(h->tc, cfg) != cudaSuccess) return V3DM_ERR_ARG;
  return V3DM_OK;
}

int v3dm_matcher_autotune(v3dm_matcher* h, float minScore, float minRatio, int reps, int* best, double* msBest) {
  if (!h || reps < 1) return V3DM_ERR_ARG;
  if (!h->allocated) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuard g(h->device);
  int n = h->kernel == V3DM_KERNEL_SIMT ? 1 : tc_num_configs();
  int keepGates = h->nGates;
  int bestCfg = 0;
  double bestMs = 1e300;
  for (int c = 0; c < n; ++c) {
    if (h->kernel != V3DM_KERNEL_SIMT && tc_set_config(h->tc, c) != cudaSuccess) continue;
    h->nGates = 0;
    int st = run_host(h, minScore, minRatio, nullptr, 0, nullptr);  // warm-up, grows the list if needed
    if (st != V3DM_OK && st != V3DM_ERR_CAPACITY) {
      h->nGates = keepGates;
      return st;
    }
    bool prof = h->profile;
    h->profile = true;
    h->evUsed = 0;
    for (int r = 0; r < reps; ++r) {
      st = enqueue_match(h, minScore, minRatio, h->dPairs);
      if (st != V3DM_OK) {
        h->profile = prof;
        h->nGates = keepGates;
        return st;
      }
    }
    V3DM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    double total = 0.0;
    for (int i = 0; i + 1 < h->evUsed; i += 2) {
      float ms = 0.f;
      V3DM_CUDA_TRY(cudaEventElapsedTime(&ms, h->evPool[i], h->evPool[i + 1]));
      total += ms;
    }
    h->evUsed = 0;
    h->profile = prof;
    st = read_info(h);
    if (st != V3DM_OK && st != -1) {
      h->nGates = keepGates;
      return st;
    }
    double avg = total / reps;
    if (avg < bestMs) {
      bestMs = avg;
      bestCfg = c;
    }
  }
  h->nGates = keepGates;
  if (h->kernel != V3DM_KERNEL_SIMT) tc_set_config(h->tc, bestCfg);
  if (best) *best = bestCfg;
  if (msBest) *msBest = bestMs;
  return V3DM_OK;
}

int v3dm_matcher_last_launches(v3dm_matcher* h, int* n) {
  if (!h || !n) return V3DM_ERR_ARG;
  *n = h->lastLaunches;
  return V3DM_OK;
}

}  // extern "C"
