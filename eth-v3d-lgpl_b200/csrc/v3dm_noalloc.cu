// v3dm_noalloc.cu -- putative matching that allocates no device memory.
//
// Some callers cannot allocate device memory while they match: a host application that
// owns every byte of GPU memory and hands plug-ins a fixed budget, a frame loop where a
// cudaMalloc/cudaFree would synchronise the device and blow the frame's latency, or a
// service that must not meet an out-of-memory error halfway through a job.  For them,
// v3dm_putative_u8_noalloc runs the dp4a matching kernels of v3dm_match.cu with all of their
// working memory in one fixed array that lives in this library's device image
// (g_noallocScratch below): every GPU that loads the library holds it until the process
// exits.  The caller passes device pointers for the descriptors and for the results only.
//
// Limits: at most kNoAllocMaxFeatures (8192) descriptors per side, and at most
// kNoAllocMaxCandidates (524288) scores at or above the candidate threshold per call
// (SIFT-like data produces about 1e-3 of nL*nR, i.e. ~67k for 8192 x 8192).  Past the
// second limit the call reports -1 as the pair count instead of a wrong result.
//
// Every call uses the same array.  Calls whose work overlaps on the GPU (two streams, two
// host threads) race on it; serialise them.  The array keeps the previous call's contents,
// so each call first clears the parts that must start at zero.  The first call on a device
// looks up the array's device address with cudaGetSymbolAddress (with that device current);
// make that first call before any stream capture begins.
#include <cstdint>
#include <mutex>

#include "v3dm_internal.h"

namespace v3dm {

namespace {

constexpr int kNoAllocMaxFeatures = V3DM_NOALLOC_MAX_FEATURES;
constexpr long long kNoAllocMaxCandidates = V3DM_NOALLOC_MAX_CANDIDATES;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of the sub-buffers inside the scratch array.
constexpr size_t kOffLBest = 0;
constexpr size_t kOffRBest = kOffLBest + align256(sizeof(unsigned long long) * kNoAllocMaxFeatures);
constexpr size_t kOffLSec = kOffRBest + align256(sizeof(unsigned long long) * kNoAllocMaxFeatures);
constexpr size_t kOffRSec = kOffLSec + align256(sizeof(unsigned int) * kNoAllocMaxFeatures);
constexpr size_t kOffInfo = kOffRSec + align256(sizeof(unsigned int) * kNoAllocMaxFeatures);
constexpr size_t kOffSegCount = kOffInfo + align256(sizeof(int32_t) * kInfoWords);
constexpr size_t kClearBytes = kOffSegCount + align256(sizeof(int));  // everything above starts at zero
constexpr size_t kOffDecisions = kClearBytes;
constexpr size_t kOffCand = kOffDecisions + align256(sizeof(int32_t) * 2 * kNoAllocMaxFeatures);
constexpr size_t kScratchBytes = kOffCand + sizeof(unsigned long long) * kNoAllocMaxCandidates;

static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

std::mutex g_scratchMutex;
void* g_scratchAddr[128] = {};  // device address of g_noallocScratch, per device ordinal

__global__ void k_noalloc_clear(uint4* p, size_t n16) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
    p[i] = make_uint4(0u, 0u, 0u, 0u);
}

// Pair count for the caller, or -1 when the candidate list overflowed or a kernel flagged
// an error.
__global__ void k_noalloc_status(const int32_t* info, long long cap, int32_t* count) {
  const bool bad = info[kInfoErr] != 0 || (long long)info[kInfoMaxSeg] > cap;
  *count = bad ? -1 : info[kInfoPairs];
}

// Makes `dev` current for the call and restores the caller's device afterwards.  ok is false
// when the device cannot be made current; the call must then queue nothing.
struct NoAllocDeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit NoAllocDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
  }
  ~NoAllocDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

}  // namespace v3dm

using namespace v3dm;

extern "C" int v3dm_putative_u8_noalloc(int device, const uint8_t* d_left, int nLeft, const uint8_t* d_right,
                                        int nRight, float minScore, float minRatio, int32_t* d_pairs,
                                        int32_t* d_count, void* stream) {
  if (nLeft < 0 || nRight < 0 || !d_count || (nLeft > 0 && !d_left) || (nRight > 0 && !d_right) ||
      (nLeft > 0 && nRight > 0 && !d_pairs) || device < 0 || device >= 128)
    return V3DM_ERR_ARG;
  // descriptors are read as 32-bit words, pairs written as int2
  if (!dev_aligned(d_left, 4) || !dev_aligned(d_right, 4) || !dev_aligned(d_pairs, 8) || !dev_aligned(d_count, 4))
    return V3DM_ERR_ARG;
  if (nLeft > kNoAllocMaxFeatures || nRight > kNoAllocMaxFeatures) return V3DM_ERR_SIZE;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess) return V3DM_ERR_NO_DEVICE;
  if (device >= nDev) return V3DM_ERR_ARG;
  // An error left pending by earlier, unrelated work would surface only after this call had
  // queued kernels; refuse up front instead, and leave the error for its owner to read.
  if (cudaPeekAtLastError() != cudaSuccess) return V3DM_ERR_CUDA;
  NoAllocDeviceGuard guard(device);
  if (!guard.ok) return V3DM_ERR_CUDA;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    if (!g_scratchAddr[device]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noallocScratch) != cudaSuccess || !p) return V3DM_ERR_CUDA;
      g_scratchAddr[device] = p;
    }
    base = static_cast<unsigned char*>(g_scratchAddr[device]);
  }
  int32_t T = 0;
  int st = host_candidate_threshold(minScore, minRatio, false, &T);
  if (st != V3DM_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  MatchArgs a{};
  a.nL = nLeft;
  a.nR = nRight;
  a.T = T;
  a.lBest = reinterpret_cast<unsigned long long*>(base + kOffLBest);
  a.rBest = reinterpret_cast<unsigned long long*>(base + kOffRBest);
  a.lSec = reinterpret_cast<unsigned int*>(base + kOffLSec);
  a.rSec = reinterpret_cast<unsigned int*>(base + kOffRSec);
  a.cand = reinterpret_cast<unsigned long long*>(base + kOffCand);
  a.segCount = reinterpret_cast<int*>(base + kOffSegCount);
  a.segCap = kNoAllocMaxCandidates;
  a.nSeg = 1;
  int32_t* info = reinterpret_cast<int32_t*>(base + kOffInfo);
  a.err = info + kInfoErr;
  a.nGates = 0;
  a.gatesDev = nullptr;
  k_noalloc_clear<<<64, 256, 0, s>>>(reinterpret_cast<uint4*>(base), kClearBytes / 16);
  if (cudaGetLastError() != cudaSuccess) return V3DM_ERR_CUDA;
  if (nLeft > 0 && nRight > 0 && T <= kMaxScore) {
    if (launch_match_simt(d_left, d_right, a, s) != cudaSuccess) return V3DM_ERR_CUDA;
    if (launch_seconds(a, s) != cudaSuccess) return V3DM_ERR_CUDA;
  }
  if (launch_finalize(a, minScore, minRatio, reinterpret_cast<int32_t*>(base + kOffDecisions), d_pairs, info, s) !=
      cudaSuccess)
    return V3DM_ERR_CUDA;
  k_noalloc_status<<<1, 1, 0, s>>>(info, kNoAllocMaxCandidates, d_count);
  return cudaGetLastError() == cudaSuccess ? V3DM_OK : V3DM_ERR_CUDA;
}
