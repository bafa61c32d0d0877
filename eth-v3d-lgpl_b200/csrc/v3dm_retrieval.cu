// v3dm_retrieval.cu -- vocabulary-tree retrieval scoring: the candidate pairs of an image sequence.
//
// The voctree app (match_using_voctree.cpp:176-222) walks the images in order; for image i it
// scores every earlier image d with LeafDocuments::computeBinomialScores
// (V3D/Base/v3d_voctree.h:233-278), keeps the nBestDocuments lowest scores, then inserts image i
// into the inverted files (insertDocument, :143-163).  For a query i and a document d:
//   k = the number of query features whose word occurs in d   (getDocumentHistogram, :165-177:
//       one count per query feature per inverted-file entry, and d has one entry per word),
//   n = min(nFeatures(d), nFeatures(i)),  p0 = max(nFeatures(d), nFeatures(i)) * (1 / nLeaves),
//   p1 = min(1, p0 + pMatch),
//   score = float((k log p0 + (n - k) log(1 - p0)) - (k log p1 + (n - k) log(1 - p1)))
// in double with one rounding per operation, ranked ascending by (score, d).
//
// All queries run at once, one CTA per query image (largest image index first):
//   k_rt_presence  the inverted files as a bitmap: bit d of leaf row w is set when image d has
//                  word w (nLeaves rows of ceil(nImages / 32) words);
//   k_rt_score     k(d) for every d < i: a thread owns a column of the bitmap (32 images) and sums
//                  that column of the leaf rows of the query's features with bit-sliced counters
//                  (a warp reads 128 contiguous bytes of a row; no atomics while counting, and the
//                  cost does not depend on how the words are distributed); the scores in the
//                  reference's operation order from logarithms computed on the host (the C
//                  library's log, as the reference's); then a radix select of the nBest smallest
//                  (score, d) keys (six 8-bit digits of a 48-bit key: the score's order bits, then
//                  d) and a rank sort of those.
// k is an exact count, so scores and order are bit-identical to the reference's.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "v3dm_internal.h"

using namespace v3dm;

namespace {

constexpr int kRtThreads = 512;
constexpr int kRtPresenceThreads = 256;

struct RtLogs {  // the four logarithms of one image's p0 = nFeatures * (1 / nLeaves)
  double lp0, l1p0, lp1, l1p1;
};

__global__ void k_rt_presence(const int32_t* __restrict__ offsets, const int32_t* __restrict__ words, int nLeaves,
                              int w32, uint32_t* __restrict__ bits, int* __restrict__ err) {
  const int i = blockIdx.x;
  const int b = offsets[i], e = offsets[i + 1];
  for (int j = b + threadIdx.x; j < e; j += blockDim.x) {
    const int w = words[j];
    if (w < 0 || w >= nLeaves) {
      atomicOr(err, 1);
      continue;
    }
    atomicOr(&bits[(size_t)w * w32 + (i >> 5)], 1u << (i & 31));
  }
}

// Order bits of a float score: unsigned comparison of these is the float order, -0 equal to +0,
// NaN after every number.
__device__ __forceinline__ uint32_t rt_order(float f) {
  if (f != f) return 0xffffffffu;
  if (f == 0.0f) return 0x80000000u;
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float rt_unorder(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// Bit-sliced column counters: bit k of plane p holds bit p of image k's count.  Sixteen rows at
// a time go through a carry-save adder tree (Harley-Seal) into the planes of weight 1, 2, 4 and
// 8; the carries of weight 16 ripple into the planes above.
constexpr int kRtHigh = 11;          // planes of weight 16 .. 2^14
constexpr int kRtSegment = 32752;    // rows per flush: a count stays below 2^15
constexpr int kRtChunk = 4096;       // row offsets staged in shared memory at a time

struct RtPlanes {
  uint32_t ones, twos, fours, eights, hi[kRtHigh];
};

__device__ __forceinline__ void rt_csa(uint32_t& hi, uint32_t& lo, uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t u = a ^ b;
  hi = (a & b) | (u & c);
  lo = u ^ c;
}

__device__ __forceinline__ void rt_clear(RtPlanes& p) {
  p.ones = p.twos = p.fours = p.eights = 0;
#pragma unroll
  for (int q = 0; q < kRtHigh; ++q) p.hi[q] = 0;
}

// Adds the counts of the images of 'mask' to kdCol[0..31] and clears the planes.
__device__ __forceinline__ void rt_flush(RtPlanes& p, uint32_t mask, uint32_t* kdCol) {
  uint32_t any = p.ones | p.twos | p.fours | p.eights;
#pragma unroll
  for (int q = 0; q < kRtHigh; ++q) any |= p.hi[q];
  any &= mask;
  while (any) {
    const int k = __ffs(any) - 1;
    any &= any - 1u;
    uint32_t cnt = ((p.ones >> k) & 1u) | (((p.twos >> k) & 1u) << 1) | (((p.fours >> k) & 1u) << 2) |
                   (((p.eights >> k) & 1u) << 3);
#pragma unroll
    for (int q = 0; q < kRtHigh; ++q) cnt |= ((p.hi[q] >> k) & 1u) << (q + 4);
    atomicAdd(&kdCol[k], cnt);
  }
  rt_clear(p);
}

// Sixteen rows of one column into the planes.
__device__ __forceinline__ void rt_add16(RtPlanes& p, const uint32_t (&x)[16]) {
  uint32_t twosA, twosB, foursA, foursB, eightsA, eightsB, sixteens;
  rt_csa(twosA, p.ones, p.ones, x[0], x[1]);
  rt_csa(twosB, p.ones, p.ones, x[2], x[3]);
  rt_csa(foursA, p.twos, p.twos, twosA, twosB);
  rt_csa(twosA, p.ones, p.ones, x[4], x[5]);
  rt_csa(twosB, p.ones, p.ones, x[6], x[7]);
  rt_csa(foursB, p.twos, p.twos, twosA, twosB);
  rt_csa(eightsA, p.fours, p.fours, foursA, foursB);
  rt_csa(twosA, p.ones, p.ones, x[8], x[9]);
  rt_csa(twosB, p.ones, p.ones, x[10], x[11]);
  rt_csa(foursA, p.twos, p.twos, twosA, twosB);
  rt_csa(twosA, p.ones, p.ones, x[12], x[13]);
  rt_csa(twosB, p.ones, p.ones, x[14], x[15]);
  rt_csa(foursB, p.twos, p.twos, twosA, twosB);
  rt_csa(eightsB, p.fours, p.fours, foursA, foursB);
  rt_csa(sixteens, p.eights, p.eights, eightsA, eightsB);
#pragma unroll
  for (int q = 0; q < kRtHigh; ++q) {
    if (!sixteens) break;
    const uint32_t t = p.hi[q] & sixteens;
    p.hi[q] ^= sixteens;
    sixteens = t;
  }
}

__global__ void __launch_bounds__(kRtThreads, 2)
k_rt_score(const int32_t* __restrict__ offsets, const int32_t* __restrict__ words, int nLeaves, int nImages, int w32,
           const uint32_t* __restrict__ bits, const RtLogs* __restrict__ logs, int nBest,
           int32_t* __restrict__ bestDocs, float* __restrict__ bestScores) {
  extern __shared__ unsigned long long rtSh[];
  unsigned long long* cand = rtSh;                             // nBest selected keys
  uint32_t* kd = reinterpret_cast<uint32_t*>(rtSh + nBest);    // k(d), then the order bits of d's score
  __shared__ uint32_t hist[256];
  __shared__ __align__(16) uint32_t rowOff[kRtChunk];
  __shared__ unsigned long long shPrefix;
  __shared__ int shRem, shCnt;

  const int i = nImages - 1 - blockIdx.x;  // the longest queries first
  const uint32_t tailMask = (i & 31) ? (1u << (i & 31)) - 1u : 0xffffffffu;  // images before i
  for (int d = threadIdx.x; d < i; d += blockDim.x) kd[d] = 0;
  if (threadIdx.x == 0) shCnt = 0;
  __syncthreads();

  // k(d): a thread owns one bitmap column (32 images) of a pass over at most blockDim.x columns
  // and adds up that column of the rows of the query's words with bit-sliced counters; the
  // threads of a pass form 'groups' groups that split the rows.  The rows' offsets are staged in
  // shared memory a chunk at a time (invalid words and the padding point to the all-zero row).
  const int b = offsets[i], e = offsets[i + 1];
  const int nw = (i + 31) >> 5;
  // one pass over the columns while they fit the block, else the fewest passes of equal width;
  // groups of threads split the rows (each extra pass repeats the staging and the flushes)
  const int passes = (nw + (int)blockDim.x - 1) / (int)blockDim.x;
  const int colsPerPass = max(1, (nw + passes - 1) / max(passes, 1));
  const int groups = min((int)blockDim.x / colsPerPass, kRtChunk / 16);  // 16 * groups <= kRtChunk
  const int g = threadIdx.x / colsPerPass;
  const bool active = g < groups;
  const int chunkRows = (kRtChunk / (16 * groups)) * 16 * groups;  // >= 16 * groups, a multiple of it
  const uint32_t zeroRow = (uint32_t)nLeaves * (uint32_t)w32;
  for (int c0 = 0; c0 < nw; c0 += colsPerPass) {
    const int col = c0 + (int)threadIdx.x % colsPerPass;
    const bool mine = active && col < nw;
    const uint32_t* bitsCol = bits + (mine ? col : 0);
    const uint32_t mask = col == nw - 1 ? tailMask : 0xffffffffu;
    RtPlanes p;
    rt_clear(p);
    int inSegment = 0;  // rows added since the last flush
    for (int f0 = b; f0 < e; f0 += chunkRows) {
      __syncthreads();  // the previous chunk has been read
      for (int r = threadIdx.x; r < chunkRows; r += blockDim.x) {
        const int j = f0 + r;
        uint32_t off = zeroRow;
        if (j < e) {
          const int w = __ldg(words + j);
          if (w >= 0 && w < nLeaves) off = (uint32_t)w * (uint32_t)w32;  // else reported by k_rt_presence
        }
        rowOff[r] = off;
      }
      __syncthreads();
      if (mine) {
        const int rows = min(chunkRows, ((e - f0) + 16 * groups - 1) / (16 * groups) * (16 * groups));
        if (inSegment + rows / groups > kRtSegment) {
          rt_flush(p, mask, kd + (col << 5));
          inSegment = 0;
        }
        inSegment += rows / groups;
        for (int r0 = 16 * g; r0 < rows; r0 += 16 * groups) {
          const uint4* ro = reinterpret_cast<const uint4*>(rowOff + r0);  // r0 is a multiple of 16
          uint32_t x[16];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint4 o = ro[q];
            x[4 * q + 0] = __ldg(bitsCol + o.x);
            x[4 * q + 1] = __ldg(bitsCol + o.y);
            x[4 * q + 2] = __ldg(bitsCol + o.z);
            x[4 * q + 3] = __ldg(bitsCol + o.w);
          }
          rt_add16(p, x);
        }
      }
    }
    if (mine) rt_flush(p, mask, kd + (col << 5));
  }
  __syncthreads();

  // scores, in the order of operations of v3d_voctree.h:250-270
  const int nq = e - b;
  for (int d = threadIdx.x; d < i; d += blockDim.x) {
    const int nd = offsets[d + 1] - offsets[d];
    const RtLogs L = logs[nd >= nq ? d : i];  // the logarithms of max(nd, nq) * (1 / nLeaves)
    const double k = (double)kd[d];
    const double n = (double)min(nd, nq);
    const double nk = __dsub_rn(n, k);
    const double z0 = __dadd_rn(__dmul_rn(k, L.lp0), __dmul_rn(nk, L.l1p0));
    const double z1 = __dadd_rn(__dmul_rn(k, L.lp1), __dmul_rn(nk, L.l1p1));
    kd[d] = rt_order(__double2float_rn(__dsub_rn(z0, z1)));
  }
  __syncthreads();

  // the need-th smallest key (order << 16 | d) by 8-bit digits, most significant first
  const int need = min(nBest, i);
  unsigned long long kstar = ~0ull;  // every key when need == i
  if (need < i) {
    unsigned long long prefix = 0;
    int rem = need;  // rank (1-based) of the sought key among the keys that start with prefix
    for (int shift = 40; shift >= 0; shift -= 8) {
      for (int t = threadIdx.x; t < 256; t += blockDim.x) hist[t] = 0;
      __syncthreads();
      for (int d = threadIdx.x; d < i; d += blockDim.x) {
        const unsigned long long key = ((unsigned long long)kd[d] << 16) | (uint32_t)d;
        if ((key >> (shift + 8)) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t c[8], s = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          c[q] = hist[lane * 8 + q];
          s += c[q];
        }
        uint32_t inc = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += v;
        }
        const uint32_t exc = inc - s;
        if (exc < (uint32_t)rem && (uint32_t)rem <= inc) {
          uint32_t acc = exc;
          int q = 0;
          while (q < 7 && acc + c[q] < (uint32_t)rem) acc += c[q++];
          shPrefix = (prefix << 8) | (unsigned long long)(lane * 8 + q);
          shRem = rem - (int)acc;
        }
      }
      __syncthreads();
      prefix = shPrefix;
      rem = shRem;
    }
    kstar = prefix;
  }

  // the need smallest keys, then each one's rank among them
  for (int d = threadIdx.x; d < i; d += blockDim.x) {
    const unsigned long long key = ((unsigned long long)kd[d] << 16) | (uint32_t)d;
    if (key <= kstar) cand[atomicAdd(&shCnt, 1)] = key;
  }
  __syncthreads();
  int32_t* docs = bestDocs + (size_t)i * nBest;
  float* scores = bestScores + (size_t)i * nBest;
  for (int c = threadIdx.x; c < need; c += blockDim.x) {
    const unsigned long long key = cand[c];
    int r = 0;
    for (int q = 0; q < need; ++q) r += cand[q] < key;
    docs[r] = (int32_t)(key & 0xffffu);
    scores[r] = rt_unorder((uint32_t)(key >> 16));
  }
  for (int j = need + threadIdx.x; j < nBest; j += blockDim.x) {
    docs[j] = -1;
    scores[j] = 0.0f;
  }
}

struct RtDeviceGuard {
  int prev = -1;
  explicit RtDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~RtDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct v3dm_retrieval {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t* dBits = nullptr;
  size_t bitsCap = 0;  // words
  int32_t* dOffsets = nullptr;
  RtLogs* dLogs = nullptr;
  int imagesCap = 0;
  int32_t* dWords = nullptr;  // host-input calls
  size_t wordsCap = 0;
  int32_t* dDocs = nullptr;
  float* dScores = nullptr;
  size_t bestCap = 0;
  int* dErr = nullptr;
  int* hErr = nullptr;  // pinned
  // pinned staging of offsets and logarithms, two slots used by alternate calls; a slot is
  // rewritten once the copies of the call two back have completed (slotDone)
  RtLogs* hLogs[2] = {nullptr, nullptr};
  int32_t* hOffsets[2] = {nullptr, nullptr};
  cudaEvent_t slotDone[2] = {nullptr, nullptr};
  int slot = 0;
  // CUDA-event timing of the two kernels (v3dm_retrieval_profile): pending event pairs
  bool profile = false;
  std::vector<cudaEvent_t> prof[2];
  double profMs[2] = {0.0, 0.0};
  int profLaunches[2] = {0, 0};
};

namespace {

#define V3DM_RT_TRY(expr)                               \
  do {                                                  \
    cudaError_t e_ = (expr);                            \
    if (e_ != cudaSuccess) {                            \
      record_cuda_error(e_, __FILE__, __LINE__, #expr); \
      return V3DM_ERR_CUDA;                             \
    }                                                   \
  } while (0)

template <class T>
cudaError_t rt_grow(T*& p, size_t& cap, size_t n) {
  if (n <= cap) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) cap = n;
  return e;
}

int rt_check(int nLeaves, int nImages, const int32_t* offsets, double pMatch, int nBest) {
  if (nLeaves < 1 || nImages < 0 || (nImages > 0 && !offsets) || nBest < 1 || nBest > V3DM_RETRIEVAL_MAX_BEST ||
      !(pMatch >= 0.0) || !std::isfinite(pMatch))
    return V3DM_ERR_ARG;
  if (nImages > V3DM_RETRIEVAL_MAX_IMAGES) return V3DM_ERR_SIZE;
  if (((size_t)nLeaves + 1) * (size_t)((nImages + 31) / 32) > 0xffffffffull) return V3DM_ERR_SIZE;  // row offsets
  if (nImages > 0 && offsets[0] != 0) return V3DM_ERR_ARG;
  for (int i = 0; i < nImages; ++i)
    if (offsets[i + 1] < offsets[i]) return V3DM_ERR_ARG;
  return V3DM_OK;
}

// With profiling on, an event on r's stream before / after kernel k (0 = presence, 1 = score).
cudaError_t rt_mark(v3dm_retrieval* r, int k) {
  if (!r->profile) return cudaSuccess;
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreate(&ev);
  if (e != cudaSuccess) return e;
  r->prof[k].push_back(ev);
  return cudaEventRecord(ev, r->stream);
}

// Both kernels on r's stream; words in device memory.  The host computes the logarithms while
// the bitmap is built.
int rt_enqueue(v3dm_retrieval* r, int nLeaves, int nImages, const int32_t* offsets, const int32_t* dWords,
               double pMatch, int nBest, int32_t* dDocs, float* dScores) {
  const int w32 = (nImages + 31) / 32;
  const size_t bitWords = ((size_t)nLeaves + 1) * w32;  // the last row stays zero
  if (bitWords > r->bitsCap || nImages + 1 > r->imagesCap) V3DM_RT_TRY(cudaStreamSynchronize(r->stream));
  V3DM_RT_TRY(rt_grow(r->dBits, r->bitsCap, bitWords));
  if (nImages + 1 > r->imagesCap) {
    cudaFree(r->dOffsets);
    cudaFree(r->dLogs);
    r->dOffsets = nullptr;
    r->dLogs = nullptr;
    for (int k = 0; k < 2; ++k) {
      cudaFreeHost(r->hLogs[k]);
      cudaFreeHost(r->hOffsets[k]);
      r->hLogs[k] = nullptr;
      r->hOffsets[k] = nullptr;
    }
    r->imagesCap = 0;
    const size_t n = (size_t)nImages + 1;
    V3DM_RT_TRY(cudaMalloc(reinterpret_cast<void**>(&r->dOffsets), n * sizeof(int32_t)));
    V3DM_RT_TRY(cudaMalloc(reinterpret_cast<void**>(&r->dLogs), n * sizeof(RtLogs)));
    for (int k = 0; k < 2; ++k) {
      V3DM_RT_TRY(cudaMallocHost(reinterpret_cast<void**>(&r->hLogs[k]), n * sizeof(RtLogs)));
      V3DM_RT_TRY(cudaMallocHost(reinterpret_cast<void**>(&r->hOffsets[k]), n * sizeof(int32_t)));
    }
    r->imagesCap = nImages + 1;
  }
  const int s = r->slot;
  r->slot ^= 1;
  V3DM_RT_TRY(cudaEventSynchronize(r->slotDone[s]));
  RtLogs* hLogs = r->hLogs[s];
  int32_t* hOffsets = r->hOffsets[s];
  std::copy(offsets, offsets + nImages + 1, hOffsets);
  V3DM_RT_TRY(cudaMemcpyAsync(r->dOffsets, hOffsets, (size_t)(nImages + 1) * sizeof(int32_t),
                              cudaMemcpyHostToDevice, r->stream));
  V3DM_RT_TRY(cudaMemsetAsync(r->dBits, 0, bitWords * sizeof(uint32_t), r->stream));
  V3DM_RT_TRY(cudaMemsetAsync(r->dErr, 0, sizeof(int), r->stream));
  V3DM_RT_TRY(rt_mark(r, 0));
  k_rt_presence<<<nImages, kRtPresenceThreads, 0, r->stream>>>(r->dOffsets, dWords, nLeaves, w32, r->dBits, r->dErr);
  V3DM_RT_TRY(cudaGetLastError());
  V3DM_RT_TRY(rt_mark(r, 0));
  // p0 = nFeatures * (1 / nLeaves) and its logarithms, in the expressions of v3d_voctree.h:252-265
  const double normalizer = 1.0 / (double)nLeaves;
  for (int i = 0; i < nImages; ++i) {
    const double p0 = (offsets[i + 1] - offsets[i]) * normalizer;
    const double p1 = std::min(1.0, p0 + pMatch);
    hLogs[i] = RtLogs{std::log(p0), std::log(1.0 - p0), std::log(p1), std::log(1.0 - p1)};
  }
  V3DM_RT_TRY(cudaMemcpyAsync(r->dLogs, hLogs, (size_t)nImages * sizeof(RtLogs), cudaMemcpyHostToDevice, r->stream));
  V3DM_RT_TRY(cudaEventRecord(r->slotDone[s], r->stream));
  const size_t smem = (size_t)nBest * sizeof(unsigned long long) + (size_t)nImages * sizeof(uint32_t);
  V3DM_RT_TRY(cudaFuncSetAttribute(k_rt_score, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  V3DM_RT_TRY(rt_mark(r, 1));
  k_rt_score<<<nImages, kRtThreads, smem, r->stream>>>(r->dOffsets, dWords, nLeaves, nImages, w32, r->dBits, r->dLogs,
                                                       nBest, dDocs, dScores);
  V3DM_RT_TRY(cudaGetLastError());
  V3DM_RT_TRY(rt_mark(r, 1));
  V3DM_RT_TRY(cudaMemcpyAsync(r->hErr, r->dErr, sizeof(int), cudaMemcpyDeviceToHost, r->stream));
  return V3DM_OK;
}

}  // namespace

extern "C" {

int v3dm_retrieval_create(v3dm_retrieval** out, int device) {
  if (!out) return V3DM_ERR_ARG;
  *out = nullptr;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return V3DM_ERR_CUDA;
  if (prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_retrieval* r = new (std::nothrow) v3dm_retrieval();
  if (!r) return V3DM_ERR_ARG;
  r->device = device;
  RtDeviceGuard g(device);
  if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&r->dErr), sizeof(int)) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&r->hErr), sizeof(int)) != cudaSuccess ||
      cudaEventCreateWithFlags(&r->slotDone[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&r->slotDone[1], cudaEventDisableTiming) != cudaSuccess) {
    if (r->slotDone[0]) cudaEventDestroy(r->slotDone[0]);
    if (r->stream) cudaStreamDestroy(r->stream);
    if (r->dErr) cudaFree(r->dErr);
    if (r->hErr) cudaFreeHost(r->hErr);
    delete r;
    return V3DM_ERR_CUDA;
  }
  *r->hErr = 0;
  *out = r;
  return V3DM_OK;
}

int v3dm_retrieval_destroy(v3dm_retrieval* r) {
  if (!r) return V3DM_OK;
  RtDeviceGuard g(r->device);
  cudaStreamSynchronize(r->stream);
  cudaFree(r->dBits);
  cudaFree(r->dOffsets);
  cudaFree(r->dLogs);
  cudaFree(r->dWords);
  cudaFree(r->dDocs);
  cudaFree(r->dScores);
  cudaFree(r->dErr);
  cudaFreeHost(r->hErr);
  for (int k = 0; k < 2; ++k) {
    cudaFreeHost(r->hLogs[k]);
    cudaFreeHost(r->hOffsets[k]);
    cudaEventDestroy(r->slotDone[k]);
    for (cudaEvent_t ev : r->prof[k]) cudaEventDestroy(ev);
  }
  cudaStreamDestroy(r->stream);
  delete r;
  return V3DM_OK;
}

int v3dm_retrieval_stream(v3dm_retrieval* r, void** stream) {
  if (!r || !stream) return V3DM_ERR_ARG;
  *stream = r->stream;
  return V3DM_OK;
}

int v3dm_retrieval_binomial_device(v3dm_retrieval* r, int nLeaves, int nImages, const int32_t* offsets,
                                   const int32_t* d_words, double pMatch, int nBest, int32_t* d_bestDocs,
                                   float* d_bestScores) {
  if (!r) return V3DM_ERR_ARG;
  const int st = rt_check(nLeaves, nImages, offsets, pMatch, nBest);
  if (st != V3DM_OK) return st;
  if (nImages == 0) return V3DM_OK;
  if ((offsets[nImages] > 0 && !d_words) || !d_bestDocs || !d_bestScores) return V3DM_ERR_ARG;
  RtDeviceGuard g(r->device);
  return rt_enqueue(r, nLeaves, nImages, offsets, d_words, pMatch, nBest, d_bestDocs, d_bestScores);
}

int v3dm_retrieval_profile(v3dm_retrieval* r, int enable) {
  if (!r) return V3DM_ERR_ARG;
  r->profile = enable != 0;
  return V3DM_OK;
}

int v3dm_retrieval_profile_read(v3dm_retrieval* r, int kernel, double* msTotal, int* launches) {
  if (!r || kernel < 0 || kernel > 1 || !msTotal || !launches) return V3DM_ERR_ARG;
  RtDeviceGuard g(r->device);
  V3DM_RT_TRY(cudaStreamSynchronize(r->stream));
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

int v3dm_retrieval_wait(v3dm_retrieval* r) {
  if (!r) return V3DM_ERR_ARG;
  RtDeviceGuard g(r->device);
  V3DM_RT_TRY(cudaStreamSynchronize(r->stream));
  const int bad = *r->hErr;
  *r->hErr = 0;
  return bad ? V3DM_ERR_ARG : V3DM_OK;
}

int v3dm_retrieval_binomial(v3dm_retrieval* r, int nLeaves, int nImages, const int32_t* offsets, const int32_t* words,
                            double pMatch, int nBest, int32_t* bestDocs, float* bestScores) {
  if (!r) return V3DM_ERR_ARG;
  int st = rt_check(nLeaves, nImages, offsets, pMatch, nBest);
  if (st != V3DM_OK) return st;
  if (nImages == 0) return V3DM_OK;
  const size_t nWords = (size_t)offsets[nImages];
  if ((nWords > 0 && !words) || !bestDocs || !bestScores) return V3DM_ERR_ARG;
  RtDeviceGuard g(r->device);
  V3DM_RT_TRY(cudaStreamSynchronize(r->stream));
  V3DM_RT_TRY(rt_grow(r->dWords, r->wordsCap, nWords));
  const size_t nOut = (size_t)nImages * nBest;
  if (nOut > r->bestCap) {
    cudaFree(r->dDocs);
    cudaFree(r->dScores);
    r->dDocs = nullptr;
    r->dScores = nullptr;
    r->bestCap = 0;
    V3DM_RT_TRY(cudaMalloc(reinterpret_cast<void**>(&r->dDocs), nOut * sizeof(int32_t)));
    V3DM_RT_TRY(cudaMalloc(reinterpret_cast<void**>(&r->dScores), nOut * sizeof(float)));
    r->bestCap = nOut;
  }
  if (nWords > 0)
    V3DM_RT_TRY(cudaMemcpyAsync(r->dWords, words, nWords * sizeof(int32_t), cudaMemcpyHostToDevice, r->stream));
  st = rt_enqueue(r, nLeaves, nImages, offsets, r->dWords, pMatch, nBest, r->dDocs, r->dScores);
  if (st != V3DM_OK) return st;
  V3DM_RT_TRY(cudaMemcpyAsync(bestDocs, r->dDocs, nOut * sizeof(int32_t), cudaMemcpyDeviceToHost, r->stream));
  V3DM_RT_TRY(cudaMemcpyAsync(bestScores, r->dScores, nOut * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
  return v3dm_retrieval_wait(r);
}

int v3dm_retrieval_pairs(int nImages, int nBest, const int32_t* bestDocs, long long cap, int32_t* pairs,
                         long long* nPairs) {
  if (nImages < 0 || nBest < 1 || (nImages > 0 && !bestDocs) || !nPairs || cap < 0 || (cap > 0 && !pairs))
    return V3DM_ERR_ARG;
  // putativePairwiseMatches (match_using_voctree.cpp:201-216): view1 = the retrieved earlier
  // image, view2 = the query; listed by view1, then view2 (map<int, set<int>> order)
  std::vector<long long> start((size_t)nImages + 1, 0);
  for (int i = 0; i < nImages; ++i)
    for (int j = 0; j < nBest; ++j) {
      const int d = bestDocs[(size_t)i * nBest + j];
      if (d < 0) continue;
      if (d >= i) return V3DM_ERR_ARG;
      ++start[(size_t)d + 1];
    }
  for (int d = 0; d < nImages; ++d) start[(size_t)d + 1] += start[d];
  const long long total = start[(size_t)nImages];
  *nPairs = total;
  if (!pairs) return V3DM_OK;  // count only
  // the queries ascend, so each view1's list fills in view2 order
  for (int i = 0; i < nImages; ++i)
    for (int j = 0; j < nBest; ++j) {
      const int d = bestDocs[(size_t)i * nBest + j];
      if (d < 0) continue;
      const long long at = start[d]++;
      if (at < cap) {
        pairs[2 * at] = d;
        pairs[2 * at + 1] = i;
      }
    }
  return total > cap ? V3DM_ERR_CAPACITY : V3DM_OK;
}

}  // extern "C"
