// v3dm_voctree.cu -- vocabulary-tree quantization (V3D_CUDA::VocabularyTreeTraversal,
// V3D/CUDA/v3d_cudamatching.h:69-105, v3d_cudamatching.cu:700-870).
//
// Tree layout as in the reference: nodeCount x 128 descriptors in breadth-first order
// without the root; level-1 nodes are 0..BF-1 and the children of node i are
// (i+1)*BF .. (i+1)*BF + BF-1 (.cu:784-785).  Each level picks the child with the largest
// dot product, the first child on ties (strict '>', .cu:781).
//
// uint8 nodes and keys (u/512 in the reference's float convention): every dot product is an
// exact integer, so leaf ids match the reference whatever the summation order.
//   - the tensor-core descent (v3dm_voctree_tc.cu) when the shape allows it (BF <= 15, enough
//     keys per bucket): phases of two levels, keys sorted by bucket between phases, each bucket's
//     keys scored against its children and grandchildren with tcgen05 int8 GEMMs;
//   - k_voctree otherwise: one launch, four threads per key (below).
// Float nodes and keys of any value:
//   - k_voctree_f32: float nodes and keys (the apps' trees are float k-means
//     centres of unit-L2 descriptors, v3d_voctree.h:38-52).  The leaf ids equal those of the
//     reference's CPU tree, VocabularyTree::findBestNodeIndex (v3d_voctree.h:82-99), which sums
//     key[i] * node[i] sequentially for i = 0..127 in FP32 (one rounded product and one rounded
//     add per term, no FMA: the reference builds for plain x86-64) and keeps the first child
//     whose score is strictly above the running maximum (initially -1e30f, child -1).
//     A fast pass scores every child with FMA partial sums (four threads per key, coalesced
//     64-byte loads) and bounds its distance to the sequential FP32 sum: both are within
//     gamma_128 * sum|k_i n_i| <= 7.63e-6 * |k| |n| of the exact dot product (the standard bound
//     for recursive summation, n = 128 terms; the FMA pass has at most 34 roundings per term),
//     so |fast - sequential| <= 1.53e-5 * |k| |n|; the kernel uses 2e-5 * |k| |n| + 1e-36 with
//     precomputed node norms rounded up.  When one child's lower bound is above every other
//     child's upper bound (and above -1e30f), it is the sequential rule's choice.  Otherwise
//     (near ties, equal children, non-finite values) one thread of the key replays the
//     reference's sequential FP32 loop over all children, with __fmul_rn / __fadd_rn.
//
// k_voctree: four threads per key, each holding 32 bytes of the key in registers; a warp
// descends eight keys.  At each level a thread loads its 32-byte slice of every child (each
// child row is one 128-byte line read by the four threads together), forms eight dp4a
// partial sums, and the four partials are summed with two butterfly shuffles.  The reference
// instead runs one 32-thread block per key with a racy warp-synchronous shared-memory
// reduction (.cu:770-779).  (Measured on the BF 10, depth 6 tree with 2M keys: 0.95 ms with
// four threads per key, 1.18 ms with eight, 1.53 ms with two, 2.86 ms with one.)
#include <algorithm>
#include <cstring>
#include <new>

#include "v3dm_internal.h"

using namespace v3dm;

namespace {

constexpr int kVtThreads = 256;

constexpr int kTpk = 4;            // threads per key
constexpr int kQ = 8 / kTpk;       // 16-byte words of the key each thread holds

__global__ void __launch_bounds__(kVtThreads)
k_voctree(const uint8_t* __restrict__ nodes, int bf, int depth, long long leafBase, const uint8_t* __restrict__ keys,
          int n, int32_t* __restrict__ out, int idMode) {
  const int gt = blockIdx.x * kVtThreads + threadIdx.x;
  const int key = gt / kTpk;
  const int part = gt % kTpk;
  const bool valid = key < n;
  uint4 kw[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q)
    kw[q] = valid ? reinterpret_cast<const uint4*>(keys + (size_t)key * kDescBytes)[part * kQ + q]
                  : make_uint4(0u, 0u, 0u, 0u);
  long long nextId = 0, leafId = 0;
  for (int d = 0; d < depth; ++d) {
    const uint4* base = reinterpret_cast<const uint4*>(nodes + (size_t)nextId * kDescBytes) + part * kQ;
    int best = 0;
    int bestScore = -1;
#pragma unroll 2
    for (int c = 0; c < bf; ++c) {
      uint32_t acc = 0;
      if (valid) {
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
          const uint4 w = __ldg(base + (size_t)c * (kDescBytes / 16) + q);
          acc = __dp4a(kw[q].x, w.x, acc);
          acc = __dp4a(kw[q].y, w.y, acc);
          acc = __dp4a(kw[q].z, w.z, acc);
          acc = __dp4a(kw[q].w, w.w, acc);
        }
      }
      int sc = (int)acc;
#pragma unroll
      for (int o = 1; o < kTpk; o <<= 1) sc += __shfl_xor_sync(0xffffffffu, sc, o);
      if (sc > bestScore) {  // strict '>': the first child wins ties (.cu:781)
        bestScore = sc;
        best = c;
      }
    }
    leafId = nextId + best;
    nextId = (leafId + 1) * bf;
  }
  if (valid && part == 0) out[key] = (int32_t)(idMode == V3DM_LEAF_LOCAL ? leafId - leafBase : leafId);
}

__global__ void k_vt_f32_to_u8(const float4* __restrict__ src, uint32_t* __restrict__ dst, long long n4, int* err) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n4) return;
  float4 v = src[i];
  float t[4] = {v.x * 512.0f, v.y * 512.0f, v.z * 512.0f, v.w * 512.0f};
  uint32_t w = 0;
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int u = __float2int_rn(t[c]);
    ok = ok && t[c] == (float)u && u >= 0 && u <= 255;
    w |= (uint32_t)(u & 255) << (8 * c);
  }
  dst[i] = w;
  if (!ok) atomicOr(err, 1);
}

// ---- bucketed descent of uint8 trees --------------------------------------------------------
// Phases of two levels (v3dm_voctree_tc.cu): the first phase descends every key from the root,
// each later one the keys of one bucket node at a time, the buckets being the nodes the previous
// phase reached.  Between phases the keys are sorted by bucket (a counting sort: k_vt_scan,
// then k_vt_scatter), and k_vt_scan cuts every bucket into work items of at most kVtItemKeys keys.
constexpr int kVtItemKeys = 2048;       // keys per work item
constexpr int kVtLocalBins = 16384;     // bucket counts kept in shared memory by k_vt_scatter (2 x 64 KB)

// Bucket offsets and the work items of a phase: (bucket, first key in sorted order, count), at
// most kVtItemKeys keys each.  One block.  With bins == 1 and single > 0, one bucket of `single`
// keys (the first phase: no histogram).
__global__ void __launch_bounds__(1024)
k_vt_scan(const int* __restrict__ hist, int bins, int single, int* __restrict__ off, int4* __restrict__ items,
          int* __restrict__ nItems) {
  __shared__ long long sh[1024];
  __shared__ long long shI[1024];
  const int T = blockDim.x, tid = threadIdx.x;
  const int per = (bins + T - 1) / T;
  const int b0 = min(bins, tid * per), b1 = min(bins, b0 + per);
  auto cnt = [&](int b) { return single > 0 ? single : hist[b]; };
  long long sk = 0, si = 0;
  for (int b = b0; b < b1; ++b) {
    sk += cnt(b);
    si += (cnt(b) + kVtItemKeys - 1) / kVtItemKeys;
  }
  sh[tid] = sk;
  shI[tid] = si;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    const long long v = tid >= o ? sh[tid - o] : 0, w = tid >= o ? shI[tid - o] : 0;
    __syncthreads();
    sh[tid] += v;
    shI[tid] += w;
    __syncthreads();
  }
  long long k = sh[tid] - sk, it = shI[tid] - si;
  for (int b = b0; b < b1; ++b) {
    const int c = cnt(b);
    off[b] = (int)k;
    for (int j = 0; j < c; j += kVtItemKeys) items[it++] = make_int4(b, (int)k + j, min(kVtItemKeys, c - j), 0);
    k += c;
  }
  if (tid == T - 1) {
    off[bins] = (int)sh[T - 1];
    *nItems = (int)shI[T - 1];
  }
}

// Keys in bucket order.  Each CTA takes a contiguous range of keys, counts them per bucket in
// shared memory, reserves its slots of every bucket with one global atomic per bucket, and
// places its keys with shared-memory ranks (the order within a bucket does not matter).
constexpr int kVtScatterThreads = 1024;
__global__ void __launch_bounds__(kVtScatterThreads)
k_vt_scatter(const int32_t* __restrict__ bucket, int n, const int* __restrict__ off, int* __restrict__ cursor,
             int32_t* __restrict__ perm, int bins) {
  extern __shared__ int vtScatterSmem[];  // 2 x bins when bins <= kVtLocalBins
  int* cnt = vtScatterSmem;
  int* base = vtScatterSmem + bins;
  const long long per = ((long long)n + gridDim.x - 1) / gridDim.x;
  const int k0 = (int)min((long long)n, per * blockIdx.x), k1 = (int)min((long long)n, per * (blockIdx.x + 1));
  if (bins > kVtLocalBins) {  // too many buckets for shared memory: one global atomic per key
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const int b = bucket[k];
      perm[off[b] + atomicAdd(&cursor[b], 1)] = k;
    }
    return;
  }
  for (int b = threadIdx.x; b < bins; b += blockDim.x) cnt[b] = 0;
  __syncthreads();
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) atomicAdd(&cnt[bucket[k]], 1);
  __syncthreads();
  for (int b = threadIdx.x; b < bins; b += blockDim.x) {
    base[b] = cnt[b] ? off[b] + atomicAdd(&cursor[b], cnt[b]) : 0;
    cnt[b] = 0;
  }
  __syncthreads();
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const int b = bucket[k];
    perm[base[b] + atomicAdd(&cnt[b], 1)] = k;
  }
}

// Bound of |FMA-pass score - sequential FP32 score| relative to |key| |node| (2 gamma_128 =
// 1.53e-5, with margin for the rounding of the norms), and an absolute term for underflow.
constexpr float kSeqRel = 2.0e-5f;
constexpr float kSeqAbs = 1.0e-36f;

// The reference's sequential FP32 scan over the children of one node (v3d_voctree.h:82-99).
__device__ __forceinline__ int seq_best_child(const float* __restrict__ key, const float* __restrict__ base, int bf) {
  int bestNode = -1;
  float maxScore = -1e30f;
#pragma unroll 1
  for (int k = 0; k < bf; ++k) {
    const float* cur = base + (size_t)k * kDescBytes;
    float score = 0.0f;
#pragma unroll 4
    for (int i = 0; i < kDescBytes; ++i) score = __fadd_rn(score, __fmul_rn(__ldg(key + i), __ldg(cur + i)));
    if (score > maxScore) {
      bestNode = k;
      maxScore = score;
    }
  }
  return bestNode;
}

// Float descent.  Four threads per key; thread `part` holds key floats q*16 + part*4 .. +3 for
// q = 0..7, so the four threads of a key read 64 contiguous bytes of a node row per load.
// nodeNorm[i] >= |node i| (L2).  exactCount (optional) counts the key-levels resolved by the
// sequential replay.  err gets kErrBadTree when a child block would leave the tree.
__global__ void __launch_bounds__(kVtThreads, 2)
k_voctree_f32(const float* __restrict__ nodes, const float* __restrict__ nodeNorm, long long nodeCount, int bf,
              int depth, long long leafBase, const float* __restrict__ keys, int n, int32_t* __restrict__ out,
              int idMode, unsigned long long* __restrict__ exactCount, int32_t* __restrict__ err) {
  const int gt = blockIdx.x * kVtThreads + threadIdx.x;
  const int key = gt / kTpk;
  const int part = gt % kTpk;
  const int lane = threadIdx.x & 31;
  const unsigned grp = 0xfu << (lane & ~3);
  const bool valid = key < n;
  const float* krow = keys + (size_t)(valid ? key : 0) * kDescBytes;
  float4 kv[8];
#pragma unroll
  for (int q = 0; q < 8; ++q)
    kv[q] = valid ? __ldg(reinterpret_cast<const float4*>(krow) + q * 4 + part) : make_float4(0.f, 0.f, 0.f, 0.f);
  float ss = 0.0f;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    ss = fmaf(kv[q].x, kv[q].x, ss);
    ss = fmaf(kv[q].y, kv[q].y, ss);
    ss = fmaf(kv[q].z, kv[q].z, ss);
    ss = fmaf(kv[q].w, kv[q].w, ss);
  }
  ss += __shfl_xor_sync(0xffffffffu, ss, 1);
  ss += __shfl_xor_sync(0xffffffffu, ss, 2);
  const float kn = __fmul_ru(__fsqrt_ru(ss), 1.000001f);
  long long nextId = 0, leafId = 0;
  unsigned long long replays = 0;
  bool ok = true;
  for (int d = 0; d < depth; ++d) {
    if (nextId < 0 || nextId + bf > nodeCount) {  // cannot happen for a finite tree; leaves the loop safely
      ok = false;
      break;
    }
    const float* base = nodes + (size_t)nextId * kDescBytes;
    float lo1 = -INFINITY, up1 = -INFINITY, up2 = -INFINITY;
    int c1 = -1, cu1 = -1;
    bool finite = true;
#pragma unroll 2
    for (int c = 0; c < bf; ++c) {
      const float4* row = reinterpret_cast<const float4*>(base + (size_t)c * kDescBytes) + part;
      float acc = 0.0f;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float4 w = __ldg(row + q * 4);
        acc = fmaf(kv[q].x, w.x, acc);
        acc = fmaf(kv[q].y, w.y, acc);
        acc = fmaf(kv[q].z, w.z, acc);
        acc = fmaf(kv[q].w, w.w, acc);
      }
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);  // fadd commutes: the four lanes agree exactly
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      const float e = __fadd_ru(__fmul_ru(__fmul_ru(kSeqRel, kn), __ldg(nodeNorm + nextId + c)), kSeqAbs);
      const float lo = __fsub_rd(acc, e), up = __fadd_ru(acc, e);
      finite = finite && isfinite(lo) && isfinite(up);
      if (lo > lo1) {
        lo1 = lo;
        c1 = c;
      }
      if (up > up1) {
        up2 = up1;
        up1 = up;
        cu1 = c;
      } else if (up > up2) {
        up2 = up;
      }
    }
    const float othersUp = cu1 == c1 ? up2 : up1;
    int best = c1;
    // the same on the four lanes of the key: their scores and bounds are bit-identical
    if (!(finite && c1 >= 0 && othersUp < lo1 && lo1 > -1e30f)) {
      int b = -1;
      if (part == 0 && valid) {
        b = seq_best_child(krow, base, bf);
        ++replays;
      }
      best = __shfl_sync(grp, b, lane & ~3);
    }
    if (!valid) best = 0;
    leafId = nextId + best;
    nextId = (leafId + 1) * bf;
  }
  if (!ok && part == 0 && valid) atomicOr(err, kErrBadTree);
  if (valid && part == 0) out[key] = (int32_t)(idMode == V3DM_LEAF_LOCAL ? leafId - leafBase : leafId);
  if (exactCount && part == 0 && replays) atomicAdd(exactCount, replays);
}

// |node i| rounded up, for the bound above (double sum, then an upward margin).
__global__ void k_node_norms(const float* __restrict__ nodes, long long nodeCount, float* __restrict__ norm) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nodeCount) return;
  const float4* r = reinterpret_cast<const float4*>(nodes + (size_t)i * kDescBytes);
  double s = 0.0;
  for (int q = 0; q < kDescBytes / 4; ++q) {
    const float4 v = r[q];
    s += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
  }
  norm[i] = __double2float_ru(sqrt(s) * (1.0 + 1e-12));
}

// u8 -> float (u/512), for float keys against a tree given as bytes.
__global__ void k_u8_to_f32(const uchar4* __restrict__ src, float4* __restrict__ dst, long long n4) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const uchar4 u = src[i];
  dst[i] = make_float4(u.x / 512.0f, u.y / 512.0f, u.z / 512.0f, u.w / 512.0f);
}

bool tree_counts(int bf, int depth, long long* nodes, long long* leaves, long long* leafBase) {
  if (bf < 1 || depth < 1) return false;
  long long total = 0, len = 1, base = 0;
  for (int d = 0; d < depth; ++d) {
    if (d == depth - 1) base = total;
    len *= bf;
    total += len;
    if (total > (1LL << 31) / kDescBytes * 64) return false;  // keeps node offsets and ids in range
  }
  *nodes = total;
  *leaves = len;
  *leafBase = base;
  return true;
}

struct DeviceGuardVt {
  int prev = -1;
  explicit DeviceGuardVt(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuardVt() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct v3dm_voctree {
  int device = 0;
  int bf = 0, depth = 0;
  long long nodeCount = 0, leafCount = 0, leafBase = 0;
  cudaStream_t stream = nullptr;
  uint8_t* dNodes = nullptr;    // u8 tree (valid when nodesU8)
  float* dNodesF = nullptr;     // float tree (valid when nodesF)
  float* dNorm = nullptr;       // |node i| rounded up (valid when nodesF)
  bool nodesU8 = false;         // the tree's values are all u/512, u in 0..255
  bool nodesF = false;
  int nMax = 0;
  uint8_t* dKeys = nullptr;
  float* dStage = nullptr;
  int32_t* dIds = nullptr;
  int32_t* dErr = nullptr;
  int32_t* hErr = nullptr;
  unsigned long long* dReplays = nullptr;  // key-levels resolved by the sequential replay
  // tensor-core descent of u8 trees in phases of two levels (tcPath false: one-kernel descent)
  bool tcPath = false;
  int phases = 0;
  long long maxBins = 1;        // buckets of the last phase
  int32_t* dBucket = nullptr;   // nMax: per key, the bucket it reached
  int32_t* dPerm = nullptr;     // nMax: keys in bucket order
  int* dHist = nullptr;         // maxBins counts, then maxBins cursors
  int* dOff = nullptr;          // maxBins + 1
  int4* dItems = nullptr;       // nMax / kVtItemKeys + maxBins + 1
  int* dNItems = nullptr;
  int numSMs = 148;
  int lastLaunches = 0;         // kernels launched by the last quantization
  CUtensorMap tmNodes;          // the u8 node rows for the tensor path's TMA loads
  bool tmValid = false;
  CUtensorMap tmKeys;           // the keys of the last call (first phase), for TMA tiles
  const uint8_t* tmKeysPtr = nullptr;
  int tmKeysRows = 0;
};

namespace {

// First global index of the nodes at depth d (1-based; the root has none).
long long level_start(int bf, int d) {
  long long start = 0, len = 1;
  for (int k = 1; k < d; ++k) {
    len *= bf;
    start += len;
  }
  return start;
}

// Phases of the tensor-core descent: ceil(depth / 2), the last one's buckets are the nodes at
// depth 2 (phases - 1).
void vt_plan(v3dm_voctree* t) {
  t->phases = (t->depth + 1) / 2;
  long long bins = 1;
  for (int k = 0; k < 2 * (t->phases - 1); ++k) bins *= t->bf;
  t->maxBins = bins;
  t->tcPath = vtc_supported(t->bf) && bins <= (1LL << 22);
}

int vt_launch(v3dm_voctree* t, int n, const uint8_t* dKeys, int32_t* dIds, int idMode) {
  t->lastLaunches = 0;
  if (n == 0) return V3DM_OK;
  // the tensor path needs its buffers and enough keys per bucket of the last phase to fill
  // 128-key tiles; otherwise the one-kernel descent
  if (t->tcPath && !t->tmValid && t->dNodes &&
      tc_rows_map(&t->tmNodes, t->dNodes, (int)t->nodeCount, kVtcBoxRows) == cudaSuccess)
    t->tmValid = true;
  if (!t->tcPath || !t->tmValid || !t->dPerm || n > t->nMax || (long long)n < 16 * t->maxBins) {
    long long threads = (long long)n * kTpk;
    unsigned blocks = (unsigned)((threads + kVtThreads - 1) / kVtThreads);
    k_voctree<<<blocks, kVtThreads, 0, t->stream>>>(t->dNodes, t->bf, t->depth, t->leafBase, dKeys, n, dIds, idMode);
    t->lastLaunches = 1;
    return cudaGetLastError() == cudaSuccess ? V3DM_OK : V3DM_ERR_CUDA;
  }
  if (t->tmKeysPtr != dKeys || t->tmKeysRows != n) {
    t->tmKeysPtr = nullptr;
    if (tc_rows_map(&t->tmKeys, dKeys, n, kVtcKeyBox) == cudaSuccess) {
      t->tmKeysPtr = dKeys;
      t->tmKeysRows = n;
    }
  }
  if (t->tmKeysPtr != dKeys) {  // keys a tensor map cannot describe (not 16-byte aligned)
    long long threads = (long long)n * kTpk;
    unsigned blocks = (unsigned)((threads + kVtThreads - 1) / kVtThreads);
    k_voctree<<<blocks, kVtThreads, 0, t->stream>>>(t->dNodes, t->bf, t->depth, t->leafBase, dKeys, n, dIds, idMode);
    t->lastLaunches = 1;
    return cudaGetLastError() == cudaSuccess ? V3DM_OK : V3DM_ERR_CUDA;
  }
  const int bf = t->bf;
  VtcArgs va;
  std::memset(&va, 0, sizeof(va));
  va.nodes = t->dNodes;
  va.bf = bf;
  va.items = t->dItems;
  va.nItems = t->dNItems;
  va.keys = dKeys;
  va.out = dIds;
  va.idMode = idMode;
  va.leafBase = t->leafBase;
  va.next = t->dBucket;
  va.hist = t->dHist;
  va.err = t->dErr;
  long long bins = 1;
  for (int p = 0; p < t->phases; ++p) {
    const int levels = std::min(2, t->depth - 2 * p);
    const bool last = p == t->phases - 1;
    const long long nextBins = bins * bf * bf;
    if (p > 0) {
      // keys sorted by the bucket the previous phase reached
      k_vt_scan<<<1, 1024, 0, t->stream>>>(t->dHist, (int)bins, 0, t->dOff, t->dItems, t->dNItems);
      if (cudaGetLastError() != cudaSuccess) return V3DM_ERR_CUDA;
      if (cudaMemsetAsync(t->dHist + t->maxBins, 0, (size_t)bins * sizeof(int), t->stream) != cudaSuccess)
        return V3DM_ERR_CUDA;
      const unsigned sg = (unsigned)std::max<long long>(
          1, std::min<long long>(((long long)n + 4095) / 4096, (long long)t->numSMs * 2));
      const size_t ssm = bins <= kVtLocalBins ? 2 * (size_t)bins * sizeof(int) : 0;
      k_vt_scatter<<<sg, kVtScatterThreads, ssm, t->stream>>>(t->dBucket, n, t->dOff, t->dHist + t->maxBins, t->dPerm,
                                                              (int)bins);
      if (cudaGetLastError() != cudaSuccess) return V3DM_ERR_CUDA;
    }
    if (!last && cudaMemsetAsync(t->dHist, 0, (size_t)nextBins * sizeof(int), t->stream) != cudaSuccess)
      return V3DM_ERR_CUDA;
    va.levels = levels;
    va.singleN = p == 0 ? n : 0;  // the first phase: one bucket (the root), items implied
    va.bucketBase = p == 0 ? -1 : level_start(bf, 2 * p);
    va.perm = p == 0 ? nullptr : t->dPerm;
    va.final = last ? 1 : 0;
    va.nextBase = last ? 0 : level_start(bf, 2 * p + 2);
    va.bins = last ? 0 : (int)nextBins;
    if (launch_vtc(va, t->tmNodes, t->tmKeys, t->numSMs, t->stream) != cudaSuccess) return V3DM_ERR_CUDA;
    t->lastLaunches += p == 0 ? 1 : 3;  // scan and scatter (after the first phase), the phase
    bins = nextBins;
  }
  return V3DM_OK;
}

int vt_launch_f32(v3dm_voctree* t, int n, const float* dKeys, int32_t* dIds, int idMode) {
  t->lastLaunches = 0;
  if (n == 0) return V3DM_OK;
  t->lastLaunches = 1;
  long long threads = (long long)n * kTpk;
  unsigned blocks = (unsigned)((threads + kVtThreads - 1) / kVtThreads);
  k_voctree_f32<<<blocks, kVtThreads, 0, t->stream>>>(t->dNodesF, t->dNorm, t->nodeCount, t->bf, t->depth,
                                                      t->leafBase, dKeys, n, dIds, idMode, t->dReplays, t->dErr);
  return cudaGetLastError() == cudaSuccess ? V3DM_OK : V3DM_ERR_CUDA;
}

// floats on the device -> u8 (u = 512 x); *exact = every value was u/512 with u in 0..255.
int vt_to_u8(v3dm_voctree* t, const float* dSrc, size_t count, uint8_t* dst, bool* exact) {
  *exact = true;
  if (count == 0) return V3DM_OK;
  if (cudaMemsetAsync(t->dErr, 0, sizeof(int32_t), t->stream) != cudaSuccess) return V3DM_ERR_CUDA;
  long long n4 = (long long)(count / 4);
  k_vt_f32_to_u8<<<(unsigned)((n4 + 255) / 256), 256, 0, t->stream>>>(reinterpret_cast<const float4*>(dSrc),
                                                                      reinterpret_cast<uint32_t*>(dst), n4, t->dErr);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(t->hErr, t->dErr, sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  *exact = *t->hErr == 0;
  return V3DM_OK;
}

// Node norms of the float tree.
int vt_norms(v3dm_voctree* t) {
  if (!t->dNorm && cudaMalloc(reinterpret_cast<void**>(&t->dNorm), (size_t)t->nodeCount * sizeof(float)) != cudaSuccess)
    return V3DM_ERR_CUDA;
  k_node_norms<<<(unsigned)((t->nodeCount + 255) / 256), 256, 0, t->stream>>>(t->dNodesF, t->nodeCount, t->dNorm);
  return cudaGetLastError() == cudaSuccess ? V3DM_OK : V3DM_ERR_CUDA;
}

int vt_alloc_float_tree(v3dm_voctree* t) {
  if (!t->dNodesF &&
      cudaMalloc(reinterpret_cast<void**>(&t->dNodesF), (size_t)t->nodeCount * kDescBytes * sizeof(float)) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return V3DM_OK;
}

// The float tree from the u8 one (u/512), when float keys meet a tree given as bytes.
int vt_ensure_float_tree(v3dm_voctree* t) {
  if (t->nodesF) return V3DM_OK;
  if (!t->nodesU8) return V3DM_ERR_NOT_ALLOCATED;
  int st = vt_alloc_float_tree(t);
  if (st != V3DM_OK) return st;
  const long long n4 = t->nodeCount * kDescBytes / 4;
  k_u8_to_f32<<<(unsigned)((n4 + 255) / 256), 256, 0, t->stream>>>(reinterpret_cast<const uchar4*>(t->dNodes),
                                                                  reinterpret_cast<float4*>(t->dNodesF), n4);
  if (cudaGetLastError() != cudaSuccess) return V3DM_ERR_CUDA;
  st = vt_norms(t);
  if (st != V3DM_OK) return st;
  t->nodesF = true;
  return V3DM_OK;
}

int vt_check_err(v3dm_voctree* t) {
  if (cudaMemcpyAsync(t->hErr, t->dErr, sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  if (*t->hErr & kErrBadTree) {
    cudaMemsetAsync(t->dErr, 0, sizeof(int32_t), t->stream);
    return V3DM_ERR_ARG;
  }
  return V3DM_OK;
}

}  // namespace

extern "C" {

int v3dm_voctree_counts(int bf, int depth, int64_t* nodeCount, int64_t* leafCount) {
  long long nc, lc, lb;
  if (!tree_counts(bf, depth, &nc, &lc, &lb)) return V3DM_ERR_ARG;
  if (nodeCount) *nodeCount = nc;
  if (leafCount) *leafCount = lc;
  return V3DM_OK;
}

int v3dm_voctree_create(v3dm_voctree** out, int device, int bf, int depth) {
  if (!out) return V3DM_ERR_ARG;
  *out = nullptr;
  long long nc, lc, lb;
  if (!tree_counts(bf, depth, &nc, &lc, &lb)) return V3DM_ERR_ARG;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return V3DM_ERR_CUDA;
  if (prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_voctree* t = new (std::nothrow) v3dm_voctree();
  if (!t) return V3DM_ERR_ARG;
  t->device = device;
  t->bf = bf;
  t->depth = depth;
  t->nodeCount = nc;
  t->leafCount = lc;
  t->leafBase = lb;
  t->numSMs = prop.multiProcessorCount;
  vt_plan(t);
  DeviceGuardVt g(device);
  if (cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dErr), sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&t->hErr), sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dReplays), sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemsetAsync(t->dErr, 0, sizeof(int32_t), t->stream) != cudaSuccess ||
      cudaMemsetAsync(t->dReplays, 0, sizeof(unsigned long long), t->stream) != cudaSuccess ||
      (t->tcPath &&
       (cudaMalloc(reinterpret_cast<void**>(&t->dHist), 2 * (size_t)t->maxBins * sizeof(int)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&t->dOff), ((size_t)t->maxBins + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&t->dNItems), sizeof(int)) != cudaSuccess ||
        cudaFuncSetAttribute(k_vt_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kVtLocalBins * (int)sizeof(int)) != cudaSuccess)) ||
      cudaStreamSynchronize(t->stream) != cudaSuccess) {
    if (t->stream) cudaStreamDestroy(t->stream);
    if (t->dErr) cudaFree(t->dErr);
    if (t->hErr) cudaFreeHost(t->hErr);
    if (t->dReplays) cudaFree(t->dReplays);
    if (t->dHist) cudaFree(t->dHist);
    if (t->dOff) cudaFree(t->dOff);
    if (t->dNItems) cudaFree(t->dNItems);
    delete t;
    return V3DM_ERR_CUDA;
  }
  *out = t;
  return V3DM_OK;
}

int v3dm_voctree_destroy(v3dm_voctree* t) {
  if (!t) return V3DM_ERR_ARG;
  DeviceGuardVt g(t->device);
  cudaStreamSynchronize(t->stream);
  if (t->dNodes) cudaFree(t->dNodes);
  if (t->dNodesF) cudaFree(t->dNodesF);
  if (t->dNorm) cudaFree(t->dNorm);
  if (t->dReplays) cudaFree(t->dReplays);
  if (t->dHist) cudaFree(t->dHist);
  if (t->dOff) cudaFree(t->dOff);
  if (t->dNItems) cudaFree(t->dNItems);
  if (t->dBucket) cudaFree(t->dBucket);
  if (t->dPerm) cudaFree(t->dPerm);
  if (t->dItems) cudaFree(t->dItems);
  if (t->dKeys) cudaFree(t->dKeys);
  if (t->dStage) cudaFree(t->dStage);
  if (t->dIds) cudaFree(t->dIds);
  if (t->dErr) cudaFree(t->dErr);
  if (t->hErr) cudaFreeHost(t->hErr);
  cudaStreamDestroy(t->stream);
  delete t;
  return V3DM_OK;
}

int v3dm_voctree_allocate(v3dm_voctree* t, int nMax) {
  if (!t || nMax < 0) return V3DM_ERR_ARG;
  DeviceGuardVt g(t->device);
  cudaStreamSynchronize(t->stream);
  if (t->dKeys) cudaFree(t->dKeys);
  if (t->dStage) cudaFree(t->dStage);
  if (t->dIds) cudaFree(t->dIds);
  if (t->dBucket) cudaFree(t->dBucket);
  if (t->dPerm) cudaFree(t->dPerm);
  if (t->dItems) cudaFree(t->dItems);
  t->dKeys = nullptr;
  t->dStage = nullptr;
  t->dIds = nullptr;
  t->dBucket = t->dPerm = nullptr;
  t->dItems = nullptr;
  t->nMax = 0;
  size_t m = nMax > 0 ? (size_t)nMax : 1;
  if (cudaMalloc(reinterpret_cast<void**>(&t->dKeys), m * kDescBytes) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dStage), m * kDescBytes * sizeof(float)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dIds), m * sizeof(int32_t)) != cudaSuccess)
    return V3DM_ERR_CUDA;
  if (t->tcPath &&
      (cudaMalloc(reinterpret_cast<void**>(&t->dBucket), m * sizeof(int32_t)) != cudaSuccess ||
       cudaMalloc(reinterpret_cast<void**>(&t->dPerm), m * sizeof(int32_t)) != cudaSuccess ||
       cudaMalloc(reinterpret_cast<void**>(&t->dItems), (m / kVtItemKeys + t->maxBins + 1) * sizeof(int4)) !=
           cudaSuccess))
    return V3DM_ERR_CUDA;
  t->nMax = nMax;
  return V3DM_OK;
}

int v3dm_voctree_set_nodes_u8(v3dm_voctree* t, const uint8_t* nodes) {
  if (!t || !nodes) return V3DM_ERR_ARG;
  DeviceGuardVt g(t->device);
  if (!t->dNodes && cudaMalloc(reinterpret_cast<void**>(&t->dNodes), (size_t)t->nodeCount * kDescBytes) != cudaSuccess)
    return V3DM_ERR_CUDA;
  t->nodesU8 = t->nodesF = false;
  if (cudaMemcpyAsync(t->dNodes, nodes, (size_t)t->nodeCount * kDescBytes, cudaMemcpyHostToDevice, t->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  t->nodesU8 = true;
  return V3DM_OK;
}

int v3dm_voctree_set_nodes_f32(v3dm_voctree* t, const float* nodes) {
  if (!t || !nodes) return V3DM_ERR_ARG;
  DeviceGuardVt g(t->device);
  t->nodesU8 = t->nodesF = false;
  int st = vt_alloc_float_tree(t);
  if (st != V3DM_OK) return st;
  if (!t->dNodes && cudaMalloc(reinterpret_cast<void**>(&t->dNodes), (size_t)t->nodeCount * kDescBytes) != cudaSuccess)
    return V3DM_ERR_CUDA;
  const size_t count = (size_t)t->nodeCount * kDescBytes;
  if (cudaMemcpyAsync(t->dNodesF, nodes, count * sizeof(float), cudaMemcpyHostToDevice, t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  st = vt_norms(t);
  if (st != V3DM_OK) return st;
  bool exact = false;
  st = vt_to_u8(t, t->dNodesF, count, t->dNodes, &exact);  // synchronises
  if (st != V3DM_OK) return st;
  t->nodesF = true;
  t->nodesU8 = exact;  // u/512 trees also keep the faster integer descent
  return V3DM_OK;
}

int v3dm_voctree_quantize_u8(v3dm_voctree* t, int n, const uint8_t* keys, int32_t* ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!keys || !ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (!(t->nodesU8 || t->nodesF) || !t->dKeys) return V3DM_ERR_NOT_ALLOCATED;
  if (n > t->nMax) return V3DM_ERR_SIZE;
  if (n == 0) return V3DM_OK;
  DeviceGuardVt g(t->device);
  if (cudaMemcpyAsync(t->dKeys, keys, (size_t)n * kDescBytes, cudaMemcpyHostToDevice, t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  int st;
  if (t->nodesU8) {
    st = vt_launch(t, n, t->dKeys, t->dIds, idMode);
  } else {  // float tree: the keys as u/512 floats through the float descent
    const long long n4 = (long long)n * kDescBytes / 4;
    k_u8_to_f32<<<(unsigned)((n4 + 255) / 256), 256, 0, t->stream>>>(reinterpret_cast<const uchar4*>(t->dKeys),
                                                                    reinterpret_cast<float4*>(t->dStage), n4);
    st = cudaGetLastError() == cudaSuccess ? vt_launch_f32(t, n, t->dStage, t->dIds, idMode) : V3DM_ERR_CUDA;
  }
  if (st != V3DM_OK) return st;
  if (cudaMemcpyAsync(ids, t->dIds, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return vt_check_err(t);
}

int v3dm_voctree_quantize_f32(v3dm_voctree* t, int n, const float* keys, int32_t* ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!keys || !ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (!(t->nodesU8 || t->nodesF) || !t->dKeys) return V3DM_ERR_NOT_ALLOCATED;
  if (n > t->nMax) return V3DM_ERR_SIZE;
  if (n == 0) return V3DM_OK;
  DeviceGuardVt g(t->device);
  const size_t count = (size_t)n * kDescBytes;
  if (cudaMemcpyAsync(t->dStage, keys, count * sizeof(float), cudaMemcpyHostToDevice, t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  bool exact = false;
  int st = V3DM_OK;
  if (t->nodesU8) {
    st = vt_to_u8(t, t->dStage, count, t->dKeys, &exact);
    if (st != V3DM_OK) return st;
  }
  if (exact) {  // u/512 keys on a u/512 tree: every dot product is exact, the integer descent gives the same ids
    st = vt_launch(t, n, t->dKeys, t->dIds, idMode);
  } else {
    st = vt_ensure_float_tree(t);
    if (st == V3DM_OK) st = vt_launch_f32(t, n, t->dStage, t->dIds, idMode);
  }
  if (st != V3DM_OK) return st;
  if (cudaMemcpyAsync(ids, t->dIds, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return vt_check_err(t);
}

// Device buffers of the quantize calls: keys read as 16-byte vectors, ids written as int32.
bool vt_aligned(const void* keys, const void* ids) { return dev_aligned(keys, 16) && dev_aligned(ids, 4); }

int v3dm_voctree_quantize_u8_device(v3dm_voctree* t, int n, const uint8_t* d_keys, int32_t* d_ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!d_keys || !d_ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (n > 0 && !vt_aligned(d_keys, d_ids)) return V3DM_ERR_ARG;
  if (!t->nodesU8) return t->nodesF ? V3DM_ERR_NOT_U8 : V3DM_ERR_NOT_ALLOCATED;
  DeviceGuardVt g(t->device);
  return vt_launch(t, n, d_keys, d_ids, idMode);
}

int v3dm_voctree_quantize_f32_device(v3dm_voctree* t, int n, const float* d_keys, int32_t* d_ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!d_keys || !d_ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (n > 0 && !vt_aligned(d_keys, d_ids)) return V3DM_ERR_ARG;
  if (!(t->nodesU8 || t->nodesF)) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuardVt g(t->device);
  int st = vt_ensure_float_tree(t);
  if (st != V3DM_OK) return st;
  return vt_launch_f32(t, n, d_keys, d_ids, idMode);
}

int v3dm_voctree_replays(v3dm_voctree* t, long long* n) {
  if (!t || !n) return V3DM_ERR_ARG;
  DeviceGuardVt g(t->device);
  unsigned long long v = 0;
  if (cudaMemcpyAsync(&v, t->dReplays, sizeof(v), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  *n = (long long)v;
  return V3DM_OK;
}

int v3dm_voctree_last_launches(v3dm_voctree* t, int* n) {
  if (!t || !n) return V3DM_ERR_ARG;
  *n = t->lastLaunches;
  return V3DM_OK;
}

int v3dm_voctree_stream(v3dm_voctree* t, void** s) {
  if (!t || !s) return V3DM_ERR_ARG;
  *s = (void*)t->stream;
  return V3DM_OK;
}

}  // extern "C"
