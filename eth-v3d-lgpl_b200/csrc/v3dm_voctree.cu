// v3dm_voctree.cu -- vocabulary-tree quantization (V3D_CUDA::VocabularyTreeTraversal,
// V3D/CUDA/v3d_cudamatching.h:69-105, v3d_cudamatching.cu:700-870).
//
// Tree layout as in the reference: nodeCount x 128 descriptors in breadth-first order
// without the root; level-1 nodes are 0..BF-1 and the children of node i are
// (i+1)*BF .. (i+1)*BF + BF-1 (.cu:784-785).  Each level picks the child with the largest
// dot product, the first child on ties (strict '>', .cu:781).  Nodes and keys are uint8
// (u/512 in the reference's float convention), so every dot product is an exact integer
// and leaf ids match the reference whatever the summation order.
//
// Kernel: four threads per key, each holding 32 bytes of the key in registers; a warp
// descends eight keys.  At each level a thread loads its 32-byte slice of every child (each
// child row is one 128-byte line read by the four threads together), forms eight dp4a
// partial sums, and the four partials are summed with two butterfly shuffles.  The reference
// instead runs one 32-thread block per key with a racy warp-synchronous shared-memory
// reduction (.cu:770-779).  (Measured on the BF 10, depth 6 tree with 2M keys: 0.95 ms with
// four threads per key, 1.18 ms with eight, 1.53 ms with two, 2.86 ms with one.)
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
  uint8_t* dNodes = nullptr;
  int nMax = 0;
  uint8_t* dKeys = nullptr;
  float* dStage = nullptr;
  int32_t* dIds = nullptr;
  int32_t* dErr = nullptr;
  int32_t* hErr = nullptr;
};

namespace {

int vt_launch(v3dm_voctree* t, int n, const uint8_t* dKeys, int32_t* dIds, int idMode) {
  if (n == 0) return V3DM_OK;
  long long threads = (long long)n * kTpk;
  unsigned blocks = (unsigned)((threads + kVtThreads - 1) / kVtThreads);
  k_voctree<<<blocks, kVtThreads, 0, t->stream>>>(t->dNodes, t->bf, t->depth, t->leafBase, dKeys, n, dIds, idMode);
  return cudaGetLastError() == cudaSuccess ? V3DM_OK : V3DM_ERR_CUDA;
}

int vt_convert(v3dm_voctree* t, const float* host, size_t count, uint8_t* dst) {
  if (count == 0) return V3DM_OK;
  if (cudaMemsetAsync(t->dErr, 0, sizeof(int32_t), t->stream) != cudaSuccess) return V3DM_ERR_CUDA;
  // stage through dStage in chunks of its capacity (nMax descriptors)
  size_t cap = (size_t)(t->nMax > 0 ? t->nMax : 1) * kDescBytes;
  for (size_t off = 0; off < count; off += cap) {
    size_t c = count - off < cap ? count - off : cap;
    if (cudaMemcpyAsync(t->dStage, host + off, c * sizeof(float), cudaMemcpyHostToDevice, t->stream) != cudaSuccess)
      return V3DM_ERR_CUDA;
    long long n4 = (long long)(c / 4);
    k_vt_f32_to_u8<<<(unsigned)((n4 + 255) / 256), 256, 0, t->stream>>>(
        reinterpret_cast<const float4*>(t->dStage), reinterpret_cast<uint32_t*>(dst + off), n4, t->dErr);
    if (cudaGetLastError() != cudaSuccess) return V3DM_ERR_CUDA;
  }
  if (cudaMemcpyAsync(t->hErr, t->dErr, sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return *t->hErr ? V3DM_ERR_NOT_U8 : V3DM_OK;
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
  DeviceGuardVt g(device);
  if (cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dErr), sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&t->hErr), sizeof(int32_t)) != cudaSuccess) {
    if (t->stream) cudaStreamDestroy(t->stream);
    if (t->dErr) cudaFree(t->dErr);
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
  t->dKeys = nullptr;
  t->dStage = nullptr;
  t->dIds = nullptr;
  t->nMax = 0;
  size_t m = nMax > 0 ? (size_t)nMax : 1;
  if (cudaMalloc(reinterpret_cast<void**>(&t->dKeys), m * kDescBytes) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dStage), m * kDescBytes * sizeof(float)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&t->dIds), m * sizeof(int32_t)) != cudaSuccess)
    return V3DM_ERR_CUDA;
  t->nMax = nMax;
  return V3DM_OK;
}

int v3dm_voctree_set_nodes_u8(v3dm_voctree* t, const uint8_t* nodes) {
  if (!t || !nodes) return V3DM_ERR_ARG;
  DeviceGuardVt g(t->device);
  if (!t->dNodes && cudaMalloc(reinterpret_cast<void**>(&t->dNodes), (size_t)t->nodeCount * kDescBytes) != cudaSuccess)
    return V3DM_ERR_CUDA;
  if (cudaMemcpyAsync(t->dNodes, nodes, (size_t)t->nodeCount * kDescBytes, cudaMemcpyHostToDevice, t->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return V3DM_OK;
}

int v3dm_voctree_set_nodes_f32(v3dm_voctree* t, const float* nodes) {
  if (!t || !nodes) return V3DM_ERR_ARG;
  if (!t->dStage) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuardVt g(t->device);
  if (!t->dNodes && cudaMalloc(reinterpret_cast<void**>(&t->dNodes), (size_t)t->nodeCount * kDescBytes) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return vt_convert(t, nodes, (size_t)t->nodeCount * kDescBytes, t->dNodes);
}

int v3dm_voctree_quantize_u8(v3dm_voctree* t, int n, const uint8_t* keys, int32_t* ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!keys || !ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (!t->dNodes || !t->dKeys) return V3DM_ERR_NOT_ALLOCATED;
  if (n > t->nMax) return V3DM_ERR_SIZE;
  if (n == 0) return V3DM_OK;
  DeviceGuardVt g(t->device);
  if (cudaMemcpyAsync(t->dKeys, keys, (size_t)n * kDescBytes, cudaMemcpyHostToDevice, t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  int st = vt_launch(t, n, t->dKeys, t->dIds, idMode);
  if (st != V3DM_OK) return st;
  if (cudaMemcpyAsync(ids, t->dIds, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return V3DM_OK;
}

int v3dm_voctree_quantize_f32(v3dm_voctree* t, int n, const float* keys, int32_t* ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!keys || !ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (!t->dNodes || !t->dKeys) return V3DM_ERR_NOT_ALLOCATED;
  if (n > t->nMax) return V3DM_ERR_SIZE;
  if (n == 0) return V3DM_OK;
  DeviceGuardVt g(t->device);
  int st = vt_convert(t, keys, (size_t)n * kDescBytes, t->dKeys);
  if (st != V3DM_OK) return st;
  st = vt_launch(t, n, t->dKeys, t->dIds, idMode);
  if (st != V3DM_OK) return st;
  if (cudaMemcpyAsync(ids, t->dIds, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
      cudaStreamSynchronize(t->stream) != cudaSuccess)
    return V3DM_ERR_CUDA;
  return V3DM_OK;
}

int v3dm_voctree_quantize_u8_device(v3dm_voctree* t, int n, const uint8_t* d_keys, int32_t* d_ids, int idMode) {
  if (!t || n < 0 || (n > 0 && (!d_keys || !d_ids)) || (idMode != V3DM_LEAF_GLOBAL && idMode != V3DM_LEAF_LOCAL))
    return V3DM_ERR_ARG;
  if (!t->dNodes) return V3DM_ERR_NOT_ALLOCATED;
  DeviceGuardVt g(t->device);
  return vt_launch(t, n, d_keys, d_ids, idMode);
}

int v3dm_voctree_stream(v3dm_voctree* t, void** s) {
  if (!t || !s) return V3DM_ERR_ARG;
  *s = (void*)t->stream;
  return V3DM_OK;
}

}  // extern "C"
