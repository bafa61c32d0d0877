// v3dm_match.cu -- SIMT matching kernel, guided-gate precompute, float->uint8 conversion
// and the finalize kernel (decisions, mutual filter, ordered compaction).
//
// The SIMT kernel computes the same candidates as the tcgen05 kernel with __dp4a on
// 64x64 tiles staged in shared memory; it is the legacy-path baseline the tensor-core
// kernel is measured against and a second implementation for cross-checks.
#include "v3dm_device.cuh"

namespace v3dm {

namespace {

constexpr int kSimtTile = 64;
constexpr int kSimtThreads = 256;

__global__ void __launch_bounds__(kSimtThreads)
k_match_simt(const uint8_t* __restrict__ L, const uint8_t* __restrict__ R, MatchArgs a) {
  __shared__ uint32_t sL[kSimtTile][33];
  __shared__ uint32_t sR[kSimtTile][33];
  const int l0 = blockIdx.y * kSimtTile, r0 = blockIdx.x * kSimtTile;
  const int tid = threadIdx.x;
  for (int i = tid; i < kSimtTile * 32; i += kSimtThreads) {
    int row = i >> 5, w = i & 31;
    int l = l0 + row, r = r0 + row;
    sL[row][w] = l < a.nL ? reinterpret_cast<const uint32_t*>(L + (size_t)l * kDescBytes)[w] : 0u;
    sR[row][w] = r < a.nR ? reinterpret_cast<const uint32_t*>(R + (size_t)r * kDescBytes)[w] : 0u;
  }
  __syncthreads();
  const int ty = tid >> 4, tx = tid & 15;
  uint32_t acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0u;
#pragma unroll 8
  for (int w = 0; w < 32; ++w) {
    uint32_t av[4], bv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) av[i] = sL[ty + 16 * i][w];
#pragma unroll
    for (int j = 0; j < 4; ++j) bv[j] = sR[tx + 16 * j][w];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = __dp4a(av[i], bv[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int l = l0 + ty + 16 * i;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int r = r0 + tx + 16 * j;
      int32_t S = (int32_t)acc[i][j];
      if (l < a.nL && r < a.nR && S >= a.T) {
        if (a.nGates && gated_out(a, l, r)) continue;
        record_best(a, l, r, S);
        int idx = atomicAdd(&a.segCount[0], 1);
        if (idx < a.segCap) a.cand[idx] = cand_pack(l, r, S);
      }
    }
  }
}

// Second values: every candidate that is not the best of its left (right) raises that
// feature's second value.  Runs after the matching kernel, when all best keys are final.
__global__ void k_seconds(MatchArgs a) {
  for (int seg = blockIdx.y; seg < a.nSeg; seg += gridDim.y) {
    long long n = a.segCount[seg];
    if (n > a.segCap) n = a.segCap;
    const unsigned long long* c = a.cand + (long long)seg * a.segCap;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
      int32_t l, r, S;
      cand_unpack(c[i], l, r, S);
      if ((unsigned long long)best_key(S, r) != a.lBest[l]) atomicMax(&a.lSec[l], (unsigned)(S + 1));
      if ((unsigned long long)best_key(S, l) != a.rBest[r]) atomicMax(&a.rSec[r], (unsigned)(S + 1));
    }
  }
}

// One CTA: decisions of every right, then of every left, the mutual filter of
// v3d_cudamatching.cu:546-551 and an ordered compaction of the pairs (ascending left).
// Every per-feature array and every segment count is cleared for the next call.
constexpr int kFinThreads = 1024;

__global__ void __launch_bounds__(kFinThreads)
k_finalize(MatchArgs a, float minScore, float minRatio, int32_t* __restrict__ rightBest,
           int32_t* __restrict__ leftBest, int2* __restrict__ pairs, int32_t* __restrict__ info) {
  __shared__ int warpSums[32];
  __shared__ int maxSeg;
  const int tid = threadIdx.x;
  if (tid == 0) maxSeg = 0;
  __syncthreads();
  for (int s = tid; s < a.nSeg; s += kFinThreads) {
    atomicMax(&maxSeg, a.segCount[s]);
    a.segCount[s] = 0;
  }
  for (int r = tid; r < a.nR; r += kFinThreads) {
    unsigned long long b = a.rBest[r];
    rightBest[r] = decide(b, a.rSec[r], minScore, minRatio);
    if (b) {
      a.rBest[r] = 0;
      a.rSec[r] = 0;
    }
  }
  __syncthreads();
  const int per = (a.nL + kFinThreads - 1) / kFinThreads;
  const int beg = min(tid * per, a.nL), end = min(beg + per, a.nL);
  int cnt = 0;
  for (int k = beg; k < end; ++k) {
    unsigned long long b = a.lBest[k];
    int r = decide(b, a.lSec[k], minScore, minRatio);
    if (b) {
      a.lBest[k] = 0;
      a.lSec[k] = 0;
    }
    bool ok = r >= 0 && rightBest[r] == k;
    leftBest[k] = ok ? r : -1;
    cnt += ok;
  }
  // block-wide exclusive scan of cnt
  const int lane = tid & 31, wid = tid >> 5;
  int inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) warpSums[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int v = warpSums[lane];
    int s = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += u;
    }
    warpSums[lane] = s - v;  // exclusive prefix of warp totals
    if (lane == 31) {
      info[kInfoPairs] = s;
      info[kInfoMaxSeg] = maxSeg;
    }
  }
  __syncthreads();
  int off = warpSums[wid] + inc - cnt;
  for (int k = beg; k < end; ++k) {
    int r = leftBest[k];
    if (r >= 0) pairs[off++] = make_int2(k, r);
  }
}

struct GateMat {
  float m[9];
};

// Per-left and per-right gate terms with the reference's expressions
// (epipolar: v3d_cudamatching.cu:289-291 and :298-299; homography: :325-330).
__global__ void k_gate_precompute(int type, GateMat g, const float2* __restrict__ lpos, int nL,
                                  const float2* __restrict__ rpos, int nR, float4* __restrict__ lv,
                                  float4* __restrict__ rv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nL) lv[i] = gate_left_terms(type, g.m, lpos[i]);
  if (i < nR) rv[i] = gate_right_terms(type, g.m, rpos[i]);
}

__device__ __forceinline__ uint32_t f32_to_u8_checked(float v, bool& ok) {
  float t = v * 512.0f;  // exact: scaling by a power of two
  int u = __float2int_rn(t);
  ok = ok && (t == (float)u) && u >= 0 && u <= 255;
  return (uint32_t)(u & 255);
}

__global__ void k_f32_to_u8(const float4* __restrict__ src, uint32_t* __restrict__ dst, long long n4, int* err) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n4) return;
  float4 v = src[i];
  bool ok = true;
  uint32_t w = f32_to_u8_checked(v.x, ok) | (f32_to_u8_checked(v.y, ok) << 8) | (f32_to_u8_checked(v.z, ok) << 16) |
               (f32_to_u8_checked(v.w, ok) << 24);
  dst[i] = w;
  if (!ok) atomicOr(err, kErrNotU8);
}

}  // namespace

cudaError_t launch_match_simt(const uint8_t* dL, const uint8_t* dR, const MatchArgs& a, cudaStream_t s) {
  dim3 grid((a.nR + kSimtTile - 1) / kSimtTile, (a.nL + kSimtTile - 1) / kSimtTile);
  k_match_simt<<<grid, kSimtThreads, 0, s>>>(dL, dR, a);
  return cudaGetLastError();
}

cudaError_t launch_seconds(const MatchArgs& a, cudaStream_t s) {
  dim3 grid(64, a.nSeg < 1024 ? a.nSeg : 1024);
  k_seconds<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const MatchArgs& a, float minScore, float minRatio, int32_t* dScratch, int32_t* dPairs,
                            int32_t* dInfo, cudaStream_t s) {
  // dScratch holds nR + nL ints: per-right decisions, then the per-left scratch.
  k_finalize<<<1, kFinThreads, 0, s>>>(a, minScore, minRatio, dScratch, dScratch + a.nR,
                                       reinterpret_cast<int2*>(dPairs), dInfo);
  return cudaGetLastError();
}

cudaError_t launch_gate_precompute(int type, const double* m, const float* dLPos, int nL, const float* dRPos,
                                   int nR, float4* lv, float4* rv, cudaStream_t s) {
  GateMat g;
  for (int i = 0; i < 9; ++i) g.m[i] = (float)m[i];  // double->float as in .cu:592-595
  int n = nL > nR ? nL : nR;
  if (n == 0) return cudaSuccess;
  k_gate_precompute<<<(n + 255) / 256, 256, 0, s>>>(type, g, reinterpret_cast<const float2*>(dLPos), nL,
                                                    reinterpret_cast<const float2*>(dRPos), nR, lv, rv);
  return cudaGetLastError();
}

cudaError_t launch_f32_to_u8(const float* src, uint8_t* dst, int n, int* err, cudaStream_t s) {
  long long n4 = (long long)n * (kDescBytes / 4);
  if (n4 == 0) return cudaSuccess;
  k_f32_to_u8<<<(unsigned)((n4 + 255) / 256), 256, 0, s>>>(reinterpret_cast<const float4*>(src),
                                                            reinterpret_cast<uint32_t*>(dst), n4, err);
  return cudaGetLastError();
}

}  // namespace v3dm
