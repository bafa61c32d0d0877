// v3dm_pair.cu -- decisions and bookkeeping around the two tcgen05 side passes of a pair.
//
//   k_records  exact work on the chunk records of a side pass (gates, chunk best, bound);
//   k_list     list pass (every chunk best that is not the descriptor's overall best raises its
//              second value);
//   k_decide   the per-descriptor decision of the reference
//              (v3d_cudamatching.cu:147-161 / :196-209, or the no-ratio test at :48 / :84).
//              With guided gates the second value is an upper bound; when the decision with
//              that bound differs from the decision with no second value at all, the
//              descriptor is flagged for an exact re-score instead.
//   k_rescore  exact second value of flagged descriptors: every score against the other
//              side that can matter, with the gates; k_rescore_decide then decides them.
//   k_choose   rights accepted by some left, de-duplicated, descriptors gathered for the
//              second side pass (the mutual filter only ever reads these rights).
//   k_mutual_count / k_mutual_write
//              mutual filter (.cu:546-551) with an ordered compaction (ascending left).
#include "v3dm_device.cuh"

namespace v3dm {

namespace {

// Merges a chunk best into a descriptor's state: best[] keeps the largest key, and whichever
// key loses the atomic comparison -- the new one, or the best it displaces -- is a second
// candidate.  Every key but the final best loses exactly one comparison, so sec[] ends as
// the exact largest of the other chunk bests.  A key carries the other side's index, so two
// equal keys are the same (left, right) scored twice (the proposal matcher's symmetric
// probing can score a pair in two cell blocks): it is one candidate, not a second value.
__device__ __forceinline__ void merge_chunk_best(unsigned long long* best, unsigned int* sec, unsigned long long cb) {
  const unsigned long long old = atomicMax(best, cb);
  if (old && old != cb) atomicMax(sec, (unsigned)((old < cb ? old : cb) >> kIndexBits));
}

// Chunk records of a side pass: the exact lane-local work the side kernel leaves out.  For
// every score >= Smin the gates decide whether it is a candidate; the chunk best is the
// largest candidate (first column on ties), every other score of the chunk (candidates,
// masked scores and scores below Smin alike) bounds the second value.  One warp per record
// segment; the segment's count is recorded (overflow check) and cleared for the next pass.
__global__ void k_records(PostArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  int32_t* info = a.err - kInfoErr;
  const int lane = threadIdx.x & 31;
  const int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int seg = warpGlobal; seg < a.nSeg; seg += nWarps) {
    const int cnt = a.segCount[seg];
    const long long n = cnt < a.segCap ? cnt : a.segCap;
    if (cnt == 0) continue;
    const uint4* recs = a.records + (long long)seg * a.segCap * kRecordQuads;
    for (long long i = lane; i < n; i += 32) {
      const uint4* rec = recs + i * kRecordQuads;
      const uint4 head = rec[0];
      const int orig = (int)head.x, col0 = (int)head.y, nB = (int)head.z, bRow0 = (int)head.w;
      unsigned long long cb = 0;
      uint32_t cw = 0;
      for (int k = 0; k < 8; ++k) {
        const uint4 q = rec[1 + k];
        const uint32_t sv[4] = {q.x, q.y, q.z, q.w};
        for (int t = 0; t < 4; ++t) {
          const int col = col0 + 4 * k + t;
          if (col >= nB) break;
          const int32_t S = (int32_t)sv[t];
          bool strong = S >= a.Smin;
          for (int gi = 0; gi < a.nGates && strong; ++gi)
            strong = !gate_rejects(a.gatesDev[gi], a.aIsLeft ? orig : col, a.aIsLeft ? col : orig);
          if (strong) {
            const unsigned long long key = best_key(S, a.bmap ? __ldg(a.bmap + bRow0 + col) : col);
            if (key > cb) {
              cw = max(cw, (uint32_t)(cb >> kIndexBits));
              cb = key;
            } else {
              cw = max(cw, (uint32_t)(S + 1));
            }
          } else {
            cw = max(cw, (uint32_t)(S + 1));
          }
        }
      }
      if (cb) merge_chunk_best(&a.best[orig], &a.sec[orig], cb);
      if (cw) atomicMax(&a.sec[orig], cw);
    }
    if (lane == 0) {
      atomicMax(&info[kInfoMaxSeg], cnt);
      a.segCount[seg] = 0;
    }
  }
}

// Chooses right r for pass B (once): flag, list entry, descriptor row gathered.
__device__ __forceinline__ void choose_one(const PostArgs& a, int r) {
  if (atomicExch(&a.chooseFlag[r], 1) != 0) return;
  const int k = atomicAdd(a.chooseCount, 1);
  a.chooseList[k] = r;
  if (a.choosePlanes) {
    for (int p = 0; p < a.choosePlanes; ++p) {
      const uint4* src = reinterpret_cast<const uint4*>(a.chooseSrc + ((size_t)p * a.chooseCapSrc + r) * 128);
      uint4* dst = reinterpret_cast<uint4*>(a.chooseDst + ((size_t)p * a.chooseCapDst + k) * 128);
#pragma unroll
      for (int w = 0; w < 8; ++w) dst[w] = src[w];
    }
  } else {
    const uint4* src = reinterpret_cast<const uint4*>(a.chooseSrc + (size_t)r * kDescBytes);
    uint4* dst = reinterpret_cast<uint4*>(a.chooseDst + (size_t)k * kDescBytes);
#pragma unroll
    for (int w = 0; w < kDescBytes / 16; ++w) dst[w] = src[w];
  }
}

// Decisions of the pass's descriptors; flags the ones whose gated bound straddles the
// decision, clears the state of the others.  With a.chooseFlag set, accepted partners are
// chosen for pass B right away.
__global__ void k_decide(PostArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  const int nRows = a.rowsPtr ? *a.rowsPtr : a.nRows;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nRows; r += gridDim.x * blockDim.x) {
    const int idx = a.amap ? a.amap[r] : r;
    const unsigned long long b = a.best[idx];
    const unsigned s = a.sec[idx];
    const int32_t d = decide(b, s, a.minScore, a.minRatio);
    if (a.gated && b != 0 && s != 0 && d != decide(b, 0u, a.minScore, a.minRatio)) {
      // the bound straddles the decision: exact re-score (k_rescore clears the state)
      const int k = atomicAdd(a.flaggedCount, 1);
      a.flagged[k] = idx;
      a.decision[idx] = -1;
      a.sec[idx] = 0;  // recomputed exactly by k_rescore
      continue;
    }
    a.decision[idx] = d;
    if (a.chooseFlag && d >= 0) choose_one(a, d);
    if (b) a.best[idx] = 0;
    if (s) a.sec[idx] = 0;
  }
}

// Exact second value of the flagged descriptors.  Their best key is already exact (the side
// pass applies the gates to every score that can pass the min-score test); the second value
// is the largest unmasked score other than the best.  Only scores >= T matter (T is chosen
// so that any second value below it, the masked -1e20f included, decides like "none").
// Each thread holds one descriptor of side B in registers and scores it against the flagged
// descriptors, staged 64 at a time in shared memory.
constexpr int kRescoreThreads = 256;
constexpr int kRescoreStage = 64;

__global__ void __launch_bounds__(kRescoreThreads) k_rescore(RescoreArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  __shared__ uint32_t sA[kRescoreStage][33];
  __shared__ int sIdx[kRescoreStage];
  __shared__ unsigned long long sBest[kRescoreStage];
  const int tid = threadIdx.x;
  const int j = blockIdx.x * kRescoreThreads + tid;
  const bool valid = j < a.nB;
  uint32_t b[32];
  if (valid) {
    const uint4* bj = reinterpret_cast<const uint4*>(a.descB + (size_t)j * kDescBytes);
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const uint4 x = bj[w];
      b[4 * w] = x.x;
      b[4 * w + 1] = x.y;
      b[4 * w + 2] = x.z;
      b[4 * w + 3] = x.w;
    }
  }
  const int n = *a.flaggedCount;
  for (int f0 = 0; f0 < n; f0 += kRescoreStage) {
    const int nf = min(kRescoreStage, n - f0);
    __syncthreads();
    for (int i = tid; i < nf * 32; i += kRescoreThreads) {
      const int f = i >> 5, w = i & 31;
      const int idx = a.flagged[f0 + f];
      sA[f][w] = reinterpret_cast<const uint32_t*>(a.descA + (size_t)idx * kDescBytes)[w];
      if (w == 0) {
        sIdx[f] = idx;
        sBest[f] = a.best[idx];
      }
    }
    __syncthreads();
    if (!valid) continue;
    for (int f = 0; f < nf; ++f) {
      uint32_t S = 0;
#pragma unroll
      for (int w = 0; w < 32; ++w) S = __dp4a(sA[f][w], b[w], S);
      if ((int32_t)S < a.T) continue;
      const int idx = sIdx[f];
      if (best_key((int32_t)S, j) == sBest[f]) continue;  // the best itself
      bool masked = false;
      for (int gi = 0; gi < a.nGates && !masked; ++gi)
        masked = gate_rejects(a.gatesDev[gi], a.aIsLeft ? idx : j, a.aIsLeft ? j : idx);
      if (!masked) atomicMax(&a.sec[idx], (unsigned)S + 1u);
    }
  }
}

// Decisions of the flagged descriptors from their exact second values; clears their state.
__global__ void k_rescore_decide(RescoreArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  const int n = *a.flaggedCount;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const int idx = a.flagged[f];
    a.decision[idx] = decide(a.best[idx], a.sec[idx], a.minScore, a.minRatio);
    a.best[idx] = 0;
    a.sec[idx] = 0;
  }
}

__global__ void k_choose(const int32_t* __restrict__ leftDec, int nL, int* chosenFlag, int* chosenList,
                         int* chosenCount, const uint8_t* __restrict__ dR, uint8_t* __restrict__ dRc) {
  pdl_wait();
  pdl_launch_dependents();
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nL; l += gridDim.x * blockDim.x) {
    const int r = leftDec[l];
    if (r < 0) continue;
    if (atomicExch(&chosenFlag[r], 1) != 0) continue;
    const int k = atomicAdd(chosenCount, 1);
    chosenList[k] = r;
    const uint4* src = reinterpret_cast<const uint4*>(dR + (size_t)r * kDescBytes);
    uint4* dst = reinterpret_cast<uint4*>(dRc + (size_t)k * kDescBytes);
#pragma unroll
    for (int w = 0; w < kDescBytes / 16; ++w) dst[w] = src[w];
  }
}

constexpr int kMutThreads = 256;
constexpr int kMutPerBlock = 2048;  // lefts per block (8 per thread, contiguous)

// Pass 1: number of mutual pairs among each block's contiguous range of lefts.
__global__ void __launch_bounds__(kMutThreads)
k_mutual_count(const int32_t* __restrict__ leftDec, int nL, const int32_t* __restrict__ rightDec,
               int* __restrict__ blockCount) {
  pdl_wait();
  pdl_launch_dependents();
  __shared__ int wsum[kMutThreads / 32];
  const int base = blockIdx.x * kMutPerBlock;
  int cnt = 0;
  for (int k = base + threadIdx.x; k < min(base + kMutPerBlock, nL); k += kMutThreads) {
    const int r = leftDec[k];
    cnt += r >= 0 && rightDec[r] == k;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kMutThreads / 32; ++w) t += wsum[w];
    blockCount[blockIdx.x] = t;
  }
}

// Pass 2: each block offsets its pairs by the counts of the blocks before it and writes them
// in ascending left order; clears the chosen-right flags.
__global__ void __launch_bounds__(kMutThreads)
k_mutual_write(const int32_t* __restrict__ leftDec, int nL, const int32_t* __restrict__ rightDec, int* chosenFlag,
               const int* __restrict__ blockCount, int nBlocks, int2* __restrict__ pairs, int32_t* info,
               int32_t* countOut) {
  pdl_wait();
  pdl_launch_dependents();
  __shared__ int blockOff;
  __shared__ int wsum[kMutThreads / 32];
  if (threadIdx.x < 32) {
    int t = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += 32) t += blockCount[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) {
      blockOff = t;
      if (blockIdx.x == nBlocks - 1) {
        info[kInfoPairs] = t + blockCount[blockIdx.x];
        if (countOut) *countOut = t + blockCount[blockIdx.x];
      }
    }
  }
  // each thread owns kMutPerBlock / kMutThreads consecutive lefts
  constexpr int kPer = kMutPerBlock / kMutThreads;
  const int beg = blockIdx.x * kMutPerBlock + threadIdx.x * kPer;
  int r[kPer];
  int cnt = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int k = beg + i;
    r[i] = k < nL ? leftDec[k] : -1;
    const bool ok = r[i] >= 0 && rightDec[r[i]] == k;
    if (r[i] >= 0) chosenFlag[r[i]] = 0;
    if (!ok) r[i] = -1;
    cnt += ok;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < wid; ++w) before += wsum[w];
  int off = blockOff + before + inc - cnt;
#pragma unroll
  for (int i = 0; i < kPer; ++i)
    if (r[i] >= 0) pairs[off++] = make_int2(beg + i, r[i]);
}

}  // namespace

cudaError_t launch_post(const PostArgs& a, cudaStream_t s) {
  const int listBlocks = (a.nSeg * 32 + 255) / 256;
  cudaError_t e = launch_pdl(k_records, dim3(listBlocks < 512 ? listBlocks : 512), dim3(256), 0, s, a);
  if (e != cudaSuccess) return e;
  int rows = a.nRows > 0 ? a.nRows : 1;
  int blocks = (rows + 255) / 256;
  return launch_pdl(k_decide, dim3(blocks < 1024 ? blocks : 1024), dim3(256), 0, s, a);
}

cudaError_t launch_rescore(const RescoreArgs& a, int grid, cudaStream_t s) {
  (void)grid;
  const int blocks = (a.nB + kRescoreThreads - 1) / kRescoreThreads;
  if (blocks > 0) {
    cudaError_t e = launch_pdl(k_rescore, dim3(blocks), dim3(kRescoreThreads), 0, s, a);
    if (e != cudaSuccess) return e;
  }
  return launch_pdl(k_rescore_decide, dim3(16), dim3(256), 0, s, a);
}

cudaError_t launch_choose(const int32_t* leftDec, int nL, int* chosenFlag, int* chosenList, int* chosenCount,
                          const uint8_t* dR, uint8_t* dRc, cudaStream_t s) {
  if (nL == 0) return cudaSuccess;
  int blocks = (nL + 255) / 256;
  if (blocks > 148) blocks = 148;
  return launch_pdl(k_choose, dim3(blocks), dim3(256), 0, s, leftDec, nL, chosenFlag, chosenList, chosenCount, dR, dRc);
}

cudaError_t launch_mutual(const int32_t* leftDec, int nL, const int32_t* rightDec, int* chosenFlag, int* blockCount,
                          int2* pairs, int32_t* info, int32_t* countOut, cudaStream_t s) {
  const int nBlocks = (nL + kMutPerBlock - 1) / kMutPerBlock;
  if (nBlocks == 0) return cudaSuccess;
  cudaError_t e = launch_pdl(k_mutual_count, dim3(nBlocks), dim3(kMutThreads), 0, s, leftDec, nL, rightDec, blockCount);
  if (e != cudaSuccess) return e;
  return launch_pdl(k_mutual_write, dim3(nBlocks), dim3(kMutThreads), 0, s, leftDec, nL, rightDec, chosenFlag,
                    blockCount, nBlocks, pairs, info, countOut);
}

}  // namespace v3dm
