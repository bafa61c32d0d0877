// v3dm_pair.cu -- decisions and bookkeeping around the two tcgen05 side passes of a pair.
//
//   k_records  exact work on the chunk records of a side pass (gates, chunk best, bound), merged
//              into each descriptor's best key and second value;
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

// Chunk records of a side pass: the exact lane-local work the side kernel leaves out.  For
// every score >= Smin the gates decide whether it is a candidate; the chunk best is the
// largest candidate (first column on ties), every other score of the chunk (candidates,
// masked scores and scores below Smin alike) bounds the second value.  kRecWarps warps share
// a record segment; a warp takes four records at a time: the eight lanes of a record hold
// four scores each (one coalesced 16-byte load), reduce the best key across the group, then
// the largest other score.  k_decide clears the segment counts for the next pass and reports
// an overflowing count (the host grows the list when it exceeds the capacity).
constexpr int kRecWarps = 4;

__global__ void k_records(PostArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  const int lane = threadIdx.x & 31;
  const int grp = lane >> 3;   // record of the four this lane works on
  const int part = lane & 7;   // its four scores: columns 4 * part .. 4 * part + 3
  const int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int w = warpGlobal; w < a.nSeg * kRecWarps; w += nWarps) {
    const int seg = w / kRecWarps, sub = w % kRecWarps;
    const int cnt = a.segCount[seg];
    if (cnt == 0) continue;
    const int n = (long long)cnt < a.segCap ? cnt : (int)a.segCap;
    const uint4* recs = a.records + (long long)seg * a.segCap * kRecordQuads;
    for (int i0 = 4 * sub; i0 < n; i0 += 4 * kRecWarps) {
      const int i = i0 + grp;
      const bool have = i < n;
      uint4 head = make_uint4(0u, 0u, 0u, 0u), q = head;
      if (have) {
        head = recs[(long long)i * kRecordQuads];
        q = recs[(long long)i * kRecordQuads + 1 + part];
      }
      const int orig = (int)head.x, col0 = (int)head.y, nB = (int)head.z, bRow0 = (int)head.w;
      const uint32_t sv[4] = {q.x, q.y, q.z, q.w};
      unsigned long long key[4];
      bool valid[4];
      unsigned long long cb = 0;
      int bPair = 0, bIdx = orig;  // batched gates: the record's pair and its A-side index
      if (a.bg.on && have) bgate_resolve(a.bg, a.aIsLeft, orig, &bPair, &bIdx);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int col = col0 + 4 * part + t;
        valid[t] = have && col < nB;
        const int32_t S = (int32_t)sv[t];
        bool strong = valid[t] && S >= a.Smin;
        if (a.bg.on && strong)
          strong = !bgate_rejects(a.bg, bPair, a.aIsLeft ? bIdx : col, a.aIsLeft ? col : bIdx);
        for (int gi = 0; gi < a.nGates && strong; ++gi)
          strong = !gate_rejects(a.gatesDev[gi], a.aIsLeft ? orig : col, a.aIsLeft ? col : orig);
        key[t] = strong ? best_key(S, a.bmap ? __ldg(a.bmap + bRow0 + col) : col) : 0ull;
        cb = key[t] > cb ? key[t] : cb;
      }
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, cb, off);
        cb = o > cb ? o : cb;
      }
      // every valid score but the chunk best's own bounds the second value
      uint32_t cw = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (valid[t] && !(key[t] != 0ull && key[t] == cb)) cw = max(cw, sv[t] + 1u);
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) cw = max(cw, __shfl_xor_sync(0xffffffffu, cw, off));
      if (have && part == 0) {
        if (cb) merge_chunk_best(&a.best[orig], &a.sec[orig], cb);
        if (cw) atomicMax(&a.sec[orig], cw);
      }
    }
  }
}

// Clears the segment counts after k_records (a separate launch: every warp of a segment reads
// the count first); reports an overflowing count.
__device__ __forceinline__ void clear_segments(const PostArgs& a) {
  int32_t* info = a.err - kInfoErr;
  for (int seg = blockIdx.x * blockDim.x + threadIdx.x; seg < a.nSeg; seg += gridDim.x * blockDim.x) {
    const int cnt = a.segCount[seg];
    if ((long long)cnt > a.segCap) atomicMax(&info[kInfoMaxSeg], cnt);
    if (cnt && !a.keepSegments) a.segCount[seg] = 0;
  }
}

// Copies right r's descriptor row to slot k of the pass-B operand.
__device__ __forceinline__ void gather_chosen(const PostArgs& a, int r, int k) {
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
// chosen for pass B right away: the first left to name a right claims it (flag exchange),
// and the claiming lanes of a warp take consecutive list slots with one counter update.
__global__ void k_decide(PostArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  clear_segments(a);
  const int lane = threadIdx.x & 31;
  const int nRows = a.rowsPtr ? *a.rowsPtr : a.nRows;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nRows; r += gridDim.x * blockDim.x) {
    const int idx = a.amap ? a.amap[r] : r;
    const unsigned long long b = a.best[idx];
    const unsigned s = a.secBound ? max(a.sec[idx], a.secBound[idx]) : a.sec[idx];
    int32_t d = decide(b, s, a.minScore, a.minRatio);
    if (a.gated && b != 0 && s != 0 && d != decide(b, 0u, a.minScore, a.minRatio)) {
      // the bound straddles the decision: exact re-score (k_rescore clears the state)
      const int k = atomicAdd(a.flaggedCount, 1);
      a.flagged[k] = idx;
      a.sec[idx] = 0;  // recomputed exactly by k_rescore
      d = -1;
    } else {
      if (b) a.best[idx] = 0;
      if (s) a.sec[idx] = 0;
    }
    a.decision[idx] = d;
    if (a.chooseFlag) {
      const bool claim = d >= 0 && atomicExch(&a.chooseFlag[d], 1) == 0;
      const unsigned act = __activemask();
      const unsigned m = __ballot_sync(act, claim);
      if (m) {
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(a.chooseCount, __popc(m));
        base = __shfl_sync(act, base, leader);
        if (claim) gather_chosen(a, d, base + __popc(m & ((1u << lane) - 1u)));
      }
    }
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

// A row is 'planes' blocks of 128 bytes, block p of row r at (p * cap + r) * 128 (one block:
// uint8 descriptors; six: the planar BF16 hi/lo layout).
__global__ void k_choose(const int32_t* __restrict__ leftDec, int nL, int* chosenFlag, int* chosenList,
                         int* chosenCount, const uint8_t* __restrict__ dR, uint8_t* __restrict__ dRc, int planes,
                         int capSrc, int capDst) {
  pdl_wait();
  pdl_launch_dependents();
  const int lane = threadIdx.x & 31;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nL; l += gridDim.x * blockDim.x) {
    const int r = leftDec[l];
    // the first left to name a right claims it; the claiming lanes of a warp take
    // consecutive list slots with one counter update
    const bool claim = r >= 0 && atomicExch(&chosenFlag[r], 1) == 0;
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, claim);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(chosenCount, __popc(m));
    base = __shfl_sync(act, base, leader);
    if (!claim) continue;
    const int k = base + __popc(m & ((1u << lane) - 1u));
    chosenList[k] = r;
    for (int p = 0; p < planes; ++p) {
      const uint4* src = reinterpret_cast<const uint4*>(dR + ((size_t)p * capSrc + r) * kDescBytes);
      uint4* dst = reinterpret_cast<uint4*>(dRc + ((size_t)p * capDst + k) * kDescBytes);
#pragma unroll
      for (int w = 0; w < kDescBytes / 16; ++w) dst[w] = src[w];
    }
  }
}

constexpr int kMutThreads = 256;
constexpr int kMutPerBlock = kMutThreads;  // one left per thread: every load of a thread in flight at once

// Pass 1: number of mutual pairs among each block's contiguous range of lefts.
__global__ void __launch_bounds__(kMutThreads)
k_mutual_count(const int32_t* __restrict__ leftDec, int nL, const int32_t* __restrict__ rightDec,
               int* __restrict__ blockCount) {
  pdl_wait();
  pdl_launch_dependents();
  __shared__ int wsum[kMutThreads / 32];
  const int k = blockIdx.x * kMutPerBlock + threadIdx.x;
  const int r = k < nL ? leftDec[k] : -1;
  int cnt = r >= 0 && rightDec[r] == k;
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

// Pass 2: each block offsets its pairs by the counts of the blocks before it (summed by the
// whole block) and writes them in ascending left order; clears the chosen-right flags.
__global__ void __launch_bounds__(kMutThreads)
k_mutual_write(const int32_t* __restrict__ leftDec, int nL, const int32_t* __restrict__ rightDec, int* chosenFlag,
               const int* __restrict__ blockCount, int nBlocks, int2* __restrict__ pairs, int32_t* info,
               int32_t* countOut) {
  pdl_wait();
  pdl_launch_dependents();
  __shared__ int wsum[kMutThreads / 32];
  __shared__ int wbefore[kMutThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k = blockIdx.x * kMutPerBlock + threadIdx.x;
  const int r = k < nL ? leftDec[k] : -1;
  const bool ok = r >= 0 && rightDec[r] == k;
  if (r >= 0) chosenFlag[r] = 0;
  int t = 0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += kMutThreads) t += blockCount[b];
  const int cnt = ok ? 1 : 0;
  int inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 31) wsum[wid] = inc;
  if (lane == 0) wbefore[wid] = t;
  __syncthreads();
  int blockOff = 0, before = 0;
  for (int w = 0; w < kMutThreads / 32; ++w) {
    blockOff += wbefore[w];
    if (w < wid) before += wsum[w];
  }
  if (ok) pairs[blockOff + before + inc - cnt] = make_int2(k, r);
  if (threadIdx.x == kMutThreads - 1 && blockIdx.x == nBlocks - 1) {
    const int total = blockOff + before + inc;
    info[kInfoPairs] = total;
    if (countOut) *countOut = total;
  }
}

}  // namespace

cudaError_t launch_post(const PostArgs& a, cudaStream_t s) {
  const int recBlocks = (a.nSeg * kRecWarps * 32 + 255) / 256;
  cudaError_t e = launch_pdl(k_records, dim3(recBlocks < 2048 ? recBlocks : 2048), dim3(256), 0, s, a);
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
  return launch_pdl(k_choose, dim3(blocks), dim3(256), 0, s, leftDec, nL, chosenFlag, chosenList, chosenCount, dR, dRc,
                    1, 0, 0);
}

cudaError_t launch_choose_planes(const int32_t* leftDec, int nL, int* chosenFlag, int* chosenList, int* chosenCount,
                                 const uint8_t* src, uint8_t* dst, int planes, int capSrc, int capDst,
                                 cudaStream_t s) {
  if (nL == 0) return cudaSuccess;
  int blocks = (nL + 255) / 256;
  if (blocks > 148) blocks = 148;
  return launch_pdl(k_choose, dim3(blocks), dim3(256), 0, s, leftDec, nL, chosenFlag, chosenList, chosenCount, src,
                    dst, planes, capSrc, capDst);
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
