// v3dm_batch.cu -- many image pairs matched with one persistent launch per side pass.
//
// The SfM apps match pairs one at a time (V3D/Apps/SfM/match_sequence.cpp:165-234): upload the
// left image, then for every right image upload it and call findPutativeMatches.  Here every
// pair's result is exactly that call's result (same rules, same order), but all pairs of a
// batch run together:
//   - the images live once in HBM, each padded with zero descriptors to a multiple of 256
//     rows (a zero descriptor scores 0, which is <= every real score, so it never changes a
//     chunk maximum);
//   - pass A is one k_side launch over a row table with one row per (pair, group of 128 or 256
//     lefts): the group against every tile of the pair's right image.  The state (best key,
//     second bound, decision) is kept per (pair, left) in HBM;
//   - every accepted left names one right.  Those rights (one per accepted left) are gathered
//     per left image, so one pass-B row scores a group of them, from all pairs of that left
//     image, against the left image;
//   - pass B is one k_side launch over that row table.  Its decisions are the reference's row
//     maxima (v3d_cudamatching.cu:164-210) for exactly the rights the mutual filter reads
//     (.cu:546-551);
//   - mutual filter and an ordered compaction into (pair, left, right) triples, grouped by pair
//     (pairs in order of their left image, then table order), ascending left within a pair.
// A guided call (v3dm_batch_match_guided) is runGuidedMatching / runGuidedHomographyMatching
// (.cu:554-694) of every pair after its findPutativeMatches, with one gate per pair: the same
// passes, the pair's gate applied on the fly wherever a score can decide (the chunk records,
// k_records), and an exact warp re-score (k_brescore) of the few descriptors whose gated
// second value the side pass could only bound.
// Float descriptors that are not all of the form u/512 (v3dm_batch_set_images_f32) take the same
// passes on the BF16 hi/lo layouts of the single-pair float matcher (v3dm_match_f.cu): groups of
// 128 lefts against tiles of 128 columns, each descriptor's exact best and second over the other
// image kept in registers (a guided call masks them with the pair's gate) and decided with the
// float rules, so each pair's result equals that matcher's.
// Every launch after the first reads its sizes from device memory, so the whole sequence is
// captured once as a CUDA graph and replayed while the images, pairs and parameters stay the same.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "v3dm_device.cuh"

namespace v3dm {

namespace {

struct BPair {          // one pair, in the batch's order (sorted by left image)
  int li, ri;           // left and right image
  int orig;             // index in the caller's pair table
  int nL;               // descriptors of the left image
  long long stateA0;    // first pass-A state of the pair
};

struct BImage {         // one image
  int rowOff;           // first row in the padded image buffer
  int n;                // descriptors
  int pairBeg, pairEnd; // pairs (batch order) whose left image this is
};

struct BImageB {        // pass-B layout of one left image (written by k_bscan)
  int cB;               // accepted lefts over all of its pairs
  int padBase;          // first row of its chosen rights in the pass-B operand buffer
  int rowStart;         // its first row in the pass-B row table
  int pad;
  long long stateB0;    // its first pass-B state
};

// Counter words of a batch call.
constexpr int kCntStates = 0;     // pass-B states (0 after an overflow)
constexpr int kCntRowsB = 1;      // pass-B rows (0 after an overflow)
constexpr int kCntOverflow = 2;   // 1: pass-B buffers too small
constexpr int kCntOut = 3;        // triples written
constexpr int kCntNeedStates = 4; // sizes the pass-B buffers need
constexpr int kCntNeedRows = 5;
constexpr int kCntNeedTable = 6;
constexpr int kCntFlagA = 7;      // guided call: pass-A states flagged for an exact re-score
constexpr int kCntFlagB = 12;     // and pass-B states
constexpr int kCntAll = 16;      // batch and proposal counter words

constexpr int kScanThreads = 1024;
constexpr int kChooseThreads = 256;
constexpr int kChoosePer = 4;     // lefts per thread and step in k_bchoose
constexpr int kBMutThreads = 256;
constexpr int kBMutPerBlock = 2048;

// Copies each image's descriptors to its padded place and zeroes its padding rows.
__global__ void k_bscatter(const uint8_t* __restrict__ src, const long long* __restrict__ srcOff,
                           const BImage* __restrict__ im, int nImages, uint8_t* __restrict__ dst) {
  for (int i = blockIdx.x; i < nImages; i += gridDim.x) {
    const BImage m = im[i];
    const long long nq = (long long)m.n * (kDescBytes / 16);
    const long long pq = (long long)((m.n + 255) & ~255) * (kDescBytes / 16);
    const uint4* s = reinterpret_cast<const uint4*>(src + srcOff[i] * kDescBytes);
    uint4* d = reinterpret_cast<uint4*>(dst + (size_t)m.rowOff * kDescBytes);
    for (long long k = threadIdx.x; k < pq; k += blockDim.x) d[k] = k < nq ? s[k] : make_uint4(0u, 0u, 0u, 0u);
  }
}

// Accepted lefts of every pair.
__global__ void __launch_bounds__(kChooseThreads)
k_bcount(const BPair* __restrict__ pairs, int nPairs, const int32_t* __restrict__ decA, int* __restrict__ cnt) {
  __shared__ int wsum[kChooseThreads / 32];
  for (int p = blockIdx.x; p < nPairs; p += gridDim.x) {
    const BPair q = pairs[p];
    int c = 0;
    for (int l = threadIdx.x; l < q.nL; l += kChooseThreads) c += decA[q.stateA0 + l] >= 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kChooseThreads / 32; ++w) t += wsum[w];
      cnt[p] = t;
    }
    __syncthreads();
  }
}

// Exclusive prefix sums of val(0..n-1), handed to out(i, prefix); returns the total.  One block.
template <class V, class O>
__device__ long long block_scan(int n, V val, O out, long long* sh) {
  const int T = blockDim.x, tid = threadIdx.x;
  const int per = (n + T - 1) / T;
  const int b = min(n, tid * per), e = min(n, b + per);
  long long s = 0;
  for (int i = b; i < e; ++i) s += val(i);
  sh[tid] = s;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    const long long v = tid >= o ? sh[tid - o] : 0;
    __syncthreads();
    sh[tid] += v;
    __syncthreads();
  }
  const long long total = sh[T - 1];
  long long run = sh[tid] - s;
  for (int i = b; i < e; ++i) {
    const long long v = val(i);
    out(i, run);
    run += v;
  }
  __syncthreads();
  return total;
}

// Pass-B layout: state and row offsets per pair and per left image, and the pass-B row table.
// One block.  When a buffer is too small it records the sizes needed and leaves pass B empty.
__global__ void __launch_bounds__(kScanThreads)
k_bscan(const int* __restrict__ cnt, int nPairs, const BImage* __restrict__ im, int nImages, int GM, int BN,
        long long capStates, long long capRows, long long capTable, long long* __restrict__ prefC,
        BImageB* __restrict__ imgB, BatchRow* __restrict__ rowsB, int* __restrict__ counters) {
  __shared__ long long sh[kScanThreads];
  const long long SB = block_scan(
      nPairs, [&](int i) { return (long long)cnt[i]; }, [&](int i, long long x) { prefC[i] = x; }, sh);
  if (threadIdx.x == 0) prefC[nPairs] = SB;
  __syncthreads();
  auto chosen = [&](int i) { return prefC[im[i].pairEnd] - prefC[im[i].pairBeg]; };
  const long long padTotal = block_scan(
      nImages, [&](int i) { return (chosen(i) + GM - 1) / GM * GM; },
      [&](int i, long long x) { imgB[i].padBase = (int)min(x, (long long)0x7fffffff); }, sh);
  const long long rowTotal = block_scan(
      nImages, [&](int i) { return (chosen(i) + GM - 1) / GM; },
      [&](int i, long long x) {
        imgB[i].rowStart = (int)min(x, (long long)0x7fffffff);
        imgB[i].cB = (int)min(chosen(i), (long long)0x7fffffff);
        imgB[i].stateB0 = prefC[im[i].pairBeg];
      },
      sh);
  const bool over = SB > capStates || padTotal > capRows || rowTotal > capTable;
  if (threadIdx.x == 0) {
    counters[kCntStates] = over ? 0 : (int)SB;
    counters[kCntRowsB] = over ? 0 : (int)rowTotal;
    counters[kCntOverflow] = over ? 1 : 0;
    counters[kCntNeedStates] = (int)min(SB, (long long)0x7fffffff);
    counters[kCntNeedRows] = (int)min(padTotal, (long long)0x7fffffff);
    counters[kCntNeedTable] = (int)min(rowTotal, (long long)0x7fffffff);
  }
  if (over) return;
  for (int i = threadIdx.x; i < nImages; i += blockDim.x) {
    const BImageB b = imgB[i];
    const BImage m = im[i];
    for (int g = 0; g * GM < b.cB; ++g) {
      BatchRow r;
      r.aRow = b.padBase + g * GM;
      r.validRows = min(GM, b.cB - g * GM);
      r.bRow0 = m.rowOff;
      r.nB = m.n;
      r.nTiles = (m.n + BN - 1) / BN;
      r.pad = 0;
      r.state0 = b.stateB0 + (long long)g * GM;
      rowsB[b.rowStart + g] = r;
    }
  }
}

// Gathers, per pair and in ascending left order, the right named by every accepted left into
// the pass-B operand buffer, with its (pair, left, right) identity.  A row is 'planes' blocks of
// 128 bytes, block p of row r at (p * planeRows + r) * 128 (one block: uint8 descriptors; six:
// the planar BF16 hi/lo layout).
__global__ void __launch_bounds__(kChooseThreads)
k_bchoose(const BPair* __restrict__ pairs, int nPairs, const BImage* __restrict__ im,
          const BImageB* __restrict__ imgB, const long long* __restrict__ prefC, const int32_t* __restrict__ decA,
          const uint8_t* __restrict__ img, uint8_t* __restrict__ dAB, int* __restrict__ chosenLeft,
          int* __restrict__ chosenRight, int* __restrict__ chosenPair, const int* __restrict__ counters, int planes,
          long long srcPlaneRows, long long dstPlaneRows) {
  __shared__ int wsum[kChooseThreads / 32];
  if (counters[kCntOverflow]) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int p = blockIdx.x; p < nPairs; p += gridDim.x) {
    const long long s0 = prefC[p];
    if (prefC[p + 1] == s0) continue;  // no accepted left (uniform over the block)
    const BPair q = pairs[p];
    const BImageB ib = imgB[q.li];
    const long long rowBase = ib.padBase + (s0 - ib.stateB0);
    const int rRowOff = im[q.ri].rowOff;
    int run = 0;
    // each thread takes kChoosePer consecutive lefts per step (their loads in flight together)
    for (int l0 = 0; l0 < q.nL; l0 += kChooseThreads * kChoosePer) {
      const int lb = l0 + threadIdx.x * kChoosePer;
      int d[kChoosePer];
#pragma unroll
      for (int i = 0; i < kChoosePer; ++i) d[i] = lb + i < q.nL ? decA[q.stateA0 + lb + i] : -1;
      int c = 0;
#pragma unroll
      for (int i = 0; i < kChoosePer; ++i) c += d[i] >= 0;
      int inc = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
      }
      if (lane == 31) wsum[w] = inc;
      __syncthreads();
      int before = 0, tot = 0;
#pragma unroll
      for (int k = 0; k < kChooseThreads / 32; ++k) {
        before += k < w ? wsum[k] : 0;
        tot += wsum[k];
      }
      int k = run + before + inc - c;  // slot of this thread's first accepted left, ascending left order
#pragma unroll
      for (int i = 0; i < kChoosePer; ++i) {
        if (d[i] < 0) continue;
        const long long st = s0 + k;
        chosenLeft[st] = lb + i;
        chosenRight[st] = d[i];
        chosenPair[st] = q.orig;
        for (int pl = 0; pl < planes; ++pl) {
          const uint4* src =
              reinterpret_cast<const uint4*>(img + ((size_t)pl * srcPlaneRows + rRowOff + d[i]) * kDescBytes);
          uint4* dst = reinterpret_cast<uint4*>(dAB + ((size_t)pl * dstPlaneRows + rowBase + k) * kDescBytes);
#pragma unroll
          for (int x = 0; x < kDescBytes / 16; ++x) dst[x] = src[x];
        }
        ++k;
      }
      run += tot;
      __syncthreads();
    }
  }
}

// Mutual filter over the pass-B states: state s is a match when the right's own decision
// (decB[s]) names the left that chose it.  Pass 1: count per block of states.
__global__ void __launch_bounds__(kBMutThreads)
k_bmutual_count(const int* __restrict__ counters, const int32_t* __restrict__ decB, const int* __restrict__ chosenLeft,
                int* __restrict__ blockCount) {
  __shared__ int wsum[kBMutThreads / 32];
  const int n = counters[kCntStates];
  const int base = blockIdx.x * kBMutPerBlock;
  int cnt = 0;
  for (int s = base + threadIdx.x; s < min(base + kBMutPerBlock, n); s += kBMutThreads)
    cnt += decB[s] == chosenLeft[s];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < kBMutThreads / 32; ++k) t += wsum[k];
    blockCount[blockIdx.x] = t;
  }
}

// Pass 2: ordered write of the (pair, left, right) triples.
__global__ void __launch_bounds__(kBMutThreads)
k_bmutual_write(int* __restrict__ counters, const int32_t* __restrict__ decB, const int* __restrict__ chosenLeft,
                const int* __restrict__ chosenRight, const int* __restrict__ chosenPair,
                const int* __restrict__ blockCount, int nBlocks, int3* __restrict__ out, int32_t* __restrict__ info) {
  __shared__ int blockOff;
  __shared__ int wsum[kBMutThreads / 32];
  const int n = counters[kCntStates];
  if (threadIdx.x < 32) {
    int t = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += 32) t += blockCount[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) {
      blockOff = t;
      if (blockIdx.x == nBlocks - 1) {
        counters[kCntOut] = t + blockCount[blockIdx.x];
        info[kInfoPairs] = t + blockCount[blockIdx.x];
      }
    }
  }
  constexpr int kPer = kBMutPerBlock / kBMutThreads;
  const int beg = blockIdx.x * kBMutPerBlock + threadIdx.x * kPer;
  bool ok[kPer];
  int cnt = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int s = beg + i;
    ok[i] = s < n && decB[s] == chosenLeft[s];
    cnt += ok[i];
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
  for (int k = 0; k < wid; ++k) before += wsum[k];
  int off = blockOff + before + inc - cnt;
#pragma unroll
  for (int i = 0; i < kPer; ++i)
    if (ok[i]) {
      const int s = beg + i;
      out[off++] = make_int3(chosenPair[s], chosenLeft[s], chosenRight[s]);
    }
}

// Exact second values of the flagged states of a guided pass (k_decide flagged the states whose
// gated bound straddles the decision), then their decisions; clears their state.  One warp per
// flagged state: every lane holds the state's descriptor, the lanes take the other image's
// descriptors in turn.  Scores >= T (below it any second value decides like none) that are not
// the best and that the pair's gate keeps give the exact second value, the reference's nextVal
// over its masked matrix (.cu:146).
constexpr int kBRescoreThreads = 256;

__global__ void __launch_bounds__(kBRescoreThreads)
k_brescore(BatchGateArgs g, int aIsLeft, const int* __restrict__ flagged, const int* __restrict__ flaggedCount,
           const BImage* __restrict__ im, const uint8_t* __restrict__ img, int32_t T, float minScore, float minRatio,
           unsigned long long* __restrict__ best, unsigned int* __restrict__ sec, int32_t* __restrict__ decision) {
  const int lane = threadIdx.x & 31;
  const int n = *flaggedCount;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; f < n; f += nWarps) {
    const int idx = flagged[f];
    int pair = 0, aIdx = 0;
    bgate_resolve(g, aIsLeft, idx, &pair, &aIdx);
    const int2 lr = g.pairLR[pair];
    const int aImg = aIsLeft ? lr.x : lr.y, bImg = aIsLeft ? lr.y : lr.x;
    const BImage ma = im[aImg], mb = im[bImg];
    uint32_t av[32];
    const uint4* ap = reinterpret_cast<const uint4*>(img + ((size_t)ma.rowOff + aIdx) * kDescBytes);
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const uint4 x = __ldg(ap + w);
      av[4 * w] = x.x;
      av[4 * w + 1] = x.y;
      av[4 * w + 2] = x.z;
      av[4 * w + 3] = x.w;
    }
    const float* m = g.gm + (size_t)pair * kBGateFloats;
    const float2 pa = g.pos[g.posOff[aImg] + aIdx];
    const float4 aT = aIsLeft ? gate_left_terms(g.type, m, pa) : gate_right_terms(g.type, m, pa);
    const unsigned long long bk = best[idx];
    unsigned s2 = 0;
    for (int j = lane; j < mb.n; j += 32) {
      const uint4* bp = reinterpret_cast<const uint4*>(img + ((size_t)mb.rowOff + j) * kDescBytes);
      uint32_t S = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        const uint4 x = __ldg(bp + w);
        S = __dp4a(av[4 * w], x.x, S);
        S = __dp4a(av[4 * w + 1], x.y, S);
        S = __dp4a(av[4 * w + 2], x.z, S);
        S = __dp4a(av[4 * w + 3], x.w, S);
      }
      if ((int32_t)S < T || best_key((int32_t)S, j) == bk) continue;
      const float2 pb = g.pos[g.posOff[bImg] + j];
      const bool masked = aIsLeft ? gate_rejects_terms(g.type, m[9], aT, gate_right_terms(g.type, m, pb))
                                  : gate_rejects_terms(g.type, m[9], gate_left_terms(g.type, m, pb), aT);
      if (!masked) s2 = max(s2, S + 1u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s2 = max(s2, __shfl_xor_sync(0xffffffffu, s2, o));
    if (lane == 0) {
      decision[idx] = decide(bk, s2, minScore, minRatio);
      best[idx] = 0;
      sec[idx] = 0;
    }
  }
}

// ---- proposal matching (learned cells) --------------------------------------------------
// Layout of the proposal: every image's descriptors are copied into an A layout, once per
// left-probed cell (its first probesL cells), and into a B layout, once per right-probed cell
// (its first probesR cells), both grouped by (image, cell).  A pair (i, j) is scored block by
// block: the lefts of i probing cell c against the rights of j probing c.  A (left, right) that
// shares several probed cells is scored in each of them with the same key; the merges treat
// equal keys as one candidate.  mapA / mapB give each layout row's index within its image.

constexpr int kCntRowsP = 8;      // counter words of the proposal (after the batch ones)
constexpr int kCntOverP = 9;      // 1: the proposal row table was too small
constexpr int kCntScored = 10;    // two words: scored (left, right) pairs, 64-bit
constexpr int kCntRowsVL = 13;    // rows of the proposal's exact verification, left side
constexpr int kCntRowsVR = 14;    // and right side

// Per image and cell: rows whose probed cells include the cell (A) and rows whose best cell
// it is (B).
__global__ void k_pcount(const BImage* __restrict__ im, int nImages, const uint8_t* __restrict__ cell, int probes,
                         int probesL, int probesR, int C, int* __restrict__ cntA, int* __restrict__ cntB) {
  extern __shared__ int pcSh[];
  for (int i = blockIdx.x; i < nImages; i += gridDim.x) {
    for (int t = threadIdx.x; t < 2 * C; t += blockDim.x) pcSh[t] = 0;
    __syncthreads();
    const BImage m = im[i];
    for (int r = threadIdx.x; r < m.n; r += blockDim.x) {
      const uint8_t* cr = cell + (size_t)(m.rowOff + r) * probes;
      for (int q = 0; q < probesL; ++q) atomicAdd(&pcSh[cr[q]], 1);
      for (int q = 0; q < probesR; ++q) atomicAdd(&pcSh[C + cr[q]], 1);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < C; t += blockDim.x) {
      cntA[i * C + t] = pcSh[t];
      cntB[i * C + t] = pcSh[C + t];
    }
    __syncthreads();
  }
}

// Block offsets of the A and B layouts (exclusive prefix sums over (image, cell)).  One block.
__global__ void __launch_bounds__(kScanThreads)
k_pscan_cells(const int* __restrict__ cntA, const int* __restrict__ cntB, int n, int* __restrict__ offA,
              int* __restrict__ offB) {
  __shared__ long long sh[kScanThreads];
  block_scan(n, [&](int i) { return (long long)cntA[i]; }, [&](int i, long long x) { offA[i] = (int)x; }, sh);
  block_scan(n, [&](int i) { return (long long)cntB[i]; }, [&](int i, long long x) { offB[i] = (int)x; }, sh);
}

// Copies the descriptors into the A and B layouts (order within a block is arbitrary: every
// result depends on the index maps, not on the order).
__global__ void k_pscatter(const BImage* __restrict__ im, int nImages, const uint8_t* __restrict__ cell, int probes,
                           int probesL, int probesR, int C, const int* __restrict__ offA, const int* __restrict__ offB,
                           const uint8_t* __restrict__ img, uint8_t* __restrict__ la, int* __restrict__ mapA,
                           uint8_t* __restrict__ lb, int* __restrict__ mapB) {
  extern __shared__ int psSh[];
  for (int i = blockIdx.x; i < nImages; i += gridDim.x) {
    for (int t = threadIdx.x; t < 2 * C; t += blockDim.x) psSh[t] = 0;
    __syncthreads();
    const BImage m = im[i];
    for (int r = threadIdx.x; r < m.n; r += blockDim.x) {
      const uint8_t* cr = cell + (size_t)(m.rowOff + r) * probes;
      const uint4* src = reinterpret_cast<const uint4*>(img + (size_t)(m.rowOff + r) * kDescBytes);
      uint4 d[kDescBytes / 16];
#pragma unroll
      for (int x = 0; x < kDescBytes / 16; ++x) d[x] = src[x];
      for (int q = 0; q < probesL; ++q) {
        const int c = cr[q];
        const int pos = offA[i * C + c] + atomicAdd(&psSh[c], 1);
        uint4* dst = reinterpret_cast<uint4*>(la + (size_t)pos * kDescBytes);
#pragma unroll
        for (int x = 0; x < kDescBytes / 16; ++x) dst[x] = d[x];
        mapA[pos] = r;
      }
      for (int q = 0; q < probesR; ++q) {
        const int c = cr[q];
        const int pos = offB[i * C + c] + atomicAdd(&psSh[C + c], 1);
        uint4* dst = reinterpret_cast<uint4*>(lb + (size_t)pos * kDescBytes);
#pragma unroll
        for (int x = 0; x < kDescBytes / 16; ++x) dst[x] = d[x];
        mapB[pos] = r;
      }
    }
    __syncthreads();
  }
}

// Row table of the proposal, cell-major: for every cell c, every left image i, every group g
// of GM lefts of i probing c, one row per pair (i, j) of the batch whose right image has
// rights under c, in batch order.  Consecutive rows then share their A block (the group), and
// the rows of one cell -- whose right blocks are what the CTAs read at the same time -- are
// together in the table.  One warp per (cell, left image) unit u = c * nImages + i.
// Pass 1 counts the unit's rows and the scored (left, right) pairs.
__global__ void k_prowcount(const BPair* __restrict__ pairs, const BImage* __restrict__ im, int nImages, int C,
                            int GM, const int* __restrict__ cntA, const int* __restrict__ cntB, int* __restrict__ rowCnt,
                            unsigned long long* __restrict__ scored) {
  const int lane = threadIdx.x & 31;
  const int nUnits = nImages * C;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < nUnits; u += (gridDim.x * blockDim.x) >> 5) {
    const int c = u / nImages, i = u - c * nImages;
    const int a = cntA[i * C + c];
    const BImage m = im[i];
    int partners = 0;
    unsigned long long sb = 0;
    if (a > 0)
      for (int p = m.pairBeg + lane; p < m.pairEnd; p += 32) {
        const int b = cntB[pairs[p].ri * C + c];
        partners += b > 0;
        sb += (unsigned long long)b;
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      partners += __shfl_xor_sync(0xffffffffu, partners, o);
      sb += __shfl_xor_sync(0xffffffffu, sb, o);
    }
    if (lane == 0) {
      rowCnt[u] = partners * ((a + GM - 1) / GM);
      if (sb) atomicAdd(scored, sb * (unsigned long long)a);
    }
  }
}

__global__ void __launch_bounds__(kScanThreads)
k_pscan_rows(const int* __restrict__ rowCnt, int nUnits, long long capRows, int* __restrict__ rowStart,
             int* __restrict__ counters) {
  __shared__ long long sh[kScanThreads];
  const long long total = block_scan(
      nUnits, [&](int i) { return (long long)rowCnt[i]; }, [&](int i, long long x) { rowStart[i] = (int)x; }, sh);
  if (threadIdx.x == 0) {
    const bool over = total > capRows;
    counters[kCntRowsP] = over ? 0 : (int)total;
    counters[kCntOverP] = over ? 1 : 0;
  }
}

// Pass 2 writes the unit's rows: groups outer, the partner pairs inner in batch order.
__global__ void k_prows(const BPair* __restrict__ pairs, const BImage* __restrict__ im, int nImages, int C, int GM,
                        int BN, const int* __restrict__ cntA, const int* __restrict__ cntB,
                        const int* __restrict__ offA, const int* __restrict__ offB, const int* __restrict__ rowStart,
                        const int* __restrict__ counters, BatchRow* __restrict__ rows) {
  if (counters[kCntOverP]) return;
  const int lane = threadIdx.x & 31;
  const int nUnits = nImages * C;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < nUnits; u += (gridDim.x * blockDim.x) >> 5) {
    const int c = u / nImages, i = u - c * nImages;
    const int a = cntA[i * C + c];
    if (a == 0) continue;
    const BImage m = im[i];
    int at = rowStart[u];
    for (int g = 0; g * GM < a; ++g) {
      for (int p0 = m.pairBeg; p0 < m.pairEnd; p0 += 32) {
        const int p = p0 + lane;
        int b = 0, ri = 0;
        if (p < m.pairEnd) {
          ri = pairs[p].ri;
          b = cntB[ri * C + c];
        }
        const unsigned mk = __ballot_sync(0xffffffffu, b > 0);
        if (b > 0) {
          BatchRow r;
          r.aRow = offA[i * C + c] + g * GM;
          r.validRows = min(GM, a - g * GM);
          r.bRow0 = offB[ri * C + c];
          r.nB = b;
          r.nTiles = (b + BN - 1) / BN;
          r.pad = 0;
          r.state0 = pairs[p].stateA0;
          rows[at + __popc(mk & ((1u << lane) - 1u))] = r;
        }
        at += __popc(mk);
      }
    }
  }
}

// Pass-B states of the proposal: exclusive prefix of the accepted lefts per pair.  One block.
__global__ void __launch_bounds__(kScanThreads)
k_pscan_states(const int* __restrict__ cnt, int nPairs, long long capStates, long long* __restrict__ prefC,
               int* __restrict__ counters) {
  __shared__ long long sh[kScanThreads];
  const long long SB = block_scan(
      nPairs, [&](int i) { return (long long)cnt[i]; }, [&](int i, long long x) { prefC[i] = x; }, sh);
  if (threadIdx.x == 0) {
    prefC[nPairs] = SB;
    const bool over = SB > capStates;
    counters[kCntStates] = over ? 0 : (int)SB;
    counters[kCntOverflow] = over ? 1 : 0;
    counters[kCntNeedStates] = (int)min(SB, (long long)0x7fffffff);
  }
}

// The accepted lefts of every pair in ascending order, with the right each one named.
__global__ void __launch_bounds__(kChooseThreads)
k_pchoose(const BPair* __restrict__ pairs, int nPairs, const long long* __restrict__ prefC,
          const int32_t* __restrict__ decA, int* __restrict__ chosenLeft, int* __restrict__ chosenRight,
          int* __restrict__ chosenPair, int* __restrict__ chosenSorted, const int* __restrict__ counters) {
  __shared__ int wsum[kChooseThreads / 32];
  if (counters[kCntOverflow]) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int p = blockIdx.x; p < nPairs; p += gridDim.x) {
    const long long s0 = prefC[p];
    if (prefC[p + 1] == s0) continue;
    const BPair q = pairs[p];
    int run = 0;
    for (int l0 = 0; l0 < q.nL; l0 += kChooseThreads) {
      const int l = l0 + threadIdx.x;
      const int d = l < q.nL ? decA[q.stateA0 + l] : -1;
      const bool acc = d >= 0;
      const unsigned m = __ballot_sync(0xffffffffu, acc);
      if (lane == 0) wsum[w] = __popc(m);
      __syncthreads();
      int before = 0, tot = 0;
#pragma unroll
      for (int k = 0; k < kChooseThreads / 32; ++k) {
        before += k < w ? wsum[k] : 0;
        tot += wsum[k];
      }
      if (acc) {
        const long long st = s0 + run + before + __popc(m & ((1u << lane) - 1u));
        chosenLeft[st] = l;
        chosenRight[st] = d;
        chosenPair[st] = q.orig;
        chosenSorted[st] = p;
      }
      run += tot;
      __syncthreads();
    }
  }
}

// Exact verification of the proposal (two gathered side passes on the tensor cores).  Pass A
// of the proposal scores each left only against its candidate rights, so its decisions (and
// those of a candidate-restricted pass B) can accept a pair that the reference's rules on the
// full score matrix reject: a missing second-best makes the ratio test more lenient.  Every
// pass-B state (an accepted left l of pair (i, j)) is therefore decided again over the full
// score matrix of its pair:
//   V-left:  l against every right of image j -> l's exact decision r (the reference's column
//            rule, v3d_cudamatching.cu:133-162);
//   V-right: that r against every left of image i -> r's exact decision (the row rule,
//            .cu:164-210).
// The state is a match when r's exact decision is l (the mutual filter, .cu:546-551).  Every
// output pair is then a pair of exhaustive matching; what the proposal can still miss are
// lefts that pass A did not accept.  V-left entries are the states grouped by right image (a
// counting sort); V-right entries are the states themselves, already grouped by left image.

// V-left, pass 1: states per right image.
__global__ void k_vcount(const BPair* __restrict__ pairs, const int* __restrict__ chosenSorted,
                         const int* __restrict__ counters, int* __restrict__ cntJ) {
  const int n = counters[kCntStates];  // 0 after a state overflow
  for (int st = blockIdx.x * blockDim.x + threadIdx.x; st < n; st += gridDim.x * blockDim.x)
    atomicAdd(&cntJ[pairs[chosenSorted[st]].ri], 1);
}

// Entry offsets per right image and row starts of both verification passes (exclusive prefix
// sums).  One block.  Row counts go to kCntRowsVL / kCntRowsVR; a row table too small raises
// the overflow flag.
__global__ void __launch_bounds__(kScanThreads)
k_vscan(const int* __restrict__ cntJ, const BImage* __restrict__ im, int nImages, const long long* __restrict__ prefC,
        int GR, long long capRows, int* __restrict__ offJ, int* __restrict__ rowStartL, int* __restrict__ rowStartR,
        int* __restrict__ counters) {
  __shared__ long long sh[kScanThreads];
  const long long total = block_scan(
      nImages, [&](int j) { return (long long)cntJ[j]; }, [&](int j, long long x) { offJ[j] = (int)x; }, sh);
  __syncthreads();
  const long long rowsL = block_scan(
      nImages, [&](int j) { return (long long)((cntJ[j] + GR - 1) / GR); },
      [&](int j, long long x) { rowStartL[j] = (int)x; }, sh);
  __syncthreads();
  const long long rowsR = block_scan(
      nImages,
      [&](int i) {
        const long long c = prefC[im[i].pairEnd] - prefC[im[i].pairBeg];
        return (c + GR - 1) / GR;
      },
      [&](int i, long long x) { rowStartR[i] = (int)x; }, sh);
  if (threadIdx.x == 0) {
    offJ[nImages] = (int)total;
    // after a state overflow there are no states: no rows either (the call is repeated)
    const bool over = counters[kCntOverflow] != 0 || rowsL > capRows || rowsR > capRows;
    counters[kCntRowsVL] = over ? 0 : (int)rowsL;
    counters[kCntRowsVR] = over ? 0 : (int)rowsR;
    if (over) counters[kCntOverflow] = 1;
  }
}

// V-left, pass 2: every state's entry (its left's descriptor row in the image buffer), grouped
// by right image.  Counts cntJ down to zero for the next call.
__global__ void k_vscatter(const BPair* __restrict__ pairs, const BImage* __restrict__ im,
                           const int* __restrict__ chosenLeft, const int* __restrict__ chosenSorted,
                           const int* __restrict__ counters, const int* __restrict__ offJ, int* __restrict__ cntJ,
                           int* __restrict__ srcRow, int* __restrict__ stateOf) {
  const int n = counters[kCntStates];
  for (int st = blockIdx.x * blockDim.x + threadIdx.x; st < n; st += gridDim.x * blockDim.x) {
    const BPair q = pairs[chosenSorted[st]];
    const int pos = offJ[q.ri] + atomicSub(&cntJ[q.ri], 1) - 1;
    srcRow[pos] = im[q.li].rowOff + chosenLeft[st];
    stateOf[pos] = st;
  }
}

// V-left, pass 3: rows of up to GR entries of one right image against that image (one thread
// per image).
__global__ void k_vrows_left(const BImage* __restrict__ im, int nImages, int GR, int BN, const int* __restrict__ offJ,
                             const int* __restrict__ rowStartL, const int* __restrict__ counters,
                             BatchRow* __restrict__ rows) {
  if (counters[kCntOverflow]) return;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nImages; j += gridDim.x * blockDim.x) {
    const int e0 = offJ[j], ne = offJ[j + 1] - e0;
    int at = rowStartL[j];
    for (int g = 0; g * GR < ne; ++g) {
      BatchRow r;
      r.aRow = e0 + g * GR;
      r.validRows = min(GR, ne - g * GR);
      r.bRow0 = im[j].rowOff;
      r.nB = im[j].n;
      r.nTiles = (im[j].n + BN - 1) / BN;
      r.pad = 0;
      r.state0 = 0;  // the state of an entry comes from stateOf
      rows[at++] = r;
    }
  }
}

// V-right: the right each state's exact left decision named (row 0 of its image when there is
// none: scored, then ignored), and rows of up to GR consecutive states of one left image
// against that image; a row's states are its entries (state0 = aRow).
__global__ void k_vsrc_right(const BPair* __restrict__ pairs, const BImage* __restrict__ im,
                             const int* __restrict__ chosenSorted, const int32_t* __restrict__ decLeft,
                             const int* __restrict__ counters, int* __restrict__ srcRow) {
  const int n = counters[kCntStates];
  for (int st = blockIdx.x * blockDim.x + threadIdx.x; st < n; st += gridDim.x * blockDim.x) {
    const int r = decLeft[st];
    srcRow[st] = im[pairs[chosenSorted[st]].ri].rowOff + (r >= 0 ? r : 0);
  }
}

__global__ void k_vrows_right(const BImage* __restrict__ im, int nImages, const long long* __restrict__ prefC, int GR,
                              int BN, const int* __restrict__ rowStartR, const int* __restrict__ counters,
                              BatchRow* __restrict__ rows) {
  if (counters[kCntOverflow]) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nImages; i += gridDim.x * blockDim.x) {
    const long long s0 = prefC[im[i].pairBeg], ns = prefC[im[i].pairEnd] - s0;
    int at = rowStartR[i];
    for (long long g = 0; g * GR < ns; ++g) {
      BatchRow r;
      r.aRow = (int)(s0 + g * GR);
      r.validRows = (int)min((long long)GR, ns - g * GR);
      r.bRow0 = im[i].rowOff;
      r.nB = im[i].n;
      r.nTiles = (im[i].n + BN - 1) / BN;
      r.pad = 0;
      r.state0 = r.aRow;
      rows[at++] = r;
    }
  }
}

// A state is a match when its left's exact decision names a right whose exact decision names
// the left back.  The right of the state becomes that exact right; decB holds the left for the
// mutual kernels (k_bmutual_*) when it is a match, else -1.
__global__ void k_vmerge(const int* __restrict__ counters, const int32_t* __restrict__ decLeft,
                         const int* __restrict__ chosenLeft, int* __restrict__ chosenRight, int32_t* __restrict__ decB) {
  const int n = counters[kCntStates];
  for (int st = blockIdx.x * blockDim.x + threadIdx.x; st < n; st += gridDim.x * blockDim.x) {
    const int r = decLeft[st], l = chosenLeft[st];
    const bool ok = r >= 0 && decB[st] == l;
    chosenRight[st] = r;
    decB[st] = ok ? l : -1;
  }
}

}  // namespace

}  // namespace v3dm

using namespace v3dm;

struct v3dm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  TcPlan* tc = nullptr;
  int schedule = 0;
  // images
  int nImages = 0;
  std::vector<int> counts;
  std::vector<long long> srcOff;   // first descriptor of each image in the caller's concatenation
  std::vector<int> rowOff;         // first row of each image in the padded buffer
  long long totalRows = 0;         // padded rows of all images
  long long totalDesc = 0;
  uint8_t* dImg = nullptr;
  long long imgCap = 0;            // bytes
  uint8_t* dStage = nullptr;
  long long stageCap = 0;          // descriptors
  long long* dSrcOff = nullptr;
  BImage* dImages = nullptr;
  int imagesCap = 0;
  bool haveImages = false;
  // pairs (batch order: stable sort by left image)
  int nPairs = 0;
  std::vector<int> pairLi, pairRi;  // caller's order
  std::vector<BPair> bp;            // batch order
  std::vector<BImage> bim;
  BPair* dPairs = nullptr;
  int pairsCap = 0;
  long long SA = 0;                 // pass-A states
  long long workOps = 0;            // sum over pairs of 2 * 128 * nL * nR
  bool havePairs = false;
  // pass A
  BatchRow* dRowsA = nullptr;
  long long rowsACap = 0;
  int nRowsA = 0;
  int rowsCfg = -1;                 // configuration the pass-A rows were built for
  bool rowsDirty = true;
  // per-state arrays (pass A states; pass B reuses the first SB entries of best/sec)
  unsigned long long* dBest = nullptr;
  unsigned int* dSec = nullptr;
  int32_t* dDecA = nullptr;
  long long stateCap = 0;
  // chunk records of the side passes
  uint4* dRecords = nullptr;
  unsigned long long* dList = nullptr;
  int* dSegCount = nullptr;
  int nSeg = 0;
  long long segCap = 0;
  // pass B
  int* dCnt = nullptr;
  long long* dPrefC = nullptr;
  BImageB* dImgB = nullptr;
  uint8_t* dAB = nullptr;
  BatchRow* dRowsB = nullptr;
  int32_t* dDecB = nullptr;
  int* dChosenLeft = nullptr;
  int* dChosenRight = nullptr;
  int* dChosenPair = nullptr;
  int* dBlockCount = nullptr;
  int3* dOut = nullptr;
  long long capB = 0, capRowsB = 0, capTableB = 0;
  // call state
  int* dCounters = nullptr;
  int32_t* dInfo = nullptr;
  int32_t* hInfo = nullptr;         // pinned: info words then counter words
  TcMaps mapsA, mapsB;
  bool mapsValid = false;
  int lastLaunches = 0;
  // graph of one call
  bool useGraph = true;
  cudaGraphExec_t graph = nullptr;
  uint32_t graphMs = 0, graphMr = 0;
  int graphLaunches = 0;
  bool pendingCheck = false;
  // proposal matching (learned cells)
  uint8_t* dCell = nullptr;         // per padded image row: its probed cells, best first
  long long cellCap = 0;
  int* dCntA = nullptr;             // per (image, cell): A-layout rows, B-layout rows, offsets
  int* dCntB = nullptr;
  int* dOffA = nullptr;
  int* dOffB = nullptr;
  long long cellTabCap = 0;
  uint8_t* dLA = nullptr;           // A layout: every descriptor once per probed cell
  long long laCap = 0;              // bytes
  int* dMapA = nullptr;
  long long mapACap = 0;
  uint8_t* dLB = nullptr;           // B layout: every descriptor once, under its best cell
  long long lbCap = 0;
  int* dMapB = nullptr;
  long long mapBCap = 0;
  int* dRowCnt = nullptr;           // per pair: proposal rows and their first index
  int* dRowStart = nullptr;
  long long pairTabCap = 0;
  BatchRow* dRowsP = nullptr;
  long long rowsPCap = 0;
  long long rowsPNeed = 0;
  long long laRows = 0, lbRows = 0;
  int* dChosenSorted = nullptr;     // per pass-B state: the pair's index in batch order
  long long chosenSortedCap = 0;
  TcMaps mapsP;
  bool mapsPValid = false;
  // proposal: exact verification of its states (gathered entries against whole images)
  int* dCntE = nullptr;             // per image: V-left entries (zero between calls)
  int* dOffE = nullptr;             // per image + 1: first V-left entry
  int* dRowStartE = nullptr;        // per image: first V-left row
  int* dRowStartR = nullptr;        // per image: first V-right row
  long long unitTabCap = 0;
  int* dSrcRowE = nullptr;          // per V-left entry: its left's row in the image buffer
  int* dStateE = nullptr;           // per V-left entry: its state
  int* dSrcRowR = nullptr;          // per state: row of the right its exact left decision named
  int32_t* dDecL = nullptr;         // per state: exact decision of its left
  long long entryCap = 0;
  BatchRow* dRowsPB = nullptr;      // row table of V-left, then of V-right
  long long rowsPBCap = 0;
  CUtensorMap mapImgG;              // B of the verification: the image buffer, gather-configuration tiles
  const uint8_t* mapImgGimg = nullptr;
  long long mapImgGrows = 0;
  const uint8_t* mapsPla = nullptr;
  const uint8_t* mapsPlb = nullptr;
  cudaGraphExec_t graphP = nullptr;
  uint32_t gpMs = 0, gpMr = 0;
  int gpProbes = 0, gpCells = 0, gpLaunches = 0;
  const v3dm_projection* gpProj = nullptr;
  long long exhaustivePairs = 0;    // sum over pairs of nL * nR
  // guided calls: positions of the images' descriptors and one gate per pair
  float2* dPos = nullptr;
  long long posCap = 0;
  bool havePositions = false;
  float* dGate = nullptr;           // kBGateFloats per pair (caller's order)
  long long gateCap = 0;
  int2* dPairLR = nullptr;          // per pair (caller's order): left, right image
  long long pairLRCap = 0;
  long long* dStateA0 = nullptr;    // per pair (batch order): first pass-A state
  int* dOrigOf = nullptr;           // per pair (batch order): index in the caller's order
  long long pairAuxCap = 0;
  int* dFlag = nullptr;             // flagged states of one pass
  long long flagCap = 0;
  // float descriptors not all of the form u/512: BF16 hi/lo layouts (6 planes of fRows x 128 B)
  bool floatMode = false;
  int numSMs = 0;
  float* dStageF = nullptr;         // the caller's floats, staged
  long long stageFCap = 0;          // floats
  int* dRowOffI = nullptr;          // per image: first row (device copy of rowOff)
  long long rowOffCap = 0;
  uint8_t* dFA = nullptr;           // A layout of every image: [hi | lo | hi]
  uint8_t* dFB = nullptr;           // B layout of every image: [hi | hi | lo]
  long long fImgCapA = 0, fImgCapB = 0;  // bytes
  int fRows = 0;                    // rows per plane of dFA / dFB
  uint8_t* dFAB = nullptr;          // pass-B A operand: the chosen rights' A rows, capRowsB rows per plane
  long long fabCap = 0;             // bytes
  CUtensorMap fmA_A, fmA_B, fmB_A, fmB_B;
  bool fMapsValid = false;
  // profiling
  bool profile = false;
  cudaEvent_t ev[4] = {};
  double profMs[2] = {0.0, 0.0};
  int profN[2] = {0, 0};
  bool profPending = false;
};

namespace {

int bfail(cudaError_t e, const char* what, int line) {
  record_cuda_error(e, "v3dm_batch.cu", line, what);
  return V3DM_ERR_CUDA;
}

#define V3DM_BTRY(expr)                                       \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) return bfail(e_, #expr, __LINE__); \
  } while (0)

struct BDeviceGuard {
  int prev = -1;
  explicit BDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~BDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <class T>
void bfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// Ensures *p holds at least 'need' elements (contents are not kept).
template <class T>
cudaError_t ensure(T** p, long long* cap, long long need) {
  if (need <= *cap && *p) return cudaSuccess;
  bfree(*p);
  *cap = 0;
  long long n = need > 0 ? need : 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), (size_t)n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  *cap = n;
  return cudaSuccess;
}

void drop_graph(v3dm_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  if (b->graphP) cudaGraphExecDestroy(b->graphP);
  b->graphP = nullptr;
}

cudaError_t alloc_records(v3dm_batch* b, long long segCap) {
  bfree(b->dRecords);
  bfree(b->dList);
  bfree(b->dSegCount);
  b->segCap = 0;
  const int nSeg = tc_segments(b->tc);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->dRecords), (size_t)nSeg * segCap * kRecordQuads * sizeof(uint4));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->dList), (size_t)nSeg * segCap * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->dSegCount), (size_t)nSeg * sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->dSegCount, 0, (size_t)nSeg * sizeof(int), b->stream);
  if (e != cudaSuccess) return e;
  b->nSeg = nSeg;
  b->segCap = segCap;
  return cudaSuccess;
}

// Pass-B buffers for capStates states.
cudaError_t alloc_passB(v3dm_batch* b, long long capStates) {
  int GM = 0, BN = 0;
  tc_config_shape(tc_get_config(b->tc), &GM, &BN);
  const long long capRows = capStates + (long long)b->nImages * 256 + 256;
  const long long capTable = capStates / 128 + b->nImages + 1;
  long long c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, c6 = 0, c7 = 0;
  bfree(b->dAB);
  bfree(b->dRowsB);
  bfree(b->dDecB);
  bfree(b->dChosenLeft);
  bfree(b->dChosenRight);
  bfree(b->dChosenPair);
  bfree(b->dBlockCount);
  bfree(b->dOut);
  bfree(b->dChosenSorted);
  b->chosenSortedCap = 0;
  b->capB = b->capRowsB = b->capTableB = 0;
  cudaError_t e = ensure(&b->dAB, &c0, capRows * kDescBytes);
  if (e == cudaSuccess) e = ensure(&b->dRowsB, &c1, capTable);
  if (e == cudaSuccess) e = ensure(&b->dDecB, &c2, capStates);
  if (e == cudaSuccess) e = ensure(&b->dChosenLeft, &c3, capStates);
  if (e == cudaSuccess) e = ensure(&b->dChosenRight, &c4, capStates);
  if (e == cudaSuccess) e = ensure(&b->dChosenPair, &c5, capStates);
  if (e == cudaSuccess) e = ensure(&b->dBlockCount, &c6, capStates / kBMutPerBlock + 1);
  if (e == cudaSuccess) e = ensure(&b->dOut, &c7, capStates);
  if (e == cudaSuccess) e = ensure(&b->dChosenSorted, &b->chosenSortedCap, capStates);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->dAB, 0, (size_t)capRows * kDescBytes, b->stream);
  if (e != cudaSuccess) return e;
  b->capB = capStates;
  b->capRowsB = capRows;
  b->capTableB = capTable;
  b->mapsValid = false;
  b->fMapsValid = false;
  return cudaSuccess;
}

// Row-table key of the float passes (the integer ones use the tile configuration).
constexpr int kFloatRowsCfg = -2;

// Pass-A rows for groups of GM lefts and tiles of BN columns; cfg names the shape.
int build_rows(v3dm_batch* b, int GM, int BN, int cfg) {
  std::vector<BatchRow> rows;
  for (const BPair& q : b->bp) {
    const int nR = b->counts[q.ri];
    if (q.nL == 0 || nR == 0) continue;
    for (int g = 0; g * GM < q.nL; ++g) {
      BatchRow r;
      r.aRow = b->rowOff[q.li] + g * GM;
      r.validRows = std::min(GM, q.nL - g * GM);
      r.bRow0 = b->rowOff[q.ri];
      r.nB = nR;
      r.nTiles = (nR + BN - 1) / BN;
      r.pad = 0;
      r.state0 = q.stateA0 + (long long)g * GM;
      rows.push_back(r);
    }
  }
  if (rows.size() > 0x7fffffffULL) return V3DM_ERR_SIZE;
  V3DM_BTRY(ensure(&b->dRowsA, &b->rowsACap, (long long)rows.size()));
  if (!rows.empty())
    V3DM_BTRY(cudaMemcpyAsync(b->dRowsA, rows.data(), rows.size() * sizeof(BatchRow), cudaMemcpyHostToDevice, b->stream));
  V3DM_BTRY(cudaStreamSynchronize(b->stream));  // 'rows' is pageable host memory
  b->nRowsA = (int)rows.size();
  b->rowsCfg = cfg;
  b->rowsDirty = false;
  b->mapsValid = false;
  drop_graph(b);
  return V3DM_OK;
}

int ensure_maps(v3dm_batch* b) {
  if (b->mapsValid && b->mapsA.cfg == tc_get_config(b->tc)) return V3DM_OK;
  V3DM_BTRY(tc_side_maps(b->tc, &b->mapsA, b->dImg, (int)b->totalRows, b->dImg, (int)b->totalRows));
  V3DM_BTRY(tc_side_maps(b->tc, &b->mapsB, b->dAB, (int)b->capRowsB, b->dImg, (int)b->totalRows));
  b->mapsValid = true;
  return V3DM_OK;
}

// Enqueues one batch call (all launches read their sizes from device memory).  With bg set, the
// call is guided: every pair's gate applies, and flagged states are re-scored exactly.
int enqueue_batch(v3dm_batch* b, float minScore, float minRatio, bool withEvents,
                  const BatchGateArgs* bg = nullptr) {
  int GM = 0, BN = 0;
  tc_config_shape(tc_get_config(b->tc), &GM, &BN);
  const int32_t Smin = host_smallest_passing_score(minScore);
  const bool gated = bg != nullptr;
  int32_t Tg = 0;
  if (gated) {
    const int st = host_candidate_threshold(minScore, minRatio, true, &Tg);
    if (st != V3DM_OK) return st;
  }
  int launches = 0;
  V3DM_BTRY(cudaMemsetAsync(b->dInfo, 0, (kInfoWords + kCntAll) * sizeof(int32_t), b->stream));
  SideArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.Smin = Smin;
  if (host_candidate_threshold(minScore, minRatio, gated, &sa.Tsec) != V3DM_OK) sa.Tsec = 0;
  sa.records = b->dRecords;
  sa.segCount = b->dSegCount;
  sa.segCap = b->segCap;
  sa.nSeg = b->nSeg;
  sa.err = b->dInfo + kInfoErr;
  PostArgs pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.records = b->dRecords;
  pa.segCount = b->dSegCount;
  pa.segCap = b->segCap;
  pa.nSeg = b->nSeg;
  pa.Smin = Smin;
  pa.minScore = minScore;
  pa.minRatio = minRatio;
  pa.best = b->dBest;
  pa.sec = b->dSec;
  pa.err = b->dInfo + kInfoErr;
  const int rescoreGrid = 4 * 148;
  if (gated) {
    pa.gated = 1;
    pa.bg = *bg;
    pa.flagged = b->dFlag;
    pa.flaggedCount = b->dCounters + kCntFlagA;
  }
  // ---- pass A: every (pair, left group) against the pair's right image
  sa.aIsLeft = 1;
  sa.best = b->dBest;
  sa.sec = b->dSec;
  sa.rows = b->dRowsA;
  sa.nRows = b->nRowsA;
  sa.schedule = b->schedule;
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[0], b->stream));
  V3DM_BTRY(launch_side_batch(b->tc, b->mapsA, sa, b->stream));
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[1], b->stream));
  launches += b->nRowsA > 0;
  pa.nRows = (int)b->SA;
  pa.aIsLeft = 1;
  pa.decision = b->dDecA;
  V3DM_BTRY(launch_post(pa, b->stream));
  launches += 3;
  if (gated) {
    k_brescore<<<rescoreGrid, kBRescoreThreads, 0, b->stream>>>(*bg, 1, b->dFlag, b->dCounters + kCntFlagA,
                                                                 b->dImages, b->dImg, Tg, minScore, minRatio,
                                                                 b->dBest, b->dSec, b->dDecA);
    V3DM_BTRY(cudaGetLastError());
    launches += 1;
  }
  // ---- pass-B layout
  const int chooseGrid = std::max(1, std::min(b->nPairs, 4 * 148));
  k_bcount<<<chooseGrid, kChooseThreads, 0, b->stream>>>(b->dPairs, b->nPairs, b->dDecA, b->dCnt);
  V3DM_BTRY(cudaGetLastError());
  k_bscan<<<1, kScanThreads, 0, b->stream>>>(b->dCnt, b->nPairs, b->dImages, b->nImages, GM, BN, b->capB,
                                             b->capRowsB, b->capTableB, b->dPrefC, b->dImgB, b->dRowsB,
                                             b->dCounters);
  V3DM_BTRY(cudaGetLastError());
  k_bchoose<<<chooseGrid, kChooseThreads, 0, b->stream>>>(b->dPairs, b->nPairs, b->dImages, b->dImgB, b->dPrefC,
                                                          b->dDecA, b->dImg, b->dAB, b->dChosenLeft, b->dChosenRight,
                                                          b->dChosenPair, b->dCounters, 1, 0, 0);
  V3DM_BTRY(cudaGetLastError());
  launches += 3;
  // ---- pass B: the rights the accepted lefts named, against their left image
  sa.aIsLeft = 0;
  sa.rows = b->dRowsB;
  sa.nRowsPtr = b->dCounters + kCntRowsB;
  sa.nRows = (int)std::min<long long>(b->capTableB, 0x7fffffff);
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[2], b->stream));
  V3DM_BTRY(launch_side_batch(b->tc, b->mapsB, sa, b->stream));
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[3], b->stream));
  pa.nRows = (int)std::min<long long>(b->capB, 0x7fffffff);
  pa.rowsPtr = b->dCounters + kCntStates;
  pa.aIsLeft = 0;
  pa.decision = b->dDecB;
  if (gated) pa.flaggedCount = b->dCounters + kCntFlagB;
  V3DM_BTRY(launch_post(pa, b->stream));
  launches += 4;
  if (gated) {
    k_brescore<<<rescoreGrid, kBRescoreThreads, 0, b->stream>>>(*bg, 0, b->dFlag, b->dCounters + kCntFlagB,
                                                                 b->dImages, b->dImg, Tg, minScore, minRatio,
                                                                 b->dBest, b->dSec, b->dDecB);
    V3DM_BTRY(cudaGetLastError());
    launches += 1;
  }
  // ---- mutual filter, ordered triples
  const int mutBlocks = (int)((b->capB + kBMutPerBlock - 1) / kBMutPerBlock);
  k_bmutual_count<<<mutBlocks, kBMutThreads, 0, b->stream>>>(b->dCounters, b->dDecB, b->dChosenLeft, b->dBlockCount);
  V3DM_BTRY(cudaGetLastError());
  k_bmutual_write<<<mutBlocks, kBMutThreads, 0, b->stream>>>(b->dCounters, b->dDecB, b->dChosenLeft,
                                                             b->dChosenRight, b->dChosenPair, b->dBlockCount,
                                                             mutBlocks, b->dOut, b->dInfo);
  V3DM_BTRY(cudaGetLastError());
  launches += 2;
  V3DM_BTRY(cudaMemcpyAsync(b->hInfo, b->dInfo, (kInfoWords + kCntAll) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            b->stream));
  b->lastLaunches = launches;
  return V3DM_OK;
}

// Enqueues one batch call on the float layouts: the passes of enqueue_batch with the float side
// kernel, which writes every state's decision itself (one CTA scores a whole row, so the exact
// best and second of each descriptor stay in registers): no chunk records, no re-score.  With bg
// set, the call is guided: each pair's gate masks its scores in both passes.
int enqueue_batch_f(v3dm_batch* b, float minScore, float minRatio, bool withEvents,
                    const BatchGateArgs* bg = nullptr) {
  const int GM = f_group_rows(), BN = f_tile_cols();
  const float Tf = host_float_threshold(minScore, minRatio);
  int launches = 0;
  V3DM_BTRY(cudaMemsetAsync(b->dInfo, 0, (kInfoWords + kCntAll) * sizeof(int32_t), b->stream));
  // pairs whose right image is empty have no rows: their lefts decide 'none'
  V3DM_BTRY(cudaMemsetAsync(b->dDecA, 0xff, (size_t)std::max<long long>(b->SA, 1) * sizeof(int32_t), b->stream));
  SideArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.err = b->dInfo + kInfoErr;
  sa.minScore = minScore;
  sa.minRatio = minRatio;
  if (bg) sa.bg = *bg;
  // ---- pass A: every (pair, group of 128 lefts) against the pair's right image
  sa.aIsLeft = 1;
  sa.rows = b->dRowsA;
  sa.nRows = b->nRowsA;
  sa.decision = b->dDecA;
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[0], b->stream));
  V3DM_BTRY(launch_side_f_batch(b->fmA_A, b->fmA_B, sa, Tf, b->numSMs, b->stream));
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[1], b->stream));
  launches += b->nRowsA > 0;
  // ---- pass-B layout: the chosen rights' A rows (six planes)
  const int chooseGrid = std::max(1, std::min(b->nPairs, 4 * 148));
  k_bcount<<<chooseGrid, kChooseThreads, 0, b->stream>>>(b->dPairs, b->nPairs, b->dDecA, b->dCnt);
  V3DM_BTRY(cudaGetLastError());
  k_bscan<<<1, kScanThreads, 0, b->stream>>>(b->dCnt, b->nPairs, b->dImages, b->nImages, GM, BN, b->capB,
                                             b->capRowsB, b->capTableB, b->dPrefC, b->dImgB, b->dRowsB,
                                             b->dCounters);
  V3DM_BTRY(cudaGetLastError());
  k_bchoose<<<chooseGrid, kChooseThreads, 0, b->stream>>>(b->dPairs, b->nPairs, b->dImages, b->dImgB, b->dPrefC,
                                                          b->dDecA, b->dFA, b->dFAB, b->dChosenLeft, b->dChosenRight,
                                                          b->dChosenPair, b->dCounters, kFloatRowBytes / kDescBytes,
                                                          b->fRows, b->capRowsB);
  V3DM_BTRY(cudaGetLastError());
  launches += 3;
  // ---- pass B: the rights the accepted lefts named, against their left image
  sa.aIsLeft = 0;
  sa.rows = b->dRowsB;
  sa.nRowsPtr = b->dCounters + kCntRowsB;
  sa.nRows = (int)std::min<long long>(b->capTableB, 0x7fffffff);
  sa.decision = b->dDecB;
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[2], b->stream));
  V3DM_BTRY(launch_side_f_batch(b->fmB_A, b->fmB_B, sa, Tf, b->numSMs, b->stream));
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[3], b->stream));
  launches += 1;
  // ---- mutual filter, ordered triples
  const int mutBlocks = (int)((b->capB + kBMutPerBlock - 1) / kBMutPerBlock);
  k_bmutual_count<<<mutBlocks, kBMutThreads, 0, b->stream>>>(b->dCounters, b->dDecB, b->dChosenLeft, b->dBlockCount);
  V3DM_BTRY(cudaGetLastError());
  k_bmutual_write<<<mutBlocks, kBMutThreads, 0, b->stream>>>(b->dCounters, b->dDecB, b->dChosenLeft,
                                                             b->dChosenRight, b->dChosenPair, b->dBlockCount,
                                                             mutBlocks, b->dOut, b->dInfo);
  V3DM_BTRY(cudaGetLastError());
  launches += 2;
  V3DM_BTRY(cudaMemcpyAsync(b->hInfo, b->dInfo, (kInfoWords + kCntAll) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            b->stream));
  b->lastLaunches = launches;
  return V3DM_OK;
}

// The float passes' rows, pass-B operand and tensor maps.
int prepare_float(v3dm_batch* b) {
  if (b->rowsDirty || b->rowsCfg != kFloatRowsCfg) {
    int st = build_rows(b, f_group_rows(), f_tile_cols(), kFloatRowsCfg);
    if (st != V3DM_OK) return st;
  }
  if (b->totalRows == 0) return V3DM_OK;
  const long long need = (long long)kFloatRowBytes * b->capRowsB;
  if (b->fabCap < need || !b->dFAB) {
    V3DM_BTRY(ensure(&b->dFAB, &b->fabCap, need));
    b->fMapsValid = false;
  }
  if (!b->fMapsValid) {
    V3DM_BTRY(f_maps(&b->fmA_A, b->dFA, b->fRows, &b->fmA_B, b->dFB, b->fRows));
    V3DM_BTRY(f_maps(&b->fmB_A, b->dFAB, (int)b->capRowsB, &b->fmB_B, b->dFB, b->fRows));
    b->fMapsValid = true;
  }
  return V3DM_OK;
}

int prepare(v3dm_batch* b) {
  if (!b->haveImages || !b->havePairs) return V3DM_ERR_NOT_ALLOCATED;
  if (b->floatMode) return prepare_float(b);
  if (b->rowsDirty || b->rowsCfg != tc_get_config(b->tc)) {
    int GM = 0, BN = 0;
    tc_config_shape(tc_get_config(b->tc), &GM, &BN);
    int st = build_rows(b, GM, BN, tc_get_config(b->tc));
    if (st != V3DM_OK) return st;
  }
  if (b->totalRows > 0) {
    int st = ensure_maps(b);
    if (st != V3DM_OK) return st;
  }
  V3DM_BTRY(tc_prepare_batch(b->tc, tc_get_config(b->tc)));
  return V3DM_OK;
}

int enqueue_call(v3dm_batch* b, float minScore, float minRatio, bool withEvents) {
  return b->floatMode ? enqueue_batch_f(b, minScore, minRatio, withEvents)
                      : enqueue_batch(b, minScore, minRatio, withEvents);
}

// One call: graph replay (or direct launches), then nothing else; the info block lands in
// hInfo when the stream reaches it.
int launch_call(v3dm_batch* b, float minScore, float minRatio) {
  int st = prepare(b);
  if (st != V3DM_OK) return st;
  b->pendingCheck = true;
  if (b->totalRows == 0 || b->nPairs == 0) {
    V3DM_BTRY(cudaMemsetAsync(b->dInfo, 0, (kInfoWords + kCntAll) * sizeof(int32_t), b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->hInfo, b->dInfo, (kInfoWords + kCntAll) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                              b->stream));
    b->lastLaunches = 0;
    return V3DM_OK;
  }
  uint32_t ms, mr;
  std::memcpy(&ms, &minScore, 4);
  std::memcpy(&mr, &minRatio, 4);
  if (b->profile) {
    for (int i = 0; i < 4; ++i)
      if (!b->ev[i]) V3DM_BTRY(cudaEventCreate(&b->ev[i]));
    st = enqueue_call(b, minScore, minRatio, true);
    if (st == V3DM_OK) b->profPending = true;
    return st;
  }
  if (!b->useGraph) return enqueue_call(b, minScore, minRatio, false);
  if (!b->graph || b->graphMs != ms || b->graphMr != mr) {
    drop_graph(b);
    cudaGraph_t g = nullptr;
    V3DM_BTRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    st = enqueue_call(b, minScore, minRatio, false);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st != V3DM_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return bfail(e, "cudaStreamEndCapture", __LINE__);
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->graph = nullptr;
      return bfail(e, "cudaGraphInstantiate", __LINE__);
    }
    b->graphMs = ms;
    b->graphMr = mr;
    b->graphLaunches = b->lastLaunches;
  }
  V3DM_BTRY(cudaGraphLaunch(b->graph, b->stream));
  b->lastLaunches = b->graphLaunches;
  return V3DM_OK;
}

// Waits for the last call and checks its info block.  Grows the buffers and returns
// V3DM_ERR_CANDIDATES when a list or a pass-B buffer overflowed (the call must be repeated).
int finish_call(v3dm_batch* b) {
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  b->pendingCheck = false;
  if (b->profPending) {
    float a = 0.f, c = 0.f;
    V3DM_BTRY(cudaEventElapsedTime(&a, b->ev[0], b->ev[1]));
    V3DM_BTRY(cudaEventElapsedTime(&c, b->ev[2], b->ev[3]));
    b->profMs[0] += a;
    b->profMs[1] += c;
    ++b->profN[0];
    ++b->profN[1];
    b->profPending = false;
  }
  const int32_t* info = b->hInfo;
  const int32_t* cnt = b->hInfo + kInfoWords;
  if (info[kInfoErr] & kErrWaitTimeout) return V3DM_ERR_TIMEOUT;
  if (info[kInfoErr]) return V3DM_ERR_CUDA;
  bool grow = false;
  if ((long long)info[kInfoMaxSeg] > b->segCap) {
    long long cap = std::max<long long>(2 * b->segCap, (long long)info[kInfoMaxSeg] * 5 / 4 + 16);
    V3DM_BTRY(alloc_records(b, cap));
    grow = true;
  }
  if (cnt[kCntOverP]) {
    b->rowsPNeed = std::max<long long>(2 * b->rowsPCap, 1024);
    grow = true;
  }
  if (cnt[kCntOverflow]) {
    long long need = std::max<long long>((long long)cnt[kCntNeedStates] * 5 / 4 + 1024, 2 * b->capB);
    V3DM_BTRY(alloc_passB(b, need));
    b->mapsValid = false;
    grow = true;
  }
  if (grow) {
    drop_graph(b);
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
    return V3DM_ERR_CANDIDATES;
  }
  return V3DM_OK;
}

// One guided call (no graph): the flagged-state buffer, the gate arguments, the launches.
int launch_call_guided(v3dm_batch* b, int type, float minScore, float minRatio) {
  int st = prepare(b);
  if (st != V3DM_OK) return st;
  b->pendingCheck = true;
  if (b->totalRows == 0 || b->nPairs == 0) {
    V3DM_BTRY(cudaMemsetAsync(b->dInfo, 0, (kInfoWords + kCntAll) * sizeof(int32_t), b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->hInfo, b->dInfo, (kInfoWords + kCntAll) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                              b->stream));
    b->lastLaunches = 0;
    return V3DM_OK;
  }
  V3DM_BTRY(ensure(&b->dFlag, &b->flagCap, std::max<long long>(std::max(b->SA, b->capB), 1)));
  BatchGateArgs bg;
  std::memset(&bg, 0, sizeof(bg));
  bg.on = 1;
  bg.type = type;
  bg.gm = b->dGate;
  bg.pairLR = b->dPairLR;
  bg.pos = b->dPos;
  bg.posOff = b->dSrcOff;
  bg.stateA0 = b->dStateA0;
  bg.origOf = b->dOrigOf;
  bg.nPairs = b->nPairs;
  bg.chosenPair = b->dChosenPair;
  bg.chosenRight = b->dChosenRight;
  if (b->profile) {
    for (int i = 0; i < 4; ++i)
      if (!b->ev[i]) V3DM_BTRY(cudaEventCreate(&b->ev[i]));
  }
  st = b->floatMode ? enqueue_batch_f(b, minScore, minRatio, b->profile, &bg)
                    : enqueue_batch(b, minScore, minRatio, b->profile, &bg);
  if (st == V3DM_OK && b->profile) b->profPending = true;
  return st;
}

int run_host(v3dm_batch* b, float minScore, float minRatio) {
  for (int attempt = 0; attempt < 6; ++attempt) {
    int st = launch_call(b, minScore, minRatio);
    if (st != V3DM_OK) return st;
    st = finish_call(b);
    if (st != V3DM_ERR_CANDIDATES) return st;
  }
  return V3DM_ERR_CANDIDATES;
}

// ---- proposal matching ----------------------------------------------------------------

// Buffers and tensor maps of a proposal call with 'probes' probed cells and C cells.
int prepare_proposal(v3dm_batch* b, int probesL, int probesR, int C) {
  const int probes = std::max(probesL, probesR);
  int st = prepare(b);
  if (st != V3DM_OK) return st;
  int GM = 0, BN = 0;
  tc_config_shape(tc_get_config(b->tc), &GM, &BN);
  const long long laRows = std::max<long long>(b->totalDesc * probesL, 256);
  const long long lbRows = std::max<long long>(b->totalDesc * probesR, 256);
  long long rowsBound = 0;
  for (const BPair& q : b->bp)
    if (b->counts[q.ri] > 0 && q.nL > 0) rowsBound += ((long long)q.nL * probesL + GM - 1) / GM + C;
  rowsBound = std::max<long long>(std::max(rowsBound, b->rowsPNeed), 1);
  if (rowsBound > 0x7fffffffLL || laRows > 0x7fffffffLL) return V3DM_ERR_SIZE;
  const uint8_t* la0 = b->dLA;
  const uint8_t* lb0 = b->dLB;
  const BatchRow* rp0 = b->dRowsP;
  V3DM_BTRY(ensure(&b->dCell, &b->cellCap, std::max<long long>(b->totalRows, 1) * probes));
  const long long tab = (long long)std::max(b->nImages, 1) * C;
  if (tab > b->cellTabCap) {
    long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    bfree(b->dCntA);
    bfree(b->dCntB);
    bfree(b->dOffA);
    bfree(b->dOffB);
    b->cellTabCap = 0;
    V3DM_BTRY(ensure(&b->dCntA, &c0, tab));
    V3DM_BTRY(ensure(&b->dCntB, &c1, tab));
    V3DM_BTRY(ensure(&b->dOffA, &c2, tab));
    V3DM_BTRY(ensure(&b->dOffB, &c3, tab));
    b->cellTabCap = tab;
  }
  V3DM_BTRY(ensure(&b->dLA, &b->laCap, laRows * kDescBytes));
  V3DM_BTRY(ensure(&b->dMapA, &b->mapACap, laRows));
  V3DM_BTRY(ensure(&b->dLB, &b->lbCap, lbRows * kDescBytes));
  V3DM_BTRY(ensure(&b->dMapB, &b->mapBCap, lbRows));
  if (tab > b->pairTabCap) {  // one entry per (cell, left image) unit
    long long c0 = 0, c1 = 0;
    bfree(b->dRowCnt);
    bfree(b->dRowStart);
    b->pairTabCap = 0;
    V3DM_BTRY(ensure(&b->dRowCnt, &c0, tab));
    V3DM_BTRY(ensure(&b->dRowStart, &c1, tab));
    b->pairTabCap = tab;
  }
  V3DM_BTRY(ensure(&b->dRowsP, &b->rowsPCap, rowsBound));
  // exact verification: one entry per state on each side, per-image tables
  const long long imgTab = (long long)std::max(b->nImages, 1) + 1;
  if (imgTab > b->unitTabCap) {
    long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    bfree(b->dCntE);
    bfree(b->dOffE);
    bfree(b->dRowStartE);
    bfree(b->dRowStartR);
    b->unitTabCap = 0;
    V3DM_BTRY(ensure(&b->dCntE, &c0, imgTab));
    V3DM_BTRY(ensure(&b->dOffE, &c1, imgTab));
    V3DM_BTRY(ensure(&b->dRowStartE, &c2, imgTab));
    V3DM_BTRY(ensure(&b->dRowStartR, &c3, imgTab));
    V3DM_BTRY(cudaMemsetAsync(b->dCntE, 0, (size_t)imgTab * sizeof(int), b->stream));
    b->unitTabCap = imgTab;
  }
  const long long entries = std::max<long long>(b->capB, 1);
  if (entries > 0x7fffffffLL) return V3DM_ERR_SIZE;
  if (entries > b->entryCap) {
    long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    bfree(b->dSrcRowE);
    bfree(b->dStateE);
    bfree(b->dSrcRowR);
    bfree(b->dDecL);
    b->entryCap = 0;
    V3DM_BTRY(ensure(&b->dSrcRowE, &c0, entries));
    V3DM_BTRY(ensure(&b->dStateE, &c1, entries));
    V3DM_BTRY(ensure(&b->dSrcRowR, &c2, entries));
    V3DM_BTRY(ensure(&b->dDecL, &c3, entries));
    b->entryCap = entries;
  }
  V3DM_BTRY(ensure(&b->dRowsPB, &b->rowsPBCap, entries / tc_gather_rows() + imgTab + 1));
  if (b->dLA != la0 || b->dLB != lb0 || b->dRowsP != rp0 || !b->mapsPValid || b->laRows != laRows ||
      b->lbRows != lbRows || b->mapsP.cfg != tc_get_config(b->tc)) {
    V3DM_BTRY(tc_side_maps(b->tc, &b->mapsP, b->dLA, (int)laRows, b->dLB, (int)lbRows));
    b->mapsPValid = true;
    b->laRows = laRows;
    b->lbRows = lbRows;
    if (b->graphP) cudaGraphExecDestroy(b->graphP);
    b->graphP = nullptr;
  }
  if (b->mapImgGimg != b->dImg || b->mapImgGrows != b->totalRows) {
    V3DM_BTRY(tc_gather_map(&b->mapImgG, b->dImg, (int)std::max<long long>(b->totalRows, 1)));
    b->mapImgGimg = b->dImg;
    b->mapImgGrows = b->totalRows;
    if (b->graphP) cudaGraphExecDestroy(b->graphP);
    b->graphP = nullptr;
  }
  return V3DM_OK;
}

int enqueue_proposal(v3dm_batch* b, const v3dm_projection* proj, int probesL, int probesR, float minScore,
                     float minRatio, bool withEvents) {
  const int probes = std::max(probesL, probesR);
  int GM = 0, BN = 0;
  tc_config_shape(tc_get_config(b->tc), &GM, &BN);
  const int C = proj_cells(proj);
  const int32_t Smin = host_smallest_passing_score(minScore);
  const int nI = b->nImages;
  const int imgGrid = std::max(1, std::min(nI, 1024));
  int launches = 0;
  V3DM_BTRY(cudaMemsetAsync(b->dInfo, 0, (kInfoWords + kCntAll) * sizeof(int32_t), b->stream));
  // cells of every descriptor, layouts, row table
  V3DM_BTRY(proj_assign(proj, b->dImg, b->totalRows, probes, b->dCell, b->stream));
  k_pcount<<<imgGrid, 256, 2 * C * sizeof(int), b->stream>>>(b->dImages, nI, b->dCell, probes, probesL, probesR, C,
                                                             b->dCntA, b->dCntB);
  V3DM_BTRY(cudaGetLastError());
  k_pscan_cells<<<1, kScanThreads, 0, b->stream>>>(b->dCntA, b->dCntB, nI * C, b->dOffA, b->dOffB);
  V3DM_BTRY(cudaGetLastError());
  k_pscatter<<<imgGrid, 256, 2 * C * sizeof(int), b->stream>>>(b->dImages, nI, b->dCell, probes, probesL, probesR, C,
                                                               b->dOffA,
                                                               b->dOffB, b->dImg, b->dLA, b->dMapA, b->dLB, b->dMapB);
  V3DM_BTRY(cudaGetLastError());
  const int unitGrid = std::max(1, std::min((nI * C + 7) / 8, 4 * 148));
  k_prowcount<<<unitGrid, 256, 0, b->stream>>>(b->dPairs, b->dImages, nI, C, GM, b->dCntA, b->dCntB, b->dRowCnt,
                                               reinterpret_cast<unsigned long long*>(b->dCounters + kCntScored));
  V3DM_BTRY(cudaGetLastError());
  k_pscan_rows<<<1, kScanThreads, 0, b->stream>>>(b->dRowCnt, nI * C, b->rowsPCap, b->dRowStart, b->dCounters);
  V3DM_BTRY(cudaGetLastError());
  k_prows<<<unitGrid, 256, 0, b->stream>>>(b->dPairs, b->dImages, nI, C, GM, BN, b->dCntA, b->dCntB, b->dOffA,
                                           b->dOffB, b->dRowStart, b->dCounters, b->dRowsP);
  V3DM_BTRY(cudaGetLastError());
  launches += 7;
  // pass A: each left against the rights under its probed cells
  SideArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.Smin = Smin;
  if (host_candidate_threshold(minScore, minRatio, false, &sa.Tsec) != V3DM_OK) sa.Tsec = 0;
  sa.records = b->dRecords;
  sa.segCount = b->dSegCount;
  sa.segCap = b->segCap;
  sa.nSeg = b->nSeg;
  sa.err = b->dInfo + kInfoErr;
  sa.aIsLeft = 1;
  sa.best = b->dBest;
  sa.sec = b->dSec;
  sa.amap = b->dMapA;
  sa.rows = b->dRowsP;
  sa.nRowsPtr = b->dCounters + kCntRowsP;
  sa.nRows = (int)b->rowsPCap;
  sa.schedule = b->schedule;
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[0], b->stream));
  V3DM_BTRY(launch_side_batch(b->tc, b->mapsP, sa, b->stream));
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[1], b->stream));
  PostArgs pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.records = b->dRecords;
  pa.bmap = b->dMapB;
  pa.segCount = b->dSegCount;
  pa.segCap = b->segCap;
  pa.nSeg = b->nSeg;
  pa.Smin = Smin;
  pa.minScore = minScore;
  pa.minRatio = minRatio;
  pa.best = b->dBest;
  pa.sec = b->dSec;
  pa.err = b->dInfo + kInfoErr;
  pa.nRows = (int)b->SA;
  pa.aIsLeft = 1;
  pa.decision = b->dDecA;
  V3DM_BTRY(launch_post(pa, b->stream));
  launches += 3;
  // pass-B states: the accepted lefts of every pair, in pair order
  const int chooseGrid = std::max(1, std::min(b->nPairs, 4 * 148));
  k_bcount<<<chooseGrid, kChooseThreads, 0, b->stream>>>(b->dPairs, b->nPairs, b->dDecA, b->dCnt);
  V3DM_BTRY(cudaGetLastError());
  k_pscan_states<<<1, kScanThreads, 0, b->stream>>>(b->dCnt, b->nPairs, b->capB, b->dPrefC, b->dCounters);
  V3DM_BTRY(cudaGetLastError());
  k_pchoose<<<chooseGrid, kChooseThreads, 0, b->stream>>>(b->dPairs, b->nPairs, b->dPrefC, b->dDecA, b->dChosenLeft,
                                                          b->dChosenRight, b->dChosenPair, b->dChosenSorted,
                                                          b->dCounters);
  V3DM_BTRY(cudaGetLastError());
  // exact verification of every state over the full score matrix of its pair
  const int GR = tc_gather_rows(), BNG = tc_gather_cols();
  const int stateGrid = 4 * 148;
  const int imgBlocks = std::max(1, (nI + 255) / 256);
  k_vcount<<<stateGrid, 256, 0, b->stream>>>(b->dPairs, b->dChosenSorted, b->dCounters, b->dCntE);
  V3DM_BTRY(cudaGetLastError());
  k_vscan<<<1, kScanThreads, 0, b->stream>>>(b->dCntE, b->dImages, nI, b->dPrefC, GR, b->rowsPBCap, b->dOffE,
                                             b->dRowStartE, b->dRowStartR, b->dCounters);
  V3DM_BTRY(cudaGetLastError());
  k_vscatter<<<stateGrid, 256, 0, b->stream>>>(b->dPairs, b->dImages, b->dChosenLeft, b->dChosenSorted, b->dCounters,
                                               b->dOffE, b->dCntE, b->dSrcRowE, b->dStateE);
  V3DM_BTRY(cudaGetLastError());
  k_vrows_left<<<imgBlocks, 256, 0, b->stream>>>(b->dImages, nI, GR, BNG, b->dOffE, b->dRowStartE, b->dCounters,
                                                 b->dRowsPB);
  V3DM_BTRY(cudaGetLastError());
  SideArgs sv;
  std::memset(&sv, 0, sizeof(sv));
  sv.Smin = Smin;
  if (host_candidate_threshold(minScore, minRatio, false, &sv.Tsec) != V3DM_OK) sv.Tsec = 0;
  sv.records = b->dRecords;
  sv.segCount = b->dSegCount;
  sv.segCap = b->segCap;
  sv.nSeg = b->nSeg;
  sv.err = b->dInfo + kInfoErr;
  sv.best = b->dBest;
  sv.sec = b->dSec;
  sv.schedule = 2;
  sv.aSrc = b->dImg;
  sv.nRows = (int)std::min<long long>(b->rowsPBCap, 0x7fffffff);
  // V-left: each state's left against every right of its pair's right image
  sv.aIsLeft = 1;
  sv.amap = b->dStateE;
  sv.aSrcRow = b->dSrcRowE;
  sv.rows = b->dRowsPB;
  sv.nRowsPtr = b->dCounters + kCntRowsVL;
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[2], b->stream));
  V3DM_BTRY(launch_side_gather(b->tc, b->mapImgG, sv, b->stream));
  PostArgs pv;
  std::memset(&pv, 0, sizeof(pv));
  pv.records = b->dRecords;
  pv.segCount = b->dSegCount;
  pv.segCap = b->segCap;
  pv.nSeg = b->nSeg;
  pv.Smin = Smin;
  pv.minScore = minScore;
  pv.minRatio = minRatio;
  pv.best = b->dBest;
  pv.sec = b->dSec;
  pv.err = b->dInfo + kInfoErr;
  pv.nRows = (int)std::min<long long>(b->capB, 0x7fffffff);
  pv.rowsPtr = b->dCounters + kCntStates;
  pv.aIsLeft = 1;
  pv.decision = b->dDecL;
  V3DM_BTRY(launch_post(pv, b->stream));
  // V-right: the right each exact left decision named, against every left of the pair's left image
  k_vsrc_right<<<stateGrid, 256, 0, b->stream>>>(b->dPairs, b->dImages, b->dChosenSorted, b->dDecL, b->dCounters,
                                                 b->dSrcRowR);
  V3DM_BTRY(cudaGetLastError());
  k_vrows_right<<<imgBlocks, 256, 0, b->stream>>>(b->dImages, nI, b->dPrefC, GR, BNG, b->dRowStartR, b->dCounters,
                                                  b->dRowsPB);
  V3DM_BTRY(cudaGetLastError());
  sv.aIsLeft = 0;
  sv.amap = nullptr;
  sv.aSrcRow = b->dSrcRowR;
  sv.nRowsPtr = b->dCounters + kCntRowsVR;
  V3DM_BTRY(launch_side_gather(b->tc, b->mapImgG, sv, b->stream));
  if (withEvents) V3DM_BTRY(cudaEventRecord(b->ev[3], b->stream));
  pv.aIsLeft = 0;
  pv.decision = b->dDecB;
  V3DM_BTRY(launch_post(pv, b->stream));
  k_vmerge<<<stateGrid, 256, 0, b->stream>>>(b->dCounters, b->dDecL, b->dChosenLeft, b->dChosenRight, b->dDecB);
  V3DM_BTRY(cudaGetLastError());
  launches += 13;  // four V-left layout kernels, two gathered side passes with their records and decisions,
                   // two V-right layout kernels, the merge
  const int mutBlocks = (int)((b->capB + kBMutPerBlock - 1) / kBMutPerBlock);
  k_bmutual_count<<<mutBlocks, kBMutThreads, 0, b->stream>>>(b->dCounters, b->dDecB, b->dChosenLeft, b->dBlockCount);
  V3DM_BTRY(cudaGetLastError());
  k_bmutual_write<<<mutBlocks, kBMutThreads, 0, b->stream>>>(b->dCounters, b->dDecB, b->dChosenLeft,
                                                             b->dChosenRight, b->dChosenPair, b->dBlockCount,
                                                             mutBlocks, b->dOut, b->dInfo);
  V3DM_BTRY(cudaGetLastError());
  launches += 5;  // pass-B states (count, scan, choose), mutual filter (two)
  V3DM_BTRY(cudaMemcpyAsync(b->hInfo, b->dInfo, (kInfoWords + kCntAll) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            b->stream));
  b->lastLaunches = launches;
  return V3DM_OK;
}

int launch_call_proposal(v3dm_batch* b, const v3dm_projection* proj, int probesL, int probesR, float minScore,
                         float minRatio) {
  if (!proj || probesL < 1 || probesL > V3DM_PROJ_MAX_PROBES || probesR < 1 || probesR > V3DM_PROJ_MAX_PROBES)
    return V3DM_ERR_ARG;
  const int C = proj_cells(proj);
  if (C < 1) return V3DM_ERR_NOT_ALLOCATED;
  if (probesL > C || probesR > C) return V3DM_ERR_ARG;
  const int probes = probesL * 16 + probesR;  // graph key
  if (!b->haveImages || !b->havePairs) return V3DM_ERR_NOT_ALLOCATED;
  if (b->floatMode) return V3DM_ERR_UNSUPPORTED;
  b->pendingCheck = true;
  if (b->totalRows == 0 || b->nPairs == 0) {
    V3DM_BTRY(cudaMemsetAsync(b->dInfo, 0, (kInfoWords + kCntAll) * sizeof(int32_t), b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->hInfo, b->dInfo, (kInfoWords + kCntAll) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                              b->stream));
    b->lastLaunches = 0;
    return V3DM_OK;
  }
  int st = prepare_proposal(b, probesL, probesR, C);
  if (st != V3DM_OK) return st;
  // the projection's parameters and cells may have been written on its own stream
  V3DM_BTRY(cudaStreamSynchronize(proj_stream(proj)));
  uint32_t ms, mr;
  std::memcpy(&ms, &minScore, 4);
  std::memcpy(&mr, &minRatio, 4);
  if (b->profile) {
    for (int i = 0; i < 4; ++i)
      if (!b->ev[i]) V3DM_BTRY(cudaEventCreate(&b->ev[i]));
    st = enqueue_proposal(b, proj, probesL, probesR, minScore, minRatio, true);
    if (st == V3DM_OK) b->profPending = true;
    return st;
  }
  if (!b->useGraph) return enqueue_proposal(b, proj, probesL, probesR, minScore, minRatio, false);
  if (!b->graphP || b->gpMs != ms || b->gpMr != mr || b->gpProbes != probes || b->gpCells != C || b->gpProj != proj) {
    if (b->graphP) cudaGraphExecDestroy(b->graphP);
    b->graphP = nullptr;
    cudaGraph_t g = nullptr;
    V3DM_BTRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    st = enqueue_proposal(b, proj, probesL, probesR, minScore, minRatio, false);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st != V3DM_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return bfail(e, "cudaStreamEndCapture", __LINE__);
    e = cudaGraphInstantiate(&b->graphP, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->graphP = nullptr;
      return bfail(e, "cudaGraphInstantiate", __LINE__);
    }
    b->gpMs = ms;
    b->gpMr = mr;
    b->gpProbes = probes;
    b->gpCells = C;
    b->gpProj = proj;
    b->gpLaunches = b->lastLaunches;
  }
  V3DM_BTRY(cudaGraphLaunch(b->graphP, b->stream));
  b->lastLaunches = b->gpLaunches;
  return V3DM_OK;
}

void free_all(v3dm_batch* b) {
  drop_graph(b);
  bfree(b->dImg);
  bfree(b->dStage);
  bfree(b->dSrcOff);
  bfree(b->dImages);
  bfree(b->dPairs);
  bfree(b->dRowsA);
  bfree(b->dBest);
  bfree(b->dSec);
  bfree(b->dDecA);
  bfree(b->dRecords);
  bfree(b->dList);
  bfree(b->dSegCount);
  bfree(b->dCnt);
  bfree(b->dPrefC);
  bfree(b->dImgB);
  bfree(b->dAB);
  bfree(b->dRowsB);
  bfree(b->dDecB);
  bfree(b->dChosenLeft);
  bfree(b->dChosenRight);
  bfree(b->dChosenPair);
  bfree(b->dBlockCount);
  bfree(b->dOut);
  bfree(b->dCell);
  bfree(b->dCntA);
  bfree(b->dCntB);
  bfree(b->dOffA);
  bfree(b->dOffB);
  bfree(b->dLA);
  bfree(b->dMapA);
  bfree(b->dLB);
  bfree(b->dMapB);
  bfree(b->dRowCnt);
  bfree(b->dRowStart);
  bfree(b->dCntE);
  bfree(b->dOffE);
  bfree(b->dRowStartE);
  bfree(b->dSrcRowE);
  bfree(b->dStateE);
  bfree(b->dSrcRowR);
  bfree(b->dDecL);
  bfree(b->dRowStartR);
  bfree(b->dRowsPB);
  bfree(b->dRowsP);
  bfree(b->dChosenSorted);
  bfree(b->dPos);
  bfree(b->dGate);
  bfree(b->dPairLR);
  bfree(b->dStateA0);
  bfree(b->dOrigOf);
  bfree(b->dFlag);
  bfree(b->dStageF);
  bfree(b->dRowOffI);
  bfree(b->dFA);
  bfree(b->dFB);
  bfree(b->dFAB);
  b->dCounters = nullptr;  // points into dInfo
  bfree(b->dInfo);
  if (b->hInfo) cudaFreeHost(b->hInfo);
  b->hInfo = nullptr;
}

// Switches between the uint8 and the float layouts; the graph and the row tables of the other
// mode are dropped.
void set_float_mode(v3dm_batch* b, bool on) {
  if (b->floatMode == on) return;
  drop_graph(b);
  b->floatMode = on;
  b->rowsDirty = true;
  b->fMapsValid = false;
}

// Layout of the images: padded row offsets, per-image table.
int set_images(v3dm_batch* b, int nImages, const int32_t* counts, const uint8_t* desc, bool onDevice) {
  if (!b || nImages < 0 || (nImages > 0 && !counts)) return V3DM_ERR_ARG;
  long long total = 0, rows = 0;
  for (int i = 0; i < nImages; ++i) {
    if (counts[i] < 0) return V3DM_ERR_ARG;
    if (counts[i] > V3DM_MAX_FEATURES) return V3DM_ERR_SIZE;
    total += counts[i];
    rows += ((long long)counts[i] + 255) / 256 * 256;
  }
  if (total > 0 && !desc) return V3DM_ERR_ARG;
  if (onDevice && (reinterpret_cast<uintptr_t>(desc) & 15)) return V3DM_ERR_ARG;
  if (rows > 0x7fffff00LL) return V3DM_ERR_SIZE;
  BDeviceGuard g(b->device);
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  b->havePositions = false;  // positions belong to the images
  // Same image sizes as before: the padded layout, the pair table and the row tables stay
  // valid, only the descriptors change (the graph reads them from the same buffer).
  const bool sameLayout = b->haveImages && nImages == b->nImages && std::equal(counts, counts + nImages, b->counts.begin());
  if (sameLayout) {
    if (total > 0) {
      const uint8_t* src = desc;
      if (!onDevice) {
        V3DM_BTRY(ensure(&b->dStage, &b->stageCap, total * kDescBytes));
        V3DM_BTRY(cudaMemcpyAsync(b->dStage, desc, (size_t)total * kDescBytes, cudaMemcpyHostToDevice, b->stream));
        src = b->dStage;
      }
      k_bscatter<<<std::min(nImages, 1024), 256, 0, b->stream>>>(src, b->dSrcOff, b->dImages, nImages, b->dImg);
      V3DM_BTRY(cudaGetLastError());
    }
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
    return V3DM_OK;
  }
  drop_graph(b);
  b->haveImages = false;
  b->havePairs = false;  // pairs index the old images
  b->nImages = nImages;
  b->counts.assign(counts, counts + nImages);
  b->srcOff.assign(nImages, 0);
  b->rowOff.assign(nImages, 0);
  long long so = 0, ro = 0;
  for (int i = 0; i < nImages; ++i) {
    b->srcOff[i] = so;
    b->rowOff[i] = (int)ro;
    so += counts[i];
    ro += ((long long)counts[i] + 255) / 256 * 256;
  }
  b->totalDesc = total;
  b->totalRows = rows;
  V3DM_BTRY(ensure(&b->dImg, &b->imgCap, std::max<long long>(rows, 256) * kDescBytes));
  if (nImages > b->imagesCap) {
    bfree(b->dSrcOff);
    bfree(b->dImages);
    bfree(b->dImgB);
    b->imagesCap = 0;
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dSrcOff), (size_t)nImages * sizeof(long long)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dImages), (size_t)nImages * sizeof(BImage)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dImgB), (size_t)nImages * sizeof(BImageB)));
    b->imagesCap = nImages;
  }
  if (nImages > 0) {
    V3DM_BTRY(cudaMemcpyAsync(b->dSrcOff, b->srcOff.data(), (size_t)nImages * sizeof(long long),
                              cudaMemcpyHostToDevice, b->stream));
    // The per-image table is completed with pair ranges by set_pairs; upload it with empty ranges.
    b->bim.assign(nImages, BImage{});
    for (int i = 0; i < nImages; ++i) b->bim[i] = BImage{b->rowOff[i], counts[i], 0, 0};
    V3DM_BTRY(cudaMemcpyAsync(b->dImages, b->bim.data(), (size_t)nImages * sizeof(BImage), cudaMemcpyHostToDevice,
                              b->stream));
  }
  if (total > 0) {
    const uint8_t* src = desc;
    if (!onDevice) {
      V3DM_BTRY(ensure(&b->dStage, &b->stageCap, total * kDescBytes));
      V3DM_BTRY(cudaMemcpyAsync(b->dStage, desc, (size_t)total * kDescBytes, cudaMemcpyHostToDevice, b->stream));
      src = b->dStage;
    }
    k_bscatter<<<std::min(nImages, 1024), 256, 0, b->stream>>>(src, b->dSrcOff, b->dImages, nImages, b->dImg);
    V3DM_BTRY(cudaGetLastError());
  }
  V3DM_BTRY(cudaStreamSynchronize(b->stream));  // host vectors and the caller's buffer may change after return
  b->haveImages = true;
  b->mapsValid = false;
  b->rowsDirty = true;
  return V3DM_OK;
}

// Float descriptors.  All of the form u/512: the uint8 layout (the integer path, whose scores
// are the float ones exactly).  Otherwise the BF16 hi/lo layouts of every image, at the rows of
// the uint8 layout, scored as the single-pair float matcher scores them.
int set_images_f32(v3dm_batch* b, int nImages, const int32_t* counts, const float* desc, bool onDevice) {
  if (!b || nImages < 0 || (nImages > 0 && !counts)) return V3DM_ERR_ARG;
  long long total = 0;
  for (int i = 0; i < nImages; ++i) {
    if (counts[i] < 0) return V3DM_ERR_ARG;
    if (counts[i] > V3DM_MAX_FEATURES) return V3DM_ERR_SIZE;
    total += counts[i];
  }
  if (total > 0 && !desc) return V3DM_ERR_ARG;
  if (onDevice && (reinterpret_cast<uintptr_t>(desc) & 15)) return V3DM_ERR_ARG;
  if (total > 0x7fffffffLL / kDescBytes) return V3DM_ERR_SIZE;  // value indices of the conversion are int32
  BDeviceGuard g(b->device);
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  int32_t* err = b->dInfo + kInfoErr;
  bool exact = true;
  const float* src = desc;
  if (total > 0) {
    if (!onDevice) {
      V3DM_BTRY(ensure(&b->dStageF, &b->stageFCap, total * kDescBytes));
      V3DM_BTRY(cudaMemcpyAsync(b->dStageF, desc, (size_t)total * kDescBytes * sizeof(float), cudaMemcpyHostToDevice,
                                b->stream));
      src = b->dStageF;
    }
    V3DM_BTRY(ensure(&b->dStage, &b->stageCap, total * kDescBytes));
    V3DM_BTRY(cudaMemsetAsync(err, 0, sizeof(int32_t), b->stream));
    V3DM_BTRY(launch_f32_to_u8(src, b->dStage, (int)total, err, b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->hInfo + kInfoErr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream));
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
    exact = (b->hInfo[kInfoErr] & kErrNotU8) == 0;
    V3DM_BTRY(cudaMemsetAsync(err, 0, sizeof(int32_t), b->stream));
  }
  // the layout (and, for exact descriptors, the integer operand) from the uint8 staging buffer
  int st = set_images(b, nImages, counts, total > 0 ? b->dStage : nullptr, true);
  if (st != V3DM_OK) return st;
  if (exact) {
    set_float_mode(b, false);
    return V3DM_OK;
  }
  b->haveImages = false;
  set_float_mode(b, true);
  b->fMapsValid = false;  // re-encoded before the next call (same buffers: same maps)
  const int fRows = (int)std::max<long long>(b->totalRows, 256);
  const uint8_t* oldA = b->dFA;
  const uint8_t* oldB = b->dFB;
  V3DM_BTRY(ensure(&b->dFA, &b->fImgCapA, (long long)fRows * kFloatRowBytes));
  V3DM_BTRY(ensure(&b->dFB, &b->fImgCapB, (long long)fRows * kFloatRowBytes));
  if (b->dFA != oldA || b->dFB != oldB || b->fRows != fRows) drop_graph(b);  // the graph's maps name the buffers
  b->fRows = fRows;
  V3DM_BTRY(ensure(&b->dRowOffI, &b->rowOffCap, std::max(nImages, 1)));
  V3DM_BTRY(cudaMemcpyAsync(b->dRowOffI, b->rowOff.data(), (size_t)nImages * sizeof(int), cudaMemcpyHostToDevice,
                            b->stream));
  V3DM_BTRY(launch_hilo_images(src, total, b->dSrcOff, b->dRowOffI, nImages, fRows, b->dFA, b->dFB, err, b->stream));
  V3DM_BTRY(cudaMemcpyAsync(b->hInfo + kInfoErr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream));
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  if (b->hInfo[kInfoErr]) {  // a value that is not finite
    cudaMemsetAsync(err, 0, sizeof(int32_t), b->stream);
    cudaStreamSynchronize(b->stream);
    return V3DM_ERR_ARG;
  }
  b->haveImages = true;
  return V3DM_OK;
}

}  // namespace

extern "C" {

int v3dm_batch_create(v3dm_batch** out, int device) {
  if (!out) return V3DM_ERR_ARG;
  *out = nullptr;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return V3DM_ERR_CUDA;
  if (prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_batch* b = new (std::nothrow) v3dm_batch();
  if (!b) return V3DM_ERR_ARG;
  b->device = device;
  b->numSMs = prop.multiProcessorCount;
  BDeviceGuard g(device);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            tc_plan_create(&b->tc, device) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&b->dInfo), (kInfoWords + kCntAll) * sizeof(int32_t)) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&b->hInfo), (kInfoWords + kCntAll) * sizeof(int32_t)) == cudaSuccess;
  if (ok) {
    b->dCounters = b->dInfo + kInfoWords;  // the counter words follow the info words
    ok = alloc_records(b, 256) == cudaSuccess;
  }
  if (!ok) {
    free_all(b);
    if (b->tc) tc_plan_destroy(b->tc);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return V3DM_ERR_CUDA;
  }
  *out = b;
  return V3DM_OK;
}

int v3dm_batch_destroy(v3dm_batch* b) {
  if (!b) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  cudaStreamSynchronize(b->stream);
  free_all(b);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->tc) tc_plan_destroy(b->tc);
  cudaStreamDestroy(b->stream);
  delete b;
  return V3DM_OK;
}

int v3dm_batch_set_images_u8(v3dm_batch* b, int nImages, const int32_t* counts, const uint8_t* desc) {
  const int st = set_images(b, nImages, counts, desc, false);
  if (st == V3DM_OK) set_float_mode(b, false);
  return st;
}

int v3dm_batch_set_images_u8_device(v3dm_batch* b, int nImages, const int32_t* counts, const uint8_t* d_desc) {
  const int st = set_images(b, nImages, counts, d_desc, true);
  if (st == V3DM_OK) set_float_mode(b, false);
  return st;
}

int v3dm_batch_set_images_f32(v3dm_batch* b, int nImages, const int32_t* counts, const float* desc) {
  return set_images_f32(b, nImages, counts, desc, false);
}

int v3dm_batch_set_images_f32_device(v3dm_batch* b, int nImages, const int32_t* counts, const float* d_desc) {
  return set_images_f32(b, nImages, counts, d_desc, true);
}

int v3dm_batch_float_mode(v3dm_batch* b, int* isFloat) {
  if (!b || !isFloat) return V3DM_ERR_ARG;
  *isFloat = b->floatMode ? 1 : 0;
  return V3DM_OK;
}

int v3dm_batch_set_pairs(v3dm_batch* b, int nPairs, const int32_t* pairs) {
  if (!b || nPairs < -1 || (nPairs > 0 && !pairs)) return V3DM_ERR_ARG;
  if (!b->haveImages) return V3DM_ERR_NOT_ALLOCATED;
  const int nI = b->nImages;
  std::vector<int> li, ri;
  if (nPairs == -1) {
    for (int i = 0; i < nI; ++i)
      for (int j = i + 1; j < nI; ++j) {
        li.push_back(i);
        ri.push_back(j);
      }
  } else {
    li.resize(nPairs);
    ri.resize(nPairs);
    for (int p = 0; p < nPairs; ++p) {
      li[p] = pairs[2 * p];
      ri[p] = pairs[2 * p + 1];
      if (li[p] < 0 || li[p] >= nI || ri[p] < 0 || ri[p] >= nI) return V3DM_ERR_ARG;
    }
  }
  if (li.size() > 0x7ffffffULL) return V3DM_ERR_SIZE;
  const int n = (int)li.size();
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return li[a] < li[c]; });
  std::vector<BPair> bp(n);
  long long SA = 0, ops = 0, exh = 0;
  for (int k = 0; k < n; ++k) {
    const int p = order[k];
    bp[k] = BPair{li[p], ri[p], p, b->counts[li[p]], SA};
    SA += b->counts[li[p]];
    ops += 2LL * kDescBytes * b->counts[li[p]] * b->counts[ri[p]];
    exh += (long long)b->counts[li[p]] * b->counts[ri[p]];
  }
  if (SA > 0x7ffffff0LL) return V3DM_ERR_SIZE;  // state indices are int32
  BDeviceGuard g(b->device);
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  drop_graph(b);
  b->havePairs = false;
  for (int i = 0; i < nI; ++i) b->bim[i].pairBeg = b->bim[i].pairEnd = 0;
  for (int k = 0; k < n;) {
    int e = k;
    while (e < n && bp[e].li == bp[k].li) ++e;
    b->bim[bp[k].li].pairBeg = k;
    b->bim[bp[k].li].pairEnd = e;
    k = e;
  }
  if (n > b->pairsCap) {
    bfree(b->dPairs);
    bfree(b->dCnt);
    bfree(b->dPrefC);
    b->pairsCap = 0;
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dPairs), (size_t)n * sizeof(BPair)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dCnt), (size_t)n * sizeof(int)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dPrefC), (size_t)(n + 1) * sizeof(long long)));
    b->pairsCap = n;
  }
  if (!b->dCnt) {
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dCnt), sizeof(int)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dPrefC), 2 * sizeof(long long)));
  }
  if (n > 0)
    V3DM_BTRY(cudaMemcpyAsync(b->dPairs, bp.data(), (size_t)n * sizeof(BPair), cudaMemcpyHostToDevice, b->stream));
  if (nI > 0)
    V3DM_BTRY(cudaMemcpyAsync(b->dImages, b->bim.data(), (size_t)nI * sizeof(BImage), cudaMemcpyHostToDevice,
                              b->stream));
  // per-state arrays; best and sec start at zero and every call leaves them at zero
  if (SA + 1 > b->stateCap) {
    bfree(b->dBest);
    bfree(b->dSec);
    bfree(b->dDecA);
    b->stateCap = 0;
    const long long cap = SA + 1;
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dBest), (size_t)cap * sizeof(unsigned long long)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dSec), (size_t)cap * sizeof(unsigned int)));
    V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dDecA), (size_t)cap * sizeof(int32_t)));
    V3DM_BTRY(cudaMemsetAsync(b->dBest, 0, (size_t)cap * sizeof(unsigned long long), b->stream));
    V3DM_BTRY(cudaMemsetAsync(b->dSec, 0, (size_t)cap * sizeof(unsigned int), b->stream));
    b->stateCap = cap;
  }
  // pass-B buffers: a first guess of 1/32 of the pass-A states, grown on overflow
  const long long wantB = std::max<long long>(65536, SA / 32);
  if (b->capB < wantB || b->capB == 0) V3DM_BTRY(alloc_passB(b, wantB));
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  b->nPairs = n;
  b->pairLi.swap(li);
  b->pairRi.swap(ri);
  b->bp.swap(bp);
  b->SA = SA;
  b->workOps = ops;
  b->exhaustivePairs = exh;
  b->havePairs = true;
  b->rowsDirty = true;
  b->mapsValid = false;
  return V3DM_OK;
}

int v3dm_batch_match(v3dm_batch* b, float minScore, float minRatio, int32_t* triples, long long cap, long long* nOut) {
  if (!b || !nOut || cap < 0 || (cap > 0 && !triples)) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  int st = run_host(b, minScore, minRatio);
  if (st != V3DM_OK) return st;
  const long long n = b->hInfo[kInfoWords + kCntOut];
  *nOut = n;
  const long long m = std::min(n, cap);
  if (m > 0) {
    V3DM_BTRY(cudaMemcpyAsync(triples, b->dOut, (size_t)m * sizeof(int3), cudaMemcpyDeviceToHost, b->stream));
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
  }
  return n > cap ? V3DM_ERR_CAPACITY : V3DM_OK;
}

int v3dm_batch_set_positions(v3dm_batch* b, const float* positions) {
  if (!b) return V3DM_ERR_ARG;
  if (!b->haveImages) return V3DM_ERR_NOT_ALLOCATED;
  if (b->totalDesc > 0 && !positions) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  b->havePositions = false;
  V3DM_BTRY(ensure(&b->dPos, &b->posCap, std::max<long long>(b->totalDesc, 1)));
  if (b->totalDesc > 0)
    V3DM_BTRY(cudaMemcpyAsync(b->dPos, positions, (size_t)b->totalDesc * sizeof(float2), cudaMemcpyDefault,
                              b->stream));
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  b->havePositions = true;
  return V3DM_OK;
}

int v3dm_batch_set_positions_device(v3dm_batch* b, const float* d_positions) {
  return v3dm_batch_set_positions(b, d_positions);
}

int v3dm_batch_match_guided(v3dm_batch* b, int type, const double* M, const float* thr, float minScore,
                            float minRatio, int32_t* triples, long long cap, long long* nOut) {
  if (!b || !nOut || cap < 0 || (cap > 0 && !triples) || (type != 1 && type != 2)) return V3DM_ERR_ARG;
  if (!b->haveImages || !b->havePairs || !b->havePositions) return V3DM_ERR_NOT_ALLOCATED;
  if (b->nPairs > 0 && (!M || !thr)) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  V3DM_BTRY(cudaStreamSynchronize(b->stream));
  const int n = b->nPairs;
  if (n > 0) {
    // per pair: the matrix as the reference's float3 rows (.cu:592-595), then thr^2 in float
    // (.cu:591); the pair's images; per batch-order pair its first state and caller index
    std::vector<float> gm((size_t)n * kBGateFloats);
    std::vector<int2> lr(n);
    for (int p = 0; p < n; ++p) {
      for (int i = 0; i < 9; ++i) gm[(size_t)p * kBGateFloats + i] = (float)M[9 * (size_t)p + i];
      gm[(size_t)p * kBGateFloats + 9] = thr[p] * thr[p];
      lr[p] = make_int2(b->pairLi[p], b->pairRi[p]);
    }
    std::vector<long long> s0(n);
    std::vector<int> oo(n);
    for (int k = 0; k < n; ++k) {
      s0[k] = b->bp[k].stateA0;
      oo[k] = b->bp[k].orig;
    }
    V3DM_BTRY(ensure(&b->dGate, &b->gateCap, (long long)n * kBGateFloats));
    V3DM_BTRY(ensure(&b->dPairLR, &b->pairLRCap, (long long)n));
    if ((long long)n > b->pairAuxCap) {
      bfree(b->dStateA0);
      bfree(b->dOrigOf);
      b->pairAuxCap = 0;
      V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dStateA0), (size_t)n * sizeof(long long)));
      V3DM_BTRY(cudaMalloc(reinterpret_cast<void**>(&b->dOrigOf), (size_t)n * sizeof(int)));
      b->pairAuxCap = n;
    }
    V3DM_BTRY(cudaMemcpyAsync(b->dGate, gm.data(), gm.size() * sizeof(float), cudaMemcpyHostToDevice, b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->dPairLR, lr.data(), lr.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->dStateA0, s0.data(), s0.size() * sizeof(long long), cudaMemcpyHostToDevice,
                              b->stream));
    V3DM_BTRY(cudaMemcpyAsync(b->dOrigOf, oo.data(), oo.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    V3DM_BTRY(cudaStreamSynchronize(b->stream));  // pageable host vectors
  }
  int st = V3DM_ERR_CANDIDATES;
  for (int attempt = 0; attempt < 6 && st == V3DM_ERR_CANDIDATES; ++attempt) {
    st = launch_call_guided(b, type, minScore, minRatio);
    if (st != V3DM_OK) return st;
    st = finish_call(b);
  }
  if (st != V3DM_OK) return st;
  const long long nT = b->hInfo[kInfoWords + kCntOut];
  *nOut = nT;
  const long long m = std::min(nT, cap);
  if (m > 0) {
    V3DM_BTRY(cudaMemcpyAsync(triples, b->dOut, (size_t)m * sizeof(int3), cudaMemcpyDeviceToHost, b->stream));
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
  }
  return nT > cap ? V3DM_ERR_CAPACITY : V3DM_OK;
}

int v3dm_batch_match_device(v3dm_batch* b, float minScore, float minRatio, int32_t* d_count) {
  if (!b) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  int st = launch_call(b, minScore, minRatio);
  if (st != V3DM_OK) return st;
  if (d_count)
    V3DM_BTRY(cudaMemcpyAsync(d_count, b->dInfo + kInfoWords + kCntOut, sizeof(int32_t), cudaMemcpyDeviceToDevice,
                              b->stream));
  return V3DM_OK;
}

int v3dm_batch_wait(v3dm_batch* b) {
  if (!b) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  if (!b->pendingCheck) {
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
    return V3DM_OK;
  }
  return finish_call(b);
}

int v3dm_batch_match_proposal(v3dm_batch* b, v3dm_projection* proj, int probesLeft, int probesRight, float minScore,
                              float minRatio, int32_t* triples, long long cap, long long* nOut) {
  if (!b || !nOut || cap < 0 || (cap > 0 && !triples)) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  int st = V3DM_ERR_CANDIDATES;
  for (int attempt = 0; attempt < 6 && st == V3DM_ERR_CANDIDATES; ++attempt) {
    st = launch_call_proposal(b, proj, probesLeft, probesRight, minScore, minRatio);
    if (st != V3DM_OK) return st;
    st = finish_call(b);
  }
  if (st != V3DM_OK) return st;
  const long long n = b->hInfo[kInfoWords + kCntOut];
  *nOut = n;
  const long long m = std::min(n, cap);
  if (m > 0) {
    V3DM_BTRY(cudaMemcpyAsync(triples, b->dOut, (size_t)m * sizeof(int3), cudaMemcpyDeviceToHost, b->stream));
    V3DM_BTRY(cudaStreamSynchronize(b->stream));
  }
  return n > cap ? V3DM_ERR_CAPACITY : V3DM_OK;
}

int v3dm_batch_match_proposal_device(v3dm_batch* b, v3dm_projection* proj, int probesLeft, int probesRight,
                                     float minScore, float minRatio, int32_t* d_count) {
  if (!b) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  int st = launch_call_proposal(b, proj, probesLeft, probesRight, minScore, minRatio);
  if (st != V3DM_OK) return st;
  if (d_count)
    V3DM_BTRY(cudaMemcpyAsync(d_count, b->dInfo + kInfoWords + kCntOut, sizeof(int32_t), cudaMemcpyDeviceToDevice,
                              b->stream));
  return V3DM_OK;
}

int v3dm_batch_proposal_scored(v3dm_batch* b, long long* scored, long long* exhaustive) {
  if (!b || !scored || !exhaustive) return V3DM_ERR_ARG;
  unsigned long long sc = 0;
  std::memcpy(&sc, b->hInfo + kInfoWords + kCntScored, sizeof(sc));
  *scored = (long long)sc;
  *exhaustive = b->havePairs ? b->exhaustivePairs : 0;
  return V3DM_OK;
}

int v3dm_batch_result_device(v3dm_batch* b, const int32_t** d_triples) {
  if (!b || !d_triples) return V3DM_ERR_ARG;
  *d_triples = reinterpret_cast<const int32_t*>(b->dOut);
  return V3DM_OK;
}

int v3dm_batch_stream(v3dm_batch* b, void** stream) {
  if (!b || !stream) return V3DM_ERR_ARG;
  *stream = b->stream;
  return V3DM_OK;
}

int v3dm_batch_use_graph(v3dm_batch* b, int enable) {
  if (!b) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  cudaStreamSynchronize(b->stream);
  b->useGraph = enable != 0;
  if (!b->useGraph) drop_graph(b);
  return V3DM_OK;
}

int v3dm_batch_set_config(v3dm_batch* b, int cfg, int schedule) {
  if (!b || schedule < 0 || schedule > 2) return V3DM_ERR_ARG;
  BDeviceGuard g(b->device);
  cudaStreamSynchronize(b->stream);
  if (tc_set_config(b->tc, cfg) != cudaSuccess) return V3DM_ERR_ARG;
  if (b->schedule != schedule || b->rowsCfg != cfg) drop_graph(b);
  b->schedule = schedule;
  return V3DM_OK;
}

int v3dm_batch_get_config(v3dm_batch* b, int* cfg, int* schedule) {
  if (!b || !cfg || !schedule) return V3DM_ERR_ARG;
  *cfg = tc_get_config(b->tc);
  *schedule = b->schedule;
  return V3DM_OK;
}

int v3dm_batch_autotune(v3dm_batch* b, float minScore, float minRatio, int reps, int* bestCfg, int* bestSchedule,
                        float* msOut) {
  if (!b || reps < 1) return V3DM_ERR_ARG;
  if (!b->haveImages || !b->havePairs) return V3DM_ERR_NOT_ALLOCATED;
  if (b->floatMode) return V3DM_ERR_UNSUPPORTED;  // one tile shape on the float layouts
  BDeviceGuard g(b->device);
  const int nCfg = tc_num_configs();
  const bool graphWas = b->useGraph;
  const bool profWas = b->profile;
  b->useGraph = false;
  b->profile = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  V3DM_BTRY(cudaEventCreate(&e0));
  V3DM_BTRY(cudaEventCreate(&e1));
  float bestMs = 1e30f;
  int bc = tc_get_config(b->tc), bs = b->schedule;
  int st = V3DM_OK;
  for (int c = 0; c < nCfg && st == V3DM_OK; ++c)
    for (int sch = 0; sch < 2 && st == V3DM_OK; ++sch) {
      tc_set_config(b->tc, c);
      b->schedule = sch;
      st = run_host(b, minScore, minRatio);  // warm-up; grows buffers if needed
      if (st != V3DM_OK) break;
      float total = 0.f;
      for (int r = 0; r < reps && st == V3DM_OK; ++r) {
        cudaEventRecord(e0, b->stream);
        st = launch_call(b, minScore, minRatio);
        cudaEventRecord(e1, b->stream);
        if (st == V3DM_OK) st = finish_call(b);
        float ms = 0.f;
        if (st == V3DM_OK) cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
      }
      const float avg = total / reps;
      if (msOut) msOut[2 * c + sch] = avg;
      if (st == V3DM_OK && avg < bestMs) {
        bestMs = avg;
        bc = c;
        bs = sch;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tc_set_config(b->tc, bc);
  b->schedule = bs;
  b->useGraph = graphWas;
  b->profile = profWas;
  drop_graph(b);
  if (bestCfg) *bestCfg = bc;
  if (bestSchedule) *bestSchedule = bs;
  return st;
}

int v3dm_batch_profile(v3dm_batch* b, int enable) {
  if (!b) return V3DM_ERR_ARG;
  b->profile = enable != 0;
  b->profMs[0] = b->profMs[1] = 0.0;
  b->profN[0] = b->profN[1] = 0;
  return V3DM_OK;
}

int v3dm_batch_profile_read(v3dm_batch* b, int pass, double* msTotal, int* launches) {
  if (!b || pass < 0 || pass > 1 || !msTotal || !launches) return V3DM_ERR_ARG;
  *msTotal = b->profMs[pass];
  *launches = b->profN[pass];
  return V3DM_OK;
}

int v3dm_batch_last_launches(v3dm_batch* b, int* n) {
  if (!b || !n) return V3DM_ERR_ARG;
  *n = b->lastLaunches;
  return V3DM_OK;
}

int v3dm_batch_work(v3dm_batch* b, long long* int8Ops, long long* nPairs) {
  if (!b || !int8Ops || !nPairs) return V3DM_ERR_ARG;
  *int8Ops = b->havePairs ? b->workOps : 0;
  *nPairs = b->havePairs ? b->nPairs : 0;
  return V3DM_OK;
}

}  // extern "C"
