// v3dm_match_tc.cu -- tcgen05 side kernel for sm_100a: one persistent launch scores one side
// of a pair against the other and keeps, for every descriptor of the A side, its best
// candidate and an upper bound of its second-best score.  Two launches (lefts x rights,
// then the chosen rights x lefts) replace cublasSgemm + the four maxima kernels of the
// reference (v3d_cudamatching.cu:529-545); no score leaves the SM.
//
//   warp 0      TMA producer: an A group (NB blocks of 128 descriptors x 128 bytes) whenever
//               the group changes, B tiles (BN x 128 bytes) through a ring of shared-memory
//               stages, 128-byte swizzle;
//   warp 1      allocates 512 TMEM columns and issues tcgen05.mma.kind::i8 (u8 x u8 -> s32,
//               M=128, N=BN, four K=32 steps per block) into 512/(NB*BN) accumulator stages;
//   warps 2-17  epilogue, four per TMEM lane quadrant.  Lane i of a warp owns A descriptor
//               'row' and reads its scores with tcgen05.ld (32 columns per chunk), hands the
//               stage back, and per chunk does one of two things:
//                 - all scores below Smin (the smallest score that can pass the min-score
//                   test): W = max(W, chunk maximum);
//                 - some score >= Smin (true matches, ~1e-6 of unrelated pairs): the lane
//                   writes a record (descriptor, first column, its 32 scores) to its warp's
//                   segment; k_records (v3dm_pair.cu) does the exact work on it: guided
//                   gates for every score >= Smin, chunk best (largest score, first index on
//                   ties, the reference's argMax rule, v3d_cudamatching.cu:145), maximum of
//                   the other scores.
//               At the end of a work unit the lane's W + 1 goes to sec[] (atomicMax).  W starts
//               as a negative float's bits (below every score) and takes the spare input of the
//               chunk's maximum tree: C = max(W, chunk); C >= Smin exactly when the chunk
//               reaches Smin (W < Smin always), else W = C.
// Resulting per-descriptor values (after the list pass in v3dm_pair.cu): best = the exact
// best over scores >= Smin that pass the gates; sec = the exact second-best score without
// gates, an upper bound of it with gates (masked scores are counted).  The decision
// accept(best, s2) is monotone in s2, so when accept(best, sec) == accept(best, none) the
// decision is exact; otherwise the descriptor is re-scored exactly (rare).
// The tile shape (NB, BN) and the stage counts are template parameters chosen at run time
// (TcConfig).  NB=2 keeps 256 A rows resident and halves the B bytes per MMA compared with one
// 128-row block; more TMEM stages hide the MMA -> epilogue -> MMA hand-off latency.
// The work is the flattened sequence (A group, B tile); each CTA takes one contiguous range
// of it.  Every role walks the same range; mbarriers order the hand-offs.  Every mbarrier wait
// is bounded: on timeout the CTA raises kErrWaitTimeout, drains its own TMA loads and MMAs,
// frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <new>
#include <type_traits>

#include "v3dm_device.cuh"
#include "v3dm_tcgen05.cuh"

namespace v3dm {

namespace {

constexpr int BM = 128;          // rows per MMA block (TMEM lanes)
constexpr int kEpiWarps = 16;    // four per TMEM lane quadrant
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr int kTmemCols = 512;

template <int NB_, int BN_, int STAGES_, int ASLOTS_ = 2, int SPLIT_ = 1, int PIPE_ = 0>
struct TcCfg {
  static constexpr int NB = NB_;                 // 128-row MMA blocks per left group
  static constexpr int BN = BN_;                 // rights per tile
  static constexpr int kStages = STAGES_;        // right-tile ring depth
  static constexpr int kASlots = ASLOTS_;        // left-group buffers (more: short rows prefetch further)
  // kSplit = 2: each tile is scored as two BN/2-column MMAs into two accumulator stages, so the MMA
  // can run further ahead of the epilogue (twice the stages of half the width)
  static constexpr int kSplit = SPLIT_;
  // kPipe = 1: the epilogue loads its second chunk while it filters the first
  static constexpr int kPipe = PIPE_;
  static constexpr int GM = BM * NB;             // left rows per group
  static constexpr int kABytes = GM * kDescBytes;
  static constexpr int kBBytes = BN * kDescBytes;
  static constexpr int kMmaN = BN / kSplit;      // columns of one MMA / accumulator block
  static constexpr int kAccCols = NB * kMmaN;    // TMEM columns per accumulator stage
  static constexpr int kAcc = kTmemCols / kAccCols;  // accumulator stages
  // Epilogue split: the four warps of a lane quadrant own (block, column quarter or half) of a
  // stage: with NB == 2 a warp owns one block and half of the columns, with NB == 1 a quarter.
  static constexpr int kWarpCols = NB == 2 ? kMmaN / 2 : kMmaN / 4;
  static constexpr int kChunks = kWarpCols / 32;
  static_assert(NB == 1 || NB == 2, "one or two blocks per group");
  static_assert(kSplit == 1 || (kSplit == 2 && NB == 1), "split tiles with one block per group");
  static_assert(kWarpCols >= 32 && kWarpCols % 32 == 0 && kChunks <= 2 && BN <= 256, "1..2 chunks per warp");
  static_assert(kPipe == 0 || kChunks == 2, "pipelined loads need two chunks");
  static_assert(kAcc >= 2, "at least two accumulator stages");
};

template <class C>
struct Smem {
  uint8_t a[C::kASlots][C::kABytes];
  uint8_t b[C::kStages][C::kBBytes];
  unsigned long long fullB[C::kStages], emptyB[C::kStages];
  unsigned long long fullA[C::kASlots], emptyA[C::kASlots];
  unsigned long long accFull[C::kAcc], accEmpty[C::kAcc];
  unsigned long long mmaDone;
  uint32_t tmemBase;
  int abort;
};

struct TcShape {
  int nGroups, nTiles;  // left groups, right tiles
  long long nWork;      // nGroups * nTiles
};

// Instruction descriptor: kind::i8, D = s32, A = B = unsigned 8-bit, both K-major, N, M = 128.
template <int N>
__device__ __forceinline__ constexpr uint32_t idesc() {
  return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int N>
__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(idesc<N>()), "r"(accumulate)
      : "memory");
}

static_assert(kMaxScore < (1 << 23), "scores are zero or subnormal as floats");

// Maximum of three scores in one instruction: the three-input max.f32 of sm_100 applied to the
// scores' bit patterns.  Scores are integers in [0, 255^2 * 128] < 2^23, i.e. zero or subnormal
// floats, whose float order is their integer order; max.f32 without .ftz keeps subnormals.
__device__ __forceinline__ uint32_t max3_bits(uint32_t a, uint32_t b, uint32_t c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(__uint_as_float(a)), "f"(__uint_as_float(b)), "f"(__uint_as_float(c)));
  return __float_as_uint(r);
}

// max(x, the 32 scores of v): a tree of three-input maxima, 16 instructions (a two-input tree
// takes 31 for the scores alone; the epilogue's filtering is what limits the side kernel).  x
// takes the spare input of the last one.
__device__ __forceinline__ uint32_t max32_bits(const uint32_t* v, uint32_t x) {
  uint32_t m[12];
#pragma unroll
  for (int i = 0; i < 10; ++i) m[i] = max3_bits(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
  m[10] = v[30];
  m[11] = v[31];
  uint32_t n[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) n[i] = max3_bits(m[3 * i], m[3 * i + 1], m[3 * i + 2]);
  return max3_bits(max3_bits(n[0], n[1], n[2]), n[3], x);
}

// Work range of this CTA in the flattened (group, tile) sequence.
__device__ __forceinline__ void cta_range(const TcShape& sh, long long& w0, long long& w1) {
  w0 = sh.nWork * blockIdx.x / gridDim.x;
  w1 = sh.nWork * (blockIdx.x + 1) / gridDim.x;
}

// Single pair: walks (group, tile) pairs of a work range with one division at the start, so
// the per-tile loops of the MMA issuer and the epilogue stay free of 64-bit divisions.
struct WorkCursor {
  int g, t, nTiles;
  long long left;
  bool fresh;  // first tile of a group
  bool newA;   // the group's A block differs from the previous one (always, with fresh)
  __device__ __forceinline__ WorkCursor(long long w0, long long w1, int nT)
      : nTiles(nT), left(w1 - w0), fresh(true), newA(true) {
    g = (int)(w0 / nT);
    t = (int)(w0 - (long long)g * nT);
  }
  __device__ __forceinline__ bool more() const { return left > 0; }
  __device__ __forceinline__ void next() {
    --left;
    fresh = false;
    if (++t == nTiles) {
      t = 0;
      ++g;
      fresh = true;
    }
    newA = fresh;
  }
  __device__ __forceinline__ void prefetch_rows() const {}
};

__device__ __forceinline__ BatchRow load_row(const BatchRow* rows, int r) {
  const int4* p = reinterpret_cast<const int4*>(rows + r);
  const int4 x = __ldg(p), y = __ldg(p + 1);
  BatchRow b;
  b.aRow = x.x;
  b.validRows = x.y;
  b.bRow0 = x.z;
  b.nB = x.w;
  b.nTiles = max(y.x, 1);  // every row advances the cursor by at least one tile
  b.pad = y.y;
  b.state0 = (long long)(((unsigned long long)(uint32_t)y.w << 32) | (uint32_t)y.z);
  return b;
}

constexpr int kChunkRows = 32;  // schedule 2: rows per chunk
constexpr int kRowAhead = 6;    // the producer prefetches the row entry this many rows ahead

// Batched pass: walks the rows of a row table, every tile of a row in order.  Schedule 0
// gives CTA b the rows b, b + grid, b + 2 grid, ...: the CTAs then work on neighbouring rows
// (the same B image) at the same time, so the B tiles are read from L2.  Schedule 1 gives
// each CTA one contiguous range of rows.  Schedule 2 deals out chunks of kChunkRows
// consecutive rows the way schedule 0 deals out rows: consecutive rows that share their A
// block (short rows of one left block against many right blocks) keep it in shared memory,
// and the CTAs still work on neighbouring rows.  The next row's entry is loaded a row ahead;
// the producer also prefetches entries kRowAhead rows ahead into L1.  newA says whether the
// current row's A block differs from the previous row's (a row's A block is identified by
// its first row aRow).
struct BatchCursor {
  const BatchRow* rows;
  int R, Rend, t, schedule;
  BatchRow cur, nxt;
  bool fresh, newA;
  __device__ __forceinline__ int step_from(int r) const {
    if (schedule == 0) return r + (int)gridDim.x;
    if (schedule == 1) return r + 1;
    ++r;
    return (r % kChunkRows) == 0 ? r + ((int)gridDim.x - 1) * kChunkRows : r;
  }
  __device__ __forceinline__ BatchCursor(const BatchRow* rows_, int nRows, int sch)
      : rows(rows_), t(0), schedule(sch), fresh(true), newA(true) {
    cur = BatchRow{};
    nxt = BatchRow{};
    if (schedule == 0) {
      R = blockIdx.x;
      Rend = nRows;
    } else if (schedule == 1) {
      R = (int)((long long)nRows * blockIdx.x / gridDim.x);
      Rend = (int)((long long)nRows * (blockIdx.x + 1) / gridDim.x);
    } else {
      R = blockIdx.x * kChunkRows;
      Rend = nRows;
    }
    if (R < Rend) cur = load_row(rows, R);
    const int R1 = step_from(R);
    if (R1 < Rend) nxt = load_row(rows, R1);
  }
  __device__ __forceinline__ bool more() const { return R < Rend; }
  __device__ __forceinline__ void next() {
    fresh = false;
    newA = false;
    if (++t == cur.nTiles) {
      t = 0;
      R = step_from(R);
      fresh = true;
      newA = nxt.aRow != cur.aRow;
      cur = nxt;
      const int R1 = step_from(R);
      if (R1 < Rend) nxt = load_row(rows, R1);
    }
  }
  // The row entry kRowAhead rows ahead, into L1 (the other roles of the CTA read it later).
  __device__ __forceinline__ void prefetch_rows() const {
    int r = R;
#pragma unroll
    for (int i = 0; i < kRowAhead; ++i) r = step_from(r);
    if (r < Rend) asm volatile("prefetch.global.L1 [%0];" ::"l"(rows + r));
  }
};

// Gathered A blocks (kGather): the producer warp copies each A row from a.aSrc (row
// a.aSrcRow[entry]) into the 128-byte-swizzled shared layout the TMA would write (16-byte
// chunk k of row r at r * 128 + ((k ^ (r & 7)) << 4)), rows past the block's valid count
// zero-filled.  The copies are cp.async (generic proxy): each lane waits for its own copies,
// fences them toward the async proxy the tensor core reads through, and lane 0 then arrives
// on the slot's full barrier.  kGatherDepth newer gathers may stay in flight while an older
// one is completed.
constexpr int kGatherDepth = 3;
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t srcBytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// kBatch = false: one pair, the flattened (group, tile) range of this CTA (WorkCursor).
// kBatch = true: rows of a.rows (BatchCursor); a row's state indices are state0 + row.
// kGather = true (batched pass only): A blocks gathered row by row from a.aSrc (tmA unused).
template <class C, bool kBatch, bool kGather = false>
__global__ void __launch_bounds__(kThreads, 1)
k_side(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int nTiles, SideArgs a) {
  static_assert(!kGather || kBatch, "gathered A blocks only in the batched pass");
  const long long lim = a.waitLimit > 0 ? a.waitLimit : kWaitCycles;
  pdl_wait();
  pdl_launch_dependents();
  extern __shared__ uint8_t smemRaw[];
  Smem<C>& s = *reinterpret_cast<Smem<C>*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  using Cursor = typename std::conditional<kBatch, BatchCursor, WorkCursor>::type;
  int nA = 0, nRows = 0;
  TcShape sh{};
  long long w0 = 0, w1 = 0;
  if constexpr (kBatch) {
    nRows = a.nRowsPtr ? *a.nRowsPtr : a.nRows;
    if (nRows <= 0) {  // nothing to score: uniform early exit
      if (warp >= 2 && lane == 0) a.segCount[blockIdx.x * kEpiWarps + (warp - 2)] = 0;
      return;
    }
  } else {
    nA = a.nAptr ? *a.nAptr : a.nA;
    sh.nGroups = (nA + C::GM - 1) / C::GM;
    sh.nTiles = nTiles;
    sh.nWork = (long long)sh.nGroups * nTiles;
    if (sh.nWork == 0) {  // nothing to score (e.g. no right was chosen): uniform early exit
      if (warp >= 2 && lane == 0) a.segCount[blockIdx.x * kEpiWarps + (warp - 2)] = 0;
      return;
    }
    cta_range(sh, w0, w1);
  }
  auto make_cursor = [&]() -> Cursor {
    if constexpr (kBatch) return BatchCursor(a.rows, nRows, a.schedule);
    else return WorkCursor(w0, w1, sh.nTiles);
  };

  if (threadIdx.x == 0) {
    for (int i = 0; i < C::kStages; ++i) {
      mbar_init(&s.fullB[i], 1);
      mbar_init(&s.emptyB[i], 1);
    }
    for (int i = 0; i < C::kASlots; ++i) {
      mbar_init(&s.fullA[i], 1);
      mbar_init(&s.emptyA[i], 1);
    }
    for (int i = 0; i < C::kAcc; ++i) {
      mbar_init(&s.accFull[i], 1);
      mbar_init(&s.accEmpty[i], kEpiWarps);
    }
    mbar_init(&s.mmaDone, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmemBase)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmemBase;
  if ((tmem & 0xFFFFu) != 0 && threadIdx.x == 0) {  // 512 columns must start at column 0
    atomicOr(a.err, kErrTmem);
    s.abort = 1;
  }
  __syncthreads();

  if (warp == 0) {
   if constexpr (kGather) {
    // ---------------- producer, gathered A: the whole warp ----------------
    if (!s.abort) {
      int stage = 0, aBuf = C::kASlots - 1;
      uint32_t phase = 0, aPhase = 1;
      uint32_t armedPhase[C::kStages];
      bool armed[C::kStages];
      for (int i = 0; i < C::kStages; ++i) armed[i] = false;
      int pend[kGatherDepth + 1] = {};  // slots whose gather still needs its arrive, oldest first
      int nPend = 0;
      int preRow = -1;                   // A block whose entry indices pre[] holds
      int pre[C::GM / 32];
#pragma unroll
      for (int k = 0; k < C::GM / 32; ++k) pre[k] = -1;
      auto arrive_oldest = [&]() {
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.fullA[pend[0]]);
        for (int i = 1; i <= kGatherDepth; ++i)
          if (i < nPend) pend[i - 1] = pend[i];
        --nPend;
      };
      auto arrive_all = [&]() {
        cp_async_wait<0>();
        while (nPend > 0) arrive_oldest();
      };
      // blocking wait by lane 0 (after handing over every pending gather, so that the MMA
      // can drain what the wait depends on); the result is broadcast
      auto wait_slot = [&](unsigned long long* bar, uint32_t par) -> bool {
        if (mbar_try(bar, par)) return true;
        arrive_all();
        int okl = 1;
        if (lane == 0) okl = mbar_wait(bar, par, &s.abort, a.err, lim) ? 1 : 0;
        return __shfl_sync(0xffffffffu, okl, 0) != 0;
      };
      for (Cursor wc = make_cursor(); wc.more(); wc.next()) {
        if (wc.fresh && lane == 0) wc.prefetch_rows();
        if (wc.newA) {
          if (++aBuf == C::kASlots) {
            aBuf = 0;
            aPhase ^= 1;
          }
          if (!wait_slot(&s.emptyA[aBuf], aPhase ^ 1)) break;
          const int aRow = wc.cur.aRow, nValid = wc.cur.validRows;
          int src[C::GM / 32];
#pragma unroll
          for (int k = 0; k < C::GM / 32; ++k) {
            const int rr = lane + 32 * k;
            src[k] = aRow == preRow ? pre[k] : (rr < nValid ? __ldg(a.aSrcRow + aRow + rr) : -1);
          }
          const uint32_t dst0 = smem_u32(s.a[aBuf]);
#pragma unroll
          for (int k = 0; k < C::GM / 32; ++k) {
            const int rr = lane + 32 * k;
            const uint8_t* g = a.aSrc + (src[k] >= 0 ? (size_t)src[k] * kDescBytes : (size_t)0);
            const uint32_t nb = src[k] >= 0 ? 16u : 0u;  // 0: zero fill
            const uint32_t d = dst0 + (uint32_t)rr * 128u;
#pragma unroll
            for (int ch = 0; ch < 8; ++ch) cp_async16(d + (uint32_t)((ch ^ (rr & 7)) << 4), g + 16 * ch, nb);
          }
          cp_async_commit();
          // the next row's entry indices, read now and used at its turn (the loads overlap)
          if (wc.nxt.aRow != aRow) {
            preRow = wc.nxt.aRow;
#pragma unroll
            for (int k = 0; k < C::GM / 32; ++k) {
              const int rr = lane + 32 * k;
              pre[k] = rr < wc.nxt.validRows ? __ldg(a.aSrcRow + preRow + rr) : -1;
            }
          }
          pend[nPend++] = aBuf;
          if (nPend > kGatherDepth) {
            cp_async_wait<kGatherDepth>();
            arrive_oldest();
          }
        }
        if (!wait_slot(&s.emptyB[stage], phase ^ 1)) break;
        if (lane == 0) {
          mbar_expect_tx(&s.fullB[stage], C::kBBytes);
          int bRow = 0;
          if constexpr (kBatch) bRow = wc.cur.bRow0 + wc.t * C::BN;
          tma_load_2d(s.b[stage], &tmB, &s.fullB[stage], 0, bRow);
        }
        armed[stage] = true;
        armedPhase[stage] = phase;
        if (++stage == C::kStages) {
          stage = 0;
          phase ^= 1;
        }
      }
      // every gather has landed (and is handed over) and every load lane 0 issued has landed
      // before the CTA may exit
      arrive_all();
      if (lane == 0)
        for (int i = 0; i < C::kStages; ++i)
          if (armed[i]) {
            long long t0c = clock64();
            while (!mbar_try(&s.fullB[i], armedPhase[i]) && clock64() - t0c < kWaitCycles) {
            }
          }
    }
   } else {
    // ---------------- TMA producer ----------------
    if (lane == 0 && !s.abort) {
      int stage = 0, aBuf = C::kASlots - 1;
      uint32_t phase = 0, aPhase = 1;
      uint32_t armedPhase[C::kStages], armedAPhase[C::kASlots];
      bool armed[C::kStages], armedA[C::kASlots];
      int nIssued = 0;  // B tile loads issued (test hook)
      for (int i = 0; i < C::kStages; ++i) armed[i] = false;
      for (int i = 0; i < C::kASlots; ++i) armedA[i] = false;
      for (Cursor wc = make_cursor(); wc.more(); wc.next()) {
        if (wc.fresh) wc.prefetch_rows();
        if (wc.newA) {
          if (++aBuf == C::kASlots) {
            aBuf = 0;
            aPhase ^= 1;
          }
          if (!mbar_wait(&s.emptyA[aBuf], aPhase ^ 1, &s.abort, a.err, lim)) break;
          mbar_expect_tx(&s.fullA[aBuf], C::kABytes);
          int aRow;
          if constexpr (kBatch) aRow = wc.cur.aRow;
          else aRow = wc.g * C::GM;
          tma_load_2d(s.a[aBuf], &tmA, &s.fullA[aBuf], 0, aRow);
          armedA[aBuf] = true;
          armedAPhase[aBuf] = aPhase;
        }
        if (!mbar_wait(&s.emptyB[stage], phase ^ 1, &s.abort, a.err, lim)) break;
        if (a.skipLoad > 0 && blockIdx.x == 0 && ++nIssued == a.skipLoad) {
          armed[stage] = false;  // test hook: this tile never arrives; the MMA's bounded wait gives up
        } else {
          mbar_expect_tx(&s.fullB[stage], C::kBBytes);
          int bRow;
          if constexpr (kBatch) bRow = wc.cur.bRow0 + wc.t * C::BN;
          else bRow = wc.t * C::BN;
          tma_load_2d(s.b[stage], &tmB, &s.fullB[stage], 0, bRow);
          armed[stage] = true;
          armedPhase[stage] = phase;
        }
        if (++stage == C::kStages) {
          stage = 0;
          phase ^= 1;
        }
      }
      // Drain: every load this thread issued has landed before the CTA may exit.
      for (int i = 0; i < C::kStages; ++i)
        if (armed[i]) {
          long long t0c = clock64();
          while (!mbar_try(&s.fullB[i], armedPhase[i]) && clock64() - t0c < kWaitCycles) {
          }
        }
      for (int i = 0; i < C::kASlots; ++i)
        if (armedA[i]) {
          long long t0c = clock64();
          while (!mbar_try(&s.fullA[i], armedAPhase[i]) && clock64() - t0c < kWaitCycles) {
          }
        }
    }
   }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0 && !s.abort) {
      int stage = 0, acc = 0, aBuf = C::kASlots - 1;
      bool anyA = false;
      uint32_t phase = 0, accPhase = 0, aPhase = 1;
      uint32_t aAddr = 0;
      for (Cursor wc = make_cursor(); wc.more(); wc.next()) {
        if (wc.newA) {
          if (anyA) mma_commit(&s.emptyA[aBuf]);
          if (++aBuf == C::kASlots) {
            aBuf = 0;
            aPhase ^= 1;
          }
          if (!mbar_wait(&s.fullA[aBuf], aPhase, &s.abort, a.err, lim)) break;
          aAddr = smem_u32(s.a[aBuf]);
          anyA = true;
        }
        if (!mbar_wait(&s.fullB[stage], phase, &s.abort, a.err, lim)) break;
        const uint32_t bAddr = smem_u32(s.b[stage]);
        bool stop = false;
#pragma unroll
        for (int h = 0; h < C::kSplit; ++h) {
          if (!mbar_wait(&s.accEmpty[acc], accPhase ^ 1, &s.abort, a.err, lim)) {
            stop = true;
            break;
          }
          tc_fence_after();
          // columns h * kMmaN .. of the tile: B rows 128 bytes each, 1024-byte aligned halves
          const uint32_t bh = bAddr + (uint32_t)(h * C::kMmaN * kDescBytes);
#pragma unroll
          for (int blk = 0; blk < C::NB; ++blk) {
            const uint32_t d = tmem + (uint32_t)(acc * C::kAccCols + blk * C::kMmaN);
            const uint32_t ab = aAddr + (uint32_t)(blk * BM * kDescBytes);
#pragma unroll
            for (int k = 0; k < kDescBytes / 32; ++k)
              mma_i8<C::kMmaN>(d, sdesc(ab + 32u * k), sdesc(bh + 32u * k), k > 0 ? 1u : 0u);
          }
          mma_commit(&s.accFull[acc]);
          if (++acc == C::kAcc) {
            acc = 0;
            accPhase ^= 1;
          }
        }
        if (stop) break;
        mma_commit(&s.emptyB[stage]);
        if (++stage == C::kStages) {
          stage = 0;
          phase ^= 1;
        }
      }
      if (anyA) mma_commit(&s.emptyA[aBuf]);
      // Every MMA this thread issued has completed before TMEM is released.
      mma_commit(&s.mmaDone);
      long long t0c = clock64();
      while (!mbar_try(&s.mmaDone, 0) && clock64() - t0c < kWaitCycles) {
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int e = warp - 2;
    const int q = warp & 3;                              // TMEM lane quadrant this warp may access
    const int sub = e >> 2;                              // 0..3 within the quadrant
    const int blk = C::NB == 2 ? (sub & 1) : 0;          // A block of the group
    const int colOff = (C::NB == 2 ? (sub >> 1) : sub) * C::kWarpCols;  // first tile column of this warp
    const int rowInGroup = blk * BM + q * 32 + lane;
    uint4* const segBase = a.records + (long long)(blockIdx.x * kEpiWarps + e) * a.segCap * kRecordQuads;
    int segN = 0;                                        // warp-uniform count of records written
    int acc = 0;
    bool started = false;
    uint32_t accPhase = 0;
    bool ok = !s.abort;
    bool rowValid = false;
    int orig = 0;
    int aLocal = 0;  // batched pass: index of this lane's A row within its image
    int nB = a.nB;
    int bRow0 = 0;
    // maximum of this lane's scores in the current unit, chunks with a record excluded; kNoScore
    // (a negative float, below every score in the max.f32 order) while there is none
    constexpr uint32_t kNoScore = 0xbf800000u;
    uint32_t lw = kNoScore;
    int32_t sminRow = 0x7fffffff;  // Smin for a valid row, above every score otherwise
    // a bound below Tsec cannot change the decision: no atomic for it
    auto flush = [&]() {
      const uint32_t w = lw == kNoScore ? 0u : lw + 1u;  // sec[] holds second + 1
      if (rowValid && w > (uint32_t)a.Tsec) atomicMax(&a.sec[orig], w);
    };
    for (Cursor wc = make_cursor(); wc.more() && ok; wc.next()) {
      if (wc.fresh) {
        if (started) flush();
        started = true;
        if constexpr (kBatch) {
          rowValid = rowInGroup < wc.cur.validRows;
          if (wc.newA)  // the A block's index map is read once per block, not once per row
            aLocal = rowValid ? (a.amap ? __ldg(a.amap + wc.cur.aRow + rowInGroup) : rowInGroup) : 0;
          orig = rowValid ? (int)(wc.cur.state0 + aLocal) : 0;
          nB = wc.cur.nB;
          bRow0 = wc.cur.bRow0;
        } else {
          const int row = wc.g * C::GM + rowInGroup;
          rowValid = row < nA;
          orig = rowValid ? (a.amap ? a.amap[row] : row) : 0;
        }
        lw = kNoScore;
        sminRow = rowValid ? a.Smin : 0x7fffffff;
      }
      for (int h = 0; h < C::kSplit; ++h) {
      const int colBase = wc.t * C::BN + h * C::kMmaN + colOff;
      ok = mbar_wait(&s.accFull[acc], accPhase, &s.abort, a.err, lim);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      const uint32_t tbase =
          tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * C::kAccCols + blk * C::kMmaN + colOff);
      // All of this warp's scores into registers, then hand the stage back at once so the
      // MMA never waits for the filtering below (kPipe: the second chunk is loaded while the
      // first is filtered, and the stage handed back after it).
      uint32_t v[C::kChunks][32];
      if constexpr (C::kPipe) {
        tmem_ld32(tbase, v[0]);
        tmem_wait(v[0]);
        tmem_ld32(tbase + 32u, v[1]);
      } else {
#pragma unroll
        for (int c = 0; c < C::kChunks; ++c) tmem_ld32(tbase + (uint32_t)(c * 32), v[c]);
#pragma unroll
        for (int c = 0; c < C::kChunks; ++c) tmem_wait(v[c]);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.accEmpty[acc]);
      }
#pragma unroll
      for (int c = 0; c < C::kChunks; ++c) {
        if constexpr (C::kPipe) {
          if (c == 1) {
            tmem_wait(v[1]);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&s.accEmpty[acc]);
          }
        }
        const int col0 = colBase + 32 * c;
        if (col0 >= nB) continue;  // chunks past the last B descriptor (warp-uniform)
        if (col0 + 32 > nB) {
          // The chunk holding the last B descriptor: the columns past it hold zero fill, zero
          // padding or the next block's descriptors; a 0 there is <= every real score, so the
          // chunk maximum stays the maximum of its real scores.
#pragma unroll
          for (int k = 0; k < 32; ++k)
            if (col0 + k >= nB) v[c][k] = 0u;
        }
        const uint32_t cm = max32_bits(v[c], lw);  // max(lw, chunk maximum)
        const bool trig = (int32_t)cm >= sminRow;   // kNoScore is negative as an int32
        if (!trig) lw = cm;                          // an invalid row's lw is never flushed
        if (__any_sync(0xffffffffu, trig)) {
          // rare: hand the chunk to k_records (its exact best, gates and other scores)
          const unsigned m = __ballot_sync(0xffffffffu, trig);
          if (trig) {
            const int idx = segN + __popc(m & ((1u << lane) - 1u));
            if (idx < a.segCap) {
              uint4* rec = segBase + (long long)idx * kRecordQuads;
              rec[0] = make_uint4((uint32_t)orig, (uint32_t)col0, (uint32_t)nB, (uint32_t)bRow0);
#pragma unroll
              for (int k = 0; k < 8; ++k)
                rec[1 + k] = make_uint4(v[c][4 * k], v[c][4 * k + 1], v[c][4 * k + 2], v[c][4 * k + 3]);
            }
          }
          segN += __popc(m);
        }
      }
      if (++acc == C::kAcc) {
        acc = 0;
        accPhase ^= 1;
      }
      }
      if (!ok) break;
    }
    if (started && ok) flush();
    if (lane == 0) a.segCount[blockIdx.x * kEpiWarps + e] = segN;
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                              : "memory");
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 2-D uint8 map over rows x 128 bytes with a box of boxRows x 128 and the 128-byte swizzle.
bool encode_rows(CUtensorMap* map, const uint8_t* base, int rows, int boxRows) {
  auto fn = get_encode();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kDescBytes, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kDescBytes};
  cuuint32_t box[2] = {(cuuint32_t)kDescBytes, (cuuint32_t)boxRows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}


// ---- configurations ------------------------------------------------------------------
// Each entry instantiates the kernel for one tile shape; shared memory per CTA is
// 2 * (NB*16 KB) for the left groups + stages * BN*128 bytes.
using Cfg0 = TcCfg<1, 256, 4>;   // 128 x 256 tiles, 2 accumulator stages, 4-deep ring
using Cfg1 = TcCfg<1, 128, 8>;   // 128 x 128 tiles, 4 accumulator stages
using Cfg2 = TcCfg<2, 128, 8>;   // 256 x 128 tiles, 2 accumulator stages
using Cfg3 = TcCfg<2, 64, 16>;   // 256 x 64 tiles, 4 accumulator stages
using Cfg4 = TcCfg<1, 256, 6>;   // 128 x 256 tiles, 2 accumulator stages, 6-deep ring
using Cfg5 = TcCfg<1, 256, 4, 4>;   // as Cfg0 with 4 left-group buffers (rows of few tiles)
using Cfg6 = TcCfg<1, 128, 6, 6>;   // 128 x 128 tiles, 6 left-group buffers
using Cfg7 = TcCfg<1, 256, 4, 4, 2>;      // as Cfg5, each tile as two 128-column MMAs (4 accumulator stages)
using Cfg8 = TcCfg<1, 256, 6, 2, 2>;      // as Cfg4, split the same way
using Cfg9 = TcCfg<1, 256, 4, 4, 1, 1>;   // as Cfg5 with the epilogue's second chunk loaded while the first is filtered

template <class C, bool kBatch, bool kGather = false>
cudaError_t launch_cfg(const CUtensorMap& mA, const CUtensorMap& mB, int nTiles, const SideArgs& a, int grid,
                       cudaStream_t st, bool& attrSet) {
  const size_t smem = sizeof(Smem<C>) + 1024;
  if (!attrSet) {
    cudaError_t e =
        cudaFuncSetAttribute(k_side<C, kBatch, kGather>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attrSet = true;
  }
  return launch_pdl(k_side<C, kBatch, kGather>, dim3(grid), dim3(kThreads), smem, st, mA, mB, nTiles, a);
}

constexpr int kNumCfg = 10;
constexpr int kCfgNB[kNumCfg] = {Cfg0::NB, Cfg1::NB, Cfg2::NB, Cfg3::NB, Cfg4::NB,
                                 Cfg5::NB, Cfg6::NB, Cfg7::NB, Cfg8::NB, Cfg9::NB};
constexpr int kCfgBN[kNumCfg] = {Cfg0::BN, Cfg1::BN, Cfg2::BN, Cfg3::BN, Cfg4::BN,
                                 Cfg5::BN, Cfg6::BN, Cfg7::BN, Cfg8::BN, Cfg9::BN};
constexpr int kDefaultCfg = 0;

}  // namespace

struct TcPlan {
  int device = 0;
  int numSMs = 148;
  int cfg = kDefaultCfg;
  bool attrSet[kNumCfg] = {};
  bool attrSetBatch[kNumCfg] = {};
  bool attrSetGather = false;
};

cudaError_t tc_plan_create(TcPlan** p, int device) {
  TcPlan* t = new (std::nothrow) TcPlan();
  if (!t) return cudaErrorMemoryAllocation;
  t->device = device;
  cudaError_t e = cudaDeviceGetAttribute(&t->numSMs, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    delete t;
    return e;
  }
  *p = t;
  return cudaSuccess;
}

void tc_plan_destroy(TcPlan* p) { delete p; }

int tc_segments(TcPlan* p) { return p->numSMs * kEpiWarps; }

int tc_num_configs() { return kNumCfg; }

int tc_get_config(TcPlan* p) { return p->cfg; }

cudaError_t tc_set_config(TcPlan* p, int cfg) {
  if (cfg < 0 || cfg >= kNumCfg) return cudaErrorInvalidValue;
  p->cfg = cfg;
  return cudaSuccess;
}

void tc_config_shape(int cfg, int* rowsPerGroup, int* colsPerTile) {
  *rowsPerGroup = kCfgNB[cfg] * BM;
  *colsPerTile = kCfgBN[cfg];
}

cudaError_t tc_side_maps(TcPlan* p, TcMaps* m, const uint8_t* dA, int rowsA, const uint8_t* dB, int rowsB) {
  const int c = p->cfg;
  if (rowsA <= 0 || rowsB <= 0) return cudaErrorInvalidValue;
  if (!encode_rows(&m->a, dA, rowsA, kCfgNB[c] * BM) || !encode_rows(&m->b, dB, rowsB, kCfgBN[c]))
    return cudaErrorInvalidValue;
  m->cfg = c;
  return cudaSuccess;
}

cudaError_t launch_side(TcPlan* p, const TcMaps& m, const SideArgs& a, cudaStream_t st) {
  const int c = m.cfg;
  const int bn = kCfgBN[c];
  const int nTiles = (a.nB + bn - 1) / bn;
  if (nTiles == 0) return cudaSuccess;
  // Persistent grid: one CTA per SM (or fewer when the work is known to be small).
  long long maxWork = (long long)((a.nA + kCfgNB[c] * BM - 1) / (kCfgNB[c] * BM)) * nTiles;
  int grid = (int)std::min<long long>(p->numSMs, std::max<long long>(1, maxWork));
  if (grid * kEpiWarps > a.nSeg) return cudaErrorInvalidValue;
  switch (c) {
    case 0: return launch_cfg<Cfg0, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[0]);
    case 1: return launch_cfg<Cfg1, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[1]);
    case 2: return launch_cfg<Cfg2, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[2]);
    case 3: return launch_cfg<Cfg3, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[3]);
    case 4: return launch_cfg<Cfg4, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[4]);
    case 5: return launch_cfg<Cfg5, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[5]);
    case 6: return launch_cfg<Cfg6, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[6]);
    case 7: return launch_cfg<Cfg7, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[7]);
    case 8: return launch_cfg<Cfg8, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[8]);
    default: return launch_cfg<Cfg9, false>(m.a, m.b, nTiles, a, grid, st, p->attrSet[9]);
  }
}

template <class C>
cudaError_t set_batch_attr(bool& attrSet) {
  if (attrSet) return cudaSuccess;
  const size_t smem = sizeof(Smem<C>) + 1024;
  cudaError_t e = cudaFuncSetAttribute(k_side<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) attrSet = true;
  return e;
}

cudaError_t tc_prepare_batch(TcPlan* p, int cfg) {
  switch (cfg) {
    case 0: return set_batch_attr<Cfg0>(p->attrSetBatch[0]);
    case 1: return set_batch_attr<Cfg1>(p->attrSetBatch[1]);
    case 2: return set_batch_attr<Cfg2>(p->attrSetBatch[2]);
    case 3: return set_batch_attr<Cfg3>(p->attrSetBatch[3]);
    case 4: return set_batch_attr<Cfg4>(p->attrSetBatch[4]);
    case 5: return set_batch_attr<Cfg5>(p->attrSetBatch[5]);
    case 6: return set_batch_attr<Cfg6>(p->attrSetBatch[6]);
    case 7: return set_batch_attr<Cfg7>(p->attrSetBatch[7]);
    case 8: return set_batch_attr<Cfg8>(p->attrSetBatch[8]);
    case 9: return set_batch_attr<Cfg9>(p->attrSetBatch[9]);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_side_batch(TcPlan* p, const TcMaps& m, const SideArgs& a, cudaStream_t st) {
  const int c = m.cfg;
  // Persistent grid: one CTA per SM (fewer when the row count is known to be small).
  int grid = p->numSMs;
  if (!a.nRowsPtr) {
    if (a.nRows <= 0) return cudaSuccess;
    grid = std::min(grid, a.nRows);
  }
  if (grid * kEpiWarps > a.nSeg || a.schedule < 0 || a.schedule > 2) return cudaErrorInvalidValue;
  switch (c) {
    case 0: return launch_cfg<Cfg0, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[0]);
    case 1: return launch_cfg<Cfg1, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[1]);
    case 2: return launch_cfg<Cfg2, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[2]);
    case 3: return launch_cfg<Cfg3, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[3]);
    case 4: return launch_cfg<Cfg4, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[4]);
    case 5: return launch_cfg<Cfg5, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[5]);
    case 6: return launch_cfg<Cfg6, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[6]);
    case 7: return launch_cfg<Cfg7, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[7]);
    case 8: return launch_cfg<Cfg8, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[8]);
    default: return launch_cfg<Cfg9, true>(m.a, m.b, 0, a, grid, st, p->attrSetBatch[9]);
  }
}

// Gathered-A batched pass: one fixed configuration (128 x 128 tiles, six A slots, so that
// several gathers are in flight while short rows are scored).
using CfgG = Cfg6;

int tc_gather_rows() { return CfgG::GM; }
int tc_gather_cols() { return CfgG::BN; }

cudaError_t tc_rows_map(CUtensorMap* m, const uint8_t* base, int rows, int boxRows) {
  if (rows <= 0 || boxRows <= 0 || boxRows > 256) return cudaErrorInvalidValue;
  return encode_rows(m, base, rows, boxRows) ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t tc_gather_map(CUtensorMap* m, const uint8_t* dB, int rowsB) {
  if (rowsB <= 0) return cudaErrorInvalidValue;
  return encode_rows(m, dB, rowsB, CfgG::BN) ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_side_gather(TcPlan* p, const CUtensorMap& mB, const SideArgs& a, cudaStream_t st) {
  int grid = p->numSMs;
  if (!a.nRowsPtr) {
    if (a.nRows <= 0) return cudaSuccess;
    grid = std::min(grid, a.nRows);
  }
  if (grid * kEpiWarps > a.nSeg || a.schedule < 0 || a.schedule > 2 || !a.aSrc || !a.aSrcRow)
    return cudaErrorInvalidValue;
  return launch_cfg<CfgG, true, true>(mB, mB, 0, a, grid, st, p->attrSetGather);
}

}  // namespace v3dm
