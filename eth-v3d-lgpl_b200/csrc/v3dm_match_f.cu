// v3dm_match_f.cu -- float descriptors: scores from a BF16 hi/lo split on the tensor cores.
//
// The reference scores float descriptors with cublasSgemm (v3d_cudamatching.cu:529-530).  For
// descriptors that are not of the exact u/512 form (the integer path's domain), each value x is
// split into hi = bf16(x) and lo = bf16(x - hi), and
//   score(a, b) = hi_a . hi_b + lo_a . hi_b + hi_a . lo_b       (the lo . lo term is dropped)
// is one K = 384 GEMM with FP32 accumulation: A rows hold [hi | lo | hi], B rows [hi | hi | lo]
// (tcgen05.mma.kind::f16, BF16 x BF16 -> F32 in TMEM).  For u/512 inputs hi is exact and lo = 0,
// so the scores equal the integer path's exactly.
//
// Selection is exact for the float scores, in one of two ways.  Tf, the float candidate
// threshold, is the smallest score a second value must reach to change any decision (scores
// below it never matter, see host_float_threshold).
//   - Flat walk (k_side_f<false>: a CTA owns a range of (A group, B tile) items, so a row's
//     scores are spread over CTAs): the side kernel hands over every 32-score chunk whose maximum
//     reaches Tf, and k_records_f / k_decide_f select from those records.
//   - Row walk (k_side_f<true>: a CTA scores a whole row, an A group against every tile of its B
//     side): each epilogue lane keeps its row's best and second in registers and writes the
//     decision itself; gates are tested only where a score could enter those two.
// Batches and pass A of a single pair take the row walk; pass B of a single pair (few chosen
// rights, too few rows to fill the CTAs) takes the flat walk.  No re-score pass exists.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "v3dm_device.cuh"
#include "v3dm_tcgen05.cuh"

namespace v3dm {

namespace {

constexpr int kFM = 128;            // rows per MMA (TMEM lanes)
constexpr int kFN = 128;            // B rows per tile (one MMA is 128 x 128 x 16: narrower MMAs ran 30% slower)
constexpr int kFChunks = kFN / 32;  // 32-column TMEM loads per tile and lane quadrant
constexpr int kFStages = 2;         // ring of 96 KB stages: a B tile or a whole A group
constexpr int kFPlanes = 6;         // 128-byte K planes per row (384 BF16 values)
constexpr int kFSteps = 24;         // K = 16 per MMA
constexpr int kFAcc = 2;            // TMEM accumulator stages of kFN columns
// The A group lives in TMEM during its tiles: it lands in a stage of the ring and is copied once
// (tcgen05.cp) into TMEM, so that shared memory serves the B tiles (the MMA reads 4 KB of B per
// 128x128x16 step instead of 8 KB of A and B) and the two stages hold B tiles between groups.
constexpr int kFAPlanes = 6;        // planes of an A group per ring stage
static_assert(kFAPlanes * kFM == kFPlanes * kFN && kFPlanes % kFAPlanes == 0, "A planes fill whole stages");
constexpr int kFACols = kFPlanes * 32;     // 128-byte K planes, 4 bytes per column: 192 columns
constexpr int kFABase = kFAcc * kFN;       // A after the accumulators
constexpr int kFTmemCols = 512;
static_assert(kFABase + kFACols <= kFTmemCols, "accumulators and the A group fit in TMEM");
constexpr int kFEpiWarps = 4;       // one per TMEM lane quadrant
constexpr int kFThreads = (2 + kFEpiWarps) * 32;

struct SmemF {
  uint8_t b[kFStages][kFPlanes][kFN][128];    // 2 x 96 KB: a B tile, or an A group
  unsigned long long fullB[kFStages], emptyB[kFStages];
  unsigned long long accFull[kFAcc], accEmpty[kFAcc];
  unsigned long long mmaDone;
  uint32_t tmemBase;
  int abort;
};
static_assert(sizeof(SmemF) + 1024 <= 227 * 1024, "shared memory of one CTA");

// kind::f16, D = F32, A = B = BF16, both K-major, M = 128, N = kFN.
__device__ __forceinline__ constexpr uint32_t idesc_f16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kFN >> 3) << 17) | ((uint32_t)(kFM >> 4) << 24);
}

// A from TMEM (lane = row, K values packed two per column), B from shared memory.
__device__ __forceinline__ void mma_bf16_ts(uint32_t dtmem, uint32_t atmem, uint64_t bd, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(dtmem),
      "r"(atmem), "l"(bd), "r"(idesc_f16()), "r"(accumulate)
      : "memory");
}

// A 128-row x 32-byte slice, described as the MMA would read it from shared memory, into TMEM
// (row i to lane i, 8 columns); executes in issue order with the MMAs of the same thread.
__device__ __forceinline__ void tmem_cp_slice(uint32_t taddr, uint64_t sd) {
  asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(taddr), "l"(sd) : "memory");
}

__device__ __forceinline__ float fmax32(const float* v) {
  float m[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) m[i] = fmaxf(v[i], v[i + 16]);
#pragma unroll
  for (int i = 0; i < 8; ++i) m[i] = fmaxf(m[i], m[i + 8]);
#pragma unroll
  for (int i = 0; i < 4; ++i) m[i] = fmaxf(m[i], m[i + 4]);
  return fmaxf(fmaxf(m[0], m[2]), fmaxf(m[1], m[3]));
}

// The work of one CTA, in the order every role walks it.  One pair (kBatch false): the flat range
// of (A group of 128 rows, B tile of 128 columns) this CTA owns.  A batch (kBatch true): the rows of
// the row table interleaved over the CTAs (row r, r + gridDim.x, ...), each an A group of one image
// against every 128-column tile of its B image; a row's state indices are state0 + its rows.  With
// no row table (a.rows null) the rows are those of one pair: row r is A rows 128r .. against all
// a.nB B rows, its states the A row indices.
template <bool kBatch>
struct FWalk {
  // one pair
  long long w, w1;
  int nTiles, nA, nB0;
  const int* amap;
  // batch
  const BatchRow* rows;
  int r, nRows, pairA, pairB;
  BatchRow cur;
  // the current item
  int t;          // B tile of the A group
  bool newA;      // the A group changes here
  __device__ void init_pair(const SideArgs& a, int nA_) {
    nA = nA_;
    nB0 = a.nB;
    amap = a.amap;
    nTiles = (a.nB + kFN - 1) / kFN;
    const long long nWork = (long long)((nA + kFM - 1) / kFM) * nTiles;
    w = nWork * blockIdx.x / gridDim.x;
    w1 = nWork * (blockIdx.x + 1) / gridDim.x;
    t = nTiles > 0 ? (int)(w % nTiles) : 0;
    newA = true;
  }
  __device__ BatchRow row_at(int rr) const {
    if (rows) return rows[rr];
    BatchRow b;
    b.aRow = rr * kFM;
    b.validRows = min(kFM, pairA - rr * kFM);
    b.bRow0 = 0;
    b.nB = pairB;
    b.nTiles = (pairB + kFN - 1) / kFN;
    b.pad = 0;
    b.state0 = (long long)rr * kFM;
    return b;
  }
  __device__ void init_batch(const SideArgs& a) {
    rows = a.rows;
    pairA = a.nA;
    pairB = a.nB;
    nRows = rows ? (a.nRowsPtr ? *a.nRowsPtr : a.nRows) : (pairB > 0 ? (pairA + kFM - 1) / kFM : 0);
    r = blockIdx.x;
    t = 0;
    newA = true;
    if (r < nRows) cur = row_at(r);
  }
  __device__ bool more() const {
    if constexpr (kBatch) return r < nRows;
    else return w < w1;
  }
  __device__ void next() {
    if constexpr (kBatch) {
      if (++t < cur.nTiles) {
        newA = false;
        return;
      }
      r += gridDim.x;
      t = 0;
      newA = true;
      if (r < nRows) cur = row_at(r);
    } else {
      ++w;
      t = (int)(w % nTiles);
      newA = t == 0;
    }
  }
  __device__ int aRow() const {
    if constexpr (kBatch) return cur.aRow;
    else return (int)(w / nTiles) * kFM;
  }
  __device__ int bRow() const {
    if constexpr (kBatch) return cur.bRow0 + t * kFN;
    else return t * kFN;
  }
  __device__ int nB() const {
    if constexpr (kBatch) return cur.nB;
    else return nB0;
  }
  // the current tile is the last of its A group's row (batch walk only)
  __device__ bool lastOfA() const { return t + 1 == cur.nTiles; }
  // the state of row i (0..127) of the current A group, or -1 past its valid rows
  __device__ long long state(int i) const {
    if constexpr (kBatch) return i < cur.validRows ? cur.state0 + i : -1;
    else {
      const int row = (int)(w / nTiles) * kFM + i;
      return row < nA ? (amap ? amap[row] : row) : -1;
    }
  }
};

// Running top two of one A row over the columns of a batch row, as ordered keys (f32_order; 0:
// none): b1 the largest, c1 its first column, b2 the largest of the other columns.
__device__ __forceinline__ void top2_push(uint32_t key, int col, uint32_t& b1, uint32_t& b2, int& c1) {
  b2 = max(b2, min(key, b1));
  c1 = key > b1 ? col : c1;
  b1 = max(b1, key);
}

// The gate of one lane's row in a guided batch (one gate per pair, the reference's expressions):
// its pair's matrix and thr^2, the positions of the B image's descriptors, the A descriptor's
// terms.
struct GateLane {
  const float* m;
  const float2* bPos;
  float4 aT;
  int type, aIsLeft;
};

// Whether the gate masks (A descriptor of the lane, column col of the B image).  Called only for
// scores that could enter the lane's top two, so it stays out of line.
__device__ __noinline__ bool gate_rejects_col(GateLane gl, int col) {
  const float2 pb = gl.bPos[col];
  if (gl.aIsLeft) return gate_rejects_terms(gl.type, gl.m[9], gl.aT, gate_right_terms(gl.type, gl.m, pb));
  return gate_rejects_terms(gl.type, gl.m[9], gate_left_terms(gl.type, gl.m, pb), gl.aT);
}

// Whether any of the single-pair matcher's gates (compounding since the last putative call) masks
// (left l, right r); out of line for the same reason.
__device__ __noinline__ bool gates_reject(const GateParams* gates, int n, int l, int r) {
  for (int g = 0; g < n; ++g)
    if (gate_rejects(gates[g], l, r)) return true;
  return false;
}

// Side A against side B.  One pair (kBatch false): nA rows (amap as in k_side) against nB rows;
// the epilogue hands every 32-score chunk whose maximum reaches Tf to k_records_f.  A batch
// (kBatch true): the row table; one CTA scores a row's A group against every tile of its B
// image, so each epilogue thread keeps its A row's exact best and second over the whole image in
// registers and writes the row's decision (a.decision[state]) after the last tile.  That is
// what k_records_f and k_decide_f make of the chunk records: the best is the largest key (first
// column on ties), the second the largest other key, both kept only when their score reaches Tf
// (a non-best candidate reaches Tf only if the second does).  Same roles and bounded waits as
// k_side; the A group is single-buffered (96 KB).  With 'dump' set (small one-pair diagnostic
// calls) every score is also written to dump[index * nB + column].
template <bool kBatch>
__global__ void __launch_bounds__(kFThreads, 1)
k_side_f(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, SideArgs a, float Tf,
         float* dump) {
  pdl_wait();
  pdl_launch_dependents();
  extern __shared__ uint8_t smemRaw[];
  SmemF& s = *reinterpret_cast<SmemF*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  FWalk<kBatch> start;
  if constexpr (kBatch) {
    start.init_batch(a);
  } else {
    start.init_pair(a, a.nAptr ? *a.nAptr : a.nA);
  }
  if (!start.more()) {
    if (!kBatch && warp >= 2 && lane == 0) a.segCount[blockIdx.x * kFEpiWarps + (warp - 2)] = 0;
    return;
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < kFStages; ++i) {
      mbar_init(&s.fullB[i], 1);
      mbar_init(&s.emptyB[i], 1);
    }
    for (int i = 0; i < kFAcc; ++i) {
      mbar_init(&s.accFull[i], 1);
      mbar_init(&s.accEmpty[i], kFEpiWarps);
    }
    mbar_init(&s.mmaDone, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmemBase)),
                 "r"(kFTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmemBase;
  __syncthreads();

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0 && !s.abort) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armedPhase[kFStages] = {};
      bool armed[kFStages] = {};
      for (FWalk<kBatch> wk = start; wk.more(); wk.next()) {
        if (wk.newA) {
          // the A group through the ring (kFAPlanes planes per stage)
          bool stop = false;
#pragma unroll
          for (int h = 0; h < kFPlanes / kFAPlanes; ++h) {
            if (!mbar_wait(&s.emptyB[stage], phase ^ 1, &s.abort, a.err)) {
              stop = true;
              break;
            }
            mbar_expect_tx(&s.fullB[stage], (uint32_t)sizeof(s.b[0]));
            tma_load_3d(&s.b[stage][0][0][0], &tmA, &s.fullB[stage], 0, wk.aRow(), h * kFAPlanes);
            armed[stage] = true;
            armedPhase[stage] = phase;
            if (++stage == kFStages) {
              stage = 0;
              phase ^= 1;
            }
          }
          if (stop) break;
        }
        if (!mbar_wait(&s.emptyB[stage], phase ^ 1, &s.abort, a.err)) break;
        mbar_expect_tx(&s.fullB[stage], (uint32_t)sizeof(s.b[0]));
        tma_load_3d(&s.b[stage][0][0][0], &tmB, &s.fullB[stage], 0, wk.bRow(), 0);
        armed[stage] = true;
        armedPhase[stage] = phase;
        if (++stage == kFStages) {
          stage = 0;
          phase ^= 1;
        }
      }
      // Drain: every load this thread issued has landed before the CTA may exit.
      for (int i = 0; i < kFStages; ++i)
        if (armed[i]) {
          long long t0c = clock64();
          while (!mbar_try(&s.fullB[i], armedPhase[i]) && clock64() - t0c < kWaitCycles) {
          }
        }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0 && !s.abort) {
      int stage = 0, acc = 0;
      uint32_t phase = 0, accPhase = 0;
      const uint32_t aT = tmem + (uint32_t)kFABase;
      for (FWalk<kBatch> wk = start; wk.more(); wk.next()) {
        if (wk.newA) {
          // the group into TMEM (after the previous group's MMAs, which were issued first); its
          // stage is free once the copies are done
          bool stop = false;
#pragma unroll
          for (int h = 0; h < kFPlanes / kFAPlanes; ++h) {
            if (!mbar_wait(&s.fullB[stage], phase, &s.abort, a.err)) {
              stop = true;
              break;
            }
            tc_fence_after();
            const uint32_t sb = smem_u32(&s.b[stage][0][0][0]);
#pragma unroll
            for (int kk = 0; kk < 4 * kFAPlanes; ++kk)
              tmem_cp_slice(aT + (uint32_t)(8 * (h * 4 * kFAPlanes + kk)),
                            sdesc(sb + (uint32_t)(kk >> 2) * (kFM * 128) + (uint32_t)((kk & 3) * 32)));
            mma_commit(&s.emptyB[stage]);
            if (++stage == kFStages) {
              stage = 0;
              phase ^= 1;
            }
          }
          if (stop) break;
        }
        if (!mbar_wait(&s.accEmpty[acc], accPhase ^ 1, &s.abort, a.err)) break;
        if (!mbar_wait(&s.fullB[stage], phase, &s.abort, a.err)) break;
        tc_fence_after();
        const uint32_t bBase = smem_u32(&s.b[stage][0][0][0]);
        const uint32_t d = tmem + (uint32_t)(acc * kFN);
#pragma unroll
        for (int k = 0; k < kFSteps; ++k) {
          const uint32_t off = (uint32_t)((k & 3) * 32);
          const uint32_t pl = (uint32_t)(k >> 2);
          mma_bf16_ts(d, aT + (uint32_t)(8 * k), sdesc(bBase + pl * (kFN * 128) + off), k > 0 ? 1u : 0u);
        }
        mma_commit(&s.emptyB[stage]);
        mma_commit(&s.accFull[acc]);
        if (++stage == kFStages) {
          stage = 0;
          phase ^= 1;
        }
        if (++acc == kFAcc) {
          acc = 0;
          accPhase ^= 1;
        }
      }
      // Every MMA this thread issued has completed before TMEM is released.
      mma_commit(&s.mmaDone);
      long long t0c = clock64();
      while (!mbar_try(&s.mmaDone, 0) && clock64() - t0c < kWaitCycles) {
      }
    }
  } else if constexpr (kBatch) {
    // ---------------- epilogue (batch rows: decisions) ----------------
    const int q = warp & 3;
    int acc = 0;
    uint32_t accPhase = 0;
    bool ok = !s.abort;
    long long st = -1;
    uint32_t b1 = 0, b2 = 0;
    int c1 = 0;
    const bool gated = a.bg.on != 0 || a.nGates > 0;
    GateLane gl{};
    for (FWalk<kBatch> wk = start; wk.more() && ok; wk.next()) {
      if (wk.newA) {
        st = wk.state(q * 32 + lane);
        b1 = b2 = 0u;
        c1 = 0;
        if (a.bg.on && st >= 0) {
          int pair = 0, aIdx = 0;
          bgate_resolve(a.bg, a.aIsLeft, st, &pair, &aIdx);
          const int2 lr = a.bg.pairLR[pair];
          const int aImg = a.aIsLeft ? lr.x : lr.y, bImg = a.aIsLeft ? lr.y : lr.x;
          gl.m = a.bg.gm + (size_t)pair * kBGateFloats;
          gl.type = a.bg.type;
          gl.aIsLeft = a.aIsLeft;
          const float2 pa = a.bg.pos[a.bg.posOff[aImg] + aIdx];
          gl.aT = a.aIsLeft ? gate_left_terms(gl.type, gl.m, pa) : gate_right_terms(gl.type, gl.m, pa);
          gl.bPos = a.bg.pos + a.bg.posOff[bImg];
        }
      }
      const int nB = wk.nB();
      ok = mbar_wait(&s.accFull[acc], accPhase, &s.abort, a.err);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kFN);
      uint32_t v[kFChunks][32];
#pragma unroll
      for (int c = 0; c < kFChunks; ++c) tmem_ld32(tbase + (uint32_t)(32 * c), v[c]);
#pragma unroll
      for (int c = 0; c < kFChunks; ++c) tmem_wait(v[c]);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s.accEmpty[acc]);
      const int col0 = wk.t * kFN;
      if (gated) {
        // a masked score counts as none (the reference's -1e20 is below Tf); the gate is tested
        // only where a score could enter the top two (a key <= b2 leaves them unchanged)
        const bool full = col0 + kFN <= nB;
#pragma unroll
        for (int c = 0; c < kFChunks; ++c)
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            const int col = col0 + 32 * c + k;
            uint32_t key = (full || col < nB) ? f32_order(__uint_as_float(v[c][k])) : 0u;
            if (key > b2) {
              if (st >= 0) {
                const bool masked = a.bg.on ? gate_rejects_col(gl, col)
                                            : gates_reject(a.gatesDev, a.nGates, a.aIsLeft ? (int)st : col,
                                                           a.aIsLeft ? col : (int)st);
                if (masked) key = 0u;
              }
              top2_push(key, col, b1, b2, c1);
            }
          }
      } else if (col0 + kFN <= nB) {  // warp-uniform: a full tile
#pragma unroll
        for (int c = 0; c < kFChunks; ++c)
#pragma unroll
          for (int k = 0; k < 32; ++k) top2_push(f32_order(__uint_as_float(v[c][k])), col0 + 32 * c + k, b1, b2, c1);
      } else {
#pragma unroll
        for (int c = 0; c < kFChunks; ++c)
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            const int col = col0 + 32 * c + k;
            top2_push(col < nB ? f32_order(__uint_as_float(v[c][k])) : 0u, col, b1, b2, c1);
          }
      }
      if (wk.lastOfA() && st >= 0) {
        const float s1 = f32_unorder(b1), s2 = f32_unorder(b2);
        const unsigned long long bk = (b1 != 0u && s1 >= Tf) ? best_key_f(s1, c1) : 0ull;
        const uint32_t so = (b2 != 0u && s2 >= Tf) ? b2 : 0u;
        a.decision[st] = decide_f(bk, so, a.minScore, a.minRatio);
      }
      if (++acc == kFAcc) {
        acc = 0;
        accPhase ^= 1;
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int e = warp - 2;
    const int q = warp & 3;
    uint4* const segBase = a.records + (long long)(blockIdx.x * kFEpiWarps + e) * a.segCap * kRecordQuads;
    int segN = 0;
    int acc = 0;
    uint32_t accPhase = 0;
    bool ok = !s.abort;
    long long st = -1;
    for (FWalk<kBatch> wk = start; wk.more() && ok; wk.next()) {
      if (wk.newA) st = wk.state(q * 32 + lane);
      const bool rowValid = st >= 0;
      const int orig = rowValid ? (int)st : 0;
      const int nB = wk.nB();
      ok = mbar_wait(&s.accFull[acc], accPhase, &s.abort, a.err);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kFN);
      uint32_t v[kFChunks][32];
#pragma unroll
      for (int c = 0; c < kFChunks; ++c) tmem_ld32(tbase + (uint32_t)(32 * c), v[c]);
#pragma unroll
      for (int c = 0; c < kFChunks; ++c) tmem_wait(v[c]);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s.accEmpty[acc]);
#pragma unroll
      for (int c = 0; c < kFChunks; ++c) {
        const int col0 = wk.t * kFN + 32 * c;
        if (col0 >= nB) break;  // warp-uniform
        float f[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) f[k] = (col0 + k < nB) ? __uint_as_float(v[c][k]) : -INFINITY;
        if (!kBatch && dump && rowValid)
          for (int k = 0; k < 32 && col0 + k < nB; ++k) dump[(size_t)orig * nB + col0 + k] = f[k];
        const float mx = fmax32(f);
        const bool trig = rowValid && mx >= Tf;
        if (__any_sync(0xffffffffu, trig)) {
          const unsigned m = __ballot_sync(0xffffffffu, trig);
          if (trig) {
            const int idx = segN + __popc(m & ((1u << lane) - 1u));
            if (idx < a.segCap) {
              uint4* rec = segBase + (long long)idx * kRecordQuads;
              rec[0] = make_uint4((uint32_t)orig, (uint32_t)col0, (uint32_t)nB, 0u);
#pragma unroll
              for (int k = 0; k < 8; ++k)
                rec[1 + k] = make_uint4(v[c][4 * k], v[c][4 * k + 1], v[c][4 * k + 2], v[c][4 * k + 3]);
            }
          }
          segN += __popc(m);
        }
      }
      if (++acc == kFAcc) {
        acc = 0;
        accPhase ^= 1;
      }
    }
    if (lane == 0) a.segCount[blockIdx.x * kFEpiWarps + e] = segN;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFTmemCols)
                              : "memory");
}

// Exact float selection on the chunk records: every unmasked score >= Tf is a candidate; the
// chunk best is the largest candidate (first column on ties), the other candidates bound the
// second value.  Scores below Tf (and masked ones, which the reference sets to -1e20) cannot
// change a decision and are left out.  Chunk bests merge as in k_records (the key that loses
// the atomic comparison is a second candidate); the lane layout is k_records' as well (eight
// lanes per record, four scores each, four records per warp at a time).
__global__ void k_records_f(PostArgs a, float Tf) {
  pdl_wait();
  pdl_launch_dependents();
  int32_t* info = a.err - kInfoErr;
  const int lane = threadIdx.x & 31;
  const int grp = lane >> 3, part = lane & 7;
  const int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int seg = warpGlobal; seg < a.nSeg; seg += nWarps) {
    const int cnt = a.segCount[seg];
    if (cnt == 0) continue;
    const int n = (long long)cnt < a.segCap ? cnt : (int)a.segCap;
    const uint4* recs = a.records + (long long)seg * a.segCap * kRecordQuads;
    for (int i0 = 0; i0 < n; i0 += 4) {
      const int i = i0 + grp;
      const bool have = i < n;
      uint4 head = make_uint4(0u, 0u, 0u, 0u), q = head;
      if (have) {
        head = recs[(long long)i * kRecordQuads];
        q = recs[(long long)i * kRecordQuads + 1 + part];
      }
      const int orig = (int)head.x, col0 = (int)head.y, nB = (int)head.z;
      const uint32_t sv[4] = {q.x, q.y, q.z, q.w};
      unsigned long long key[4];
      unsigned long long cb = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int col = col0 + 4 * part + t;
        const float sc = __uint_as_float(sv[t]);
        bool cand = have && col < nB && sc >= Tf;
        for (int gi = 0; gi < a.nGates && cand; ++gi)
          cand = !gate_rejects(a.gatesDev[gi], a.aIsLeft ? orig : col, a.aIsLeft ? col : orig);
        key[t] = cand ? best_key_f(sc, col) : 0ull;
        cb = key[t] > cb ? key[t] : cb;
      }
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, cb, off);
        cb = o > cb ? o : cb;
      }
      uint32_t cw = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (key[t] != 0ull && key[t] != cb) cw = max(cw, (uint32_t)(key[t] >> kIndexBits));
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) cw = max(cw, __shfl_xor_sync(0xffffffffu, cw, off));
      if (have && part == 0) {
        if (cb) {
          const unsigned long long old = atomicMax(&a.best[orig], cb);
          if (old && old != cb) atomicMax(&a.sec[orig], (unsigned)((old < cb ? old : cb) >> kIndexBits));
        }
        if (cw) atomicMax(&a.sec[orig], cw);
      }
    }
    if (lane == 0) {
      if ((long long)cnt > a.segCap) atomicMax(&info[kInfoMaxSeg], cnt);  // overflow only
      a.segCount[seg] = 0;
    }
  }
}

__global__ void k_decide_f(PostArgs a) {
  pdl_wait();
  pdl_launch_dependents();
  const int lane = threadIdx.x & 31;
  const int nRows = a.rowsPtr ? *a.rowsPtr : a.nRows;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nRows; r += gridDim.x * blockDim.x) {
    const int idx = a.amap ? a.amap[r] : r;
    const unsigned long long b = a.best[idx];
    const unsigned s = a.sec[idx];
    const int32_t d = decide_f(b, s, a.minScore, a.minRatio);
    a.decision[idx] = d;
    if (a.chooseFlag) {
      // chosen for pass B: listed once (the claiming lanes of a warp take consecutive slots
      // with one counter update), planar row gathered
      const bool claim = d >= 0 && atomicExch(&a.chooseFlag[d], 1) == 0;
      const unsigned act = __activemask();
      const unsigned m = __ballot_sync(act, claim);
      if (m) {
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(a.chooseCount, __popc(m));
        base = __shfl_sync(act, base, leader);
        if (claim) {
          const int k = base + __popc(m & ((1u << lane) - 1u));
          a.chooseList[k] = d;
          for (int p = 0; p < kFPlanes; ++p) {
            const uint4* src = reinterpret_cast<const uint4*>(a.chooseSrc + ((size_t)p * a.chooseCapSrc + d) * 128);
            uint4* dst = reinterpret_cast<uint4*>(a.chooseDst + ((size_t)p * a.chooseCapDst + k) * 128);
#pragma unroll
            for (int w = 0; w < 8; ++w) dst[w] = src[w];
          }
        }
      }
    }
    if (b) a.best[idx] = 0;
    if (s) a.sec[idx] = 0;
  }
}

// A and B layouts of n descriptors: float values (or uint8 values u, read as u / 512) split
// into BF16 hi and lo.  A row = [hi | lo | hi], B row = [hi | hi | lo] (384 values along K),
// stored planar: plane p holds K positions 64p .. 64p + 63 of every row, rowsCap rows of 128 B
// per plane.  Sets *err when a value is not finite.  With srcOff set, the n descriptors are the
// concatenation of nImages images (image i starts at descriptor srcOff[i], ascending) and image
// i's descriptors go to rows rowOff[i] onwards; otherwise descriptor d goes to row d.
__global__ void k_hilo(const float* __restrict__ f, const uint8_t* __restrict__ u, long long n, int rowsCap,
                       __nv_bfloat16* __restrict__ la, __nv_bfloat16* __restrict__ lb, int* err,
                       const long long* __restrict__ srcOff, const int* __restrict__ rowOff, int nImages) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kDescBytes) return;
  const long long src = i / kDescBytes;
  long long d = src;
  if (srcOff) {
    int lo = 0, hi = nImages - 1;  // last image whose first descriptor is <= src
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (srcOff[mid] <= src) lo = mid;
      else hi = mid - 1;
    }
    d = rowOff[lo] + (src - srcOff[lo]);
  }
  const int k = (int)(i % kDescBytes);
  const float x = f ? f[i] : (float)u[i] * (1.0f / 512.0f);
  if (!isfinite(x)) atomicOr(err, kErrNotU8);
  const __nv_bfloat16 hi = __float2bfloat16_rn(x);
  const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
  const int half = k >> 6, off = k & 63;
  auto at = [&](__nv_bfloat16* base, int seg) -> __nv_bfloat16& {
    return base[((size_t)(2 * seg + half) * rowsCap + d) * 64 + off];
  };
  at(la, 0) = hi;
  at(la, 1) = lo;
  at(la, 2) = hi;
  at(lb, 0) = hi;
  at(lb, 1) = hi;
  at(lb, 2) = lo;
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode_f() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 3-D BF16 map over a planar layout (64 values of a K slice, row, plane), box (64, boxRows,
// boxPlanes), 128-byte swizzle: one load fills boxPlanes swizzled [boxRows][128 B] blocks.
bool encode_f(CUtensorMap* map, const void* base, int rows, int boxRows, int boxPlanes) {
  auto fn = get_encode_f();
  if (!fn) return false;
  cuuint64_t dims[3] = {64, (cuuint64_t)rows, (cuuint64_t)kFPlanes};
  cuuint64_t strides[2] = {128, (cuuint64_t)rows * 128};
  cuuint32_t box[3] = {64, (cuuint32_t)boxRows, (cuuint32_t)boxPlanes};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

int f_segments(int numSMs) { return numSMs * kFEpiWarps; }

cudaError_t f_maps(CUtensorMap* mA, const void* dA, int rowsA, CUtensorMap* mB, const void* dB, int rowsB) {
  if (rowsA < kFM || rowsB < kFN) return cudaErrorInvalidValue;
  if (!encode_f(mA, dA, rowsA, kFM, kFAPlanes) || !encode_f(mB, dB, rowsB, kFN, kFPlanes))
    return cudaErrorInvalidValue;
  return cudaSuccess;
}

cudaError_t launch_side_f(const CUtensorMap& mA, const CUtensorMap& mB, const SideArgs& a, float Tf, float* dump,
                          int numSMs, cudaStream_t st) {
  const size_t smem = sizeof(SmemF) + 1024;
  static bool attrSet[128] = {};  // per device ordinal
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
  if (!attrSet[dev]) {
    e = cudaFuncSetAttribute(k_side_f<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attrSet[dev] = true;
  }
  const int nTiles = (a.nB + kFN - 1) / kFN;
  if (nTiles == 0) return cudaSuccess;
  const long long maxWork = (long long)((a.nA + kFM - 1) / kFM) * nTiles;
  const int grid = (int)std::min<long long>(numSMs, std::max<long long>(1, maxWork));
  if (grid * kFEpiWarps > a.nSeg) return cudaErrorInvalidValue;
  return launch_pdl(k_side_f<false>, dim3(grid), dim3(kFThreads), smem, st, mA, mB, a, Tf, dump);
}

cudaError_t launch_side_f_batch(const CUtensorMap& mA, const CUtensorMap& mB, const SideArgs& a, float Tf,
                                int numSMs, cudaStream_t st) {
  const size_t smem = sizeof(SmemF) + 1024;
  static bool attrSet[128] = {};  // per device ordinal
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
  if (!attrSet[dev]) {
    e = cudaFuncSetAttribute(k_side_f<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attrSet[dev] = true;
  }
  int grid = numSMs;
  if (!a.rows) {  // one pair: its rows are implicit
    if (a.nA <= 0 || a.nB <= 0) return cudaSuccess;
    grid = std::min(grid, (a.nA + kFM - 1) / kFM);
  } else if (!a.nRowsPtr) {
    if (a.nRows <= 0) return cudaSuccess;
    grid = std::min(grid, a.nRows);
  }
  if (!a.decision) return cudaErrorInvalidValue;
  return launch_pdl(k_side_f<true>, dim3(grid), dim3(kFThreads), smem, st, mA, mB, a, Tf, (float*)nullptr);
}

int f_group_rows() { return kFM; }
int f_tile_cols() { return kFN; }

cudaError_t launch_post_f(const PostArgs& a, float Tf, cudaStream_t s) {
  const int listBlocks = (a.nSeg * 32 + 255) / 256;
  cudaError_t e = launch_pdl(k_records_f, dim3(listBlocks < 512 ? listBlocks : 512), dim3(256), 0, s, a, Tf);
  if (e != cudaSuccess) return e;
  const int rows = a.nRows > 0 ? a.nRows : 1;
  const int blocks = (rows + 255) / 256;
  return launch_pdl(k_decide_f, dim3(blocks < 1024 ? blocks : 1024), dim3(256), 0, s, a);
}

cudaError_t launch_hilo(const float* f, const uint8_t* u, int n, int rowsCap, void* la, void* lb, int* err,
                        cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (n > rowsCap) return cudaErrorInvalidValue;
  const long long total = (long long)n * kDescBytes;
  k_hilo<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(f, u, n, rowsCap, static_cast<__nv_bfloat16*>(la),
                                                         static_cast<__nv_bfloat16*>(lb), err, nullptr, nullptr, 0);
  return cudaGetLastError();
}

cudaError_t launch_hilo_images(const float* f, long long n, const long long* srcOff, const int* rowOff, int nImages,
                               int rowsCap, void* la, void* lb, int* err, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (nImages <= 0 || !srcOff || !rowOff) return cudaErrorInvalidValue;
  const long long total = n * kDescBytes;
  k_hilo<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(f, nullptr, n, rowsCap, static_cast<__nv_bfloat16*>(la),
                                                         static_cast<__nv_bfloat16*>(lb), err, srcOff, rowOff,
                                                         nImages);
  return cudaGetLastError();
}

// Smallest float score a second value must reach to change any decision.  accept(s1, s2) is
// monotone: for a fixed s1 it can only turn false as s2 grows, for a fixed s2 only true as s1
// grows, so the boundary at s1 = the smallest float above minScore bounds every s1.  Without a
// ratio test (or when no second value can matter) only candidates above minScore are needed.
float host_float_threshold(float minScore, float minRatio) {
  const float s1min = std::nextafter(minScore, INFINITY);
  if (!(minRatio == minRatio) || minRatio < 0.0f || !(minScore == minScore)) return s1min;
  if (!accept_scores(s1min, kNone, minScore, minRatio)) return s1min;
  if (accept_scores(s1min, INFINITY, minScore, minRatio)) return s1min;
  // accept(s1min, unorder(lo)) is true, accept(s1min, unorder(hi)) false
  uint32_t lo = f32_order(kNone), hi = f32_order(INFINITY);
  while (hi - lo > 1) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (accept_scores(s1min, f32_unorder(mid), minScore, minRatio)) lo = mid;
    else hi = mid;
  }
  const float t = f32_unorder(hi);  // the smallest second value that can flip a decision
  return t < s1min ? t : s1min;
}

}  // namespace v3dm
