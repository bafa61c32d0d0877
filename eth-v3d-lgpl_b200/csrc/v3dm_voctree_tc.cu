// v3dm_voctree_tc.cu -- tensor-core descent of uint8 vocabulary trees (sm_100a).
//
// The reference descends one key per 32-thread block, level by level, with a dot product per
// child (V3D/CUDA/v3d_cudamatching.cu:745-792).  Here the keys are grouped so that the child
// rows they score are shared, and the scoring is a tcgen05 int8 GEMM:
//   - a phase descends up to two levels below a bucket node r (the root for the first phase):
//     level a scores r's BF children, level b all BF^2 grandchildren (children of node
//     (r + 1) BF + c are the BF rows from ((r + 1) BF + c + 1) BF, so the grandchildren are one
//     contiguous block of BF^2 rows, BFS order);
//   - the CTA stages that subtree (BF + BF^2 rows) in shared memory once per work item and
//     multiplies tiles of 128 keys of the bucket by it in one MMA chain (K = 128, u8 x u8 ->
//     s32 in TMEM, N = BF^2 rounded up to 16, plus 16): its first columns are D2 = keys x
//     grandchildren, its last 16 D1 = keys x children (the B rows are laid out that way);
//   - the epilogue (one key per thread, its row of D1 and D2 read with tcgen05.ld) takes the
//     first child with the largest D1 score (strict '>', .cu:781), then the BF scores of that
//     child's children out of D2 (a select network over the chosen child) and again the first
//     largest.  Scoring all BF^2 grandchildren costs BF times the MMA work of the BF needed,
//     which the tensor core absorbs; no dp4a is left.
// Between phases the keys are sorted by the node they reached (k_vt_scan / k_vt_scatter in
// v3dm_voctree.cu), so every bucket's keys come as consecutive positions of a permutation.  The
// dot products are exact integers (at most 255 * 255 * 128 < 2^23), so the leaf ids are the
// reference's whatever the summation order; ties keep the first child.
//
// Roles (one persistent CTA per SM, 352 threads):
//   warps 0-1   producers, alternate tiles: the first phase's keys are consecutive and come as
//               one TMA tile (128 rows, 128-byte swizzle); later phases gather their rows through
//               the permutation with cp.async (16-byte chunks into the same swizzle, eight lanes
//               per row, rows past the bucket zero), each lane's copies completing on the slot's
//               mbarrier (cp.async.mbarrier.arrive).  Producer 0 also loads every item's
//               subtree rows with TMA (boxes of 16 rows) into a ring of B buffers; the
//               rows past the BF children and BF^2 grandchildren that a box brings along only fill
//               columns the epilogue never reads;
//   warp 2      allocates 512 TMEM columns and issues the MMAs of a tile into one of
//               512 / (N2 + 16) accumulator stages;
//   warps 3-10  epilogue, two warps per TMEM lane quadrant taking alternate tiles.
// Every mbarrier wait is bounded (kWaitCycles); on timeout the CTA records kErrWaitTimeout,
// drains its own copies and MMAs, frees TMEM and returns.
#include <cuda.h>

#include <algorithm>

#include "v3dm_device.cuh"
#include "v3dm_tcgen05.cuh"

namespace v3dm {

namespace {

constexpr int kVtcProducers = 2;                // producer warps, taking alternate tiles
constexpr int kVtcMmaWarp = kVtcProducers;      // the MMA issuer's warp
constexpr int kVtcEpiWarp0 = kVtcProducers + 1; // first epilogue warp
constexpr int kVtcEpiHalves = 2;                // epilogue warps per TMEM lane quadrant
constexpr int kVtcThreads = (kVtcEpiWarp0 + 4 * kVtcEpiHalves) * 32;
constexpr int kVtcRows = 128;                   // keys per tile (TMEM lanes)
constexpr int kVtcASlots = 6;                   // key-tile ring depth
constexpr int kVtcTmemCols = 512;
constexpr int kVtcLocalBins = 4096;             // next-phase histogram kept in shared memory up to this
constexpr int kVtcItemKeys = 2048;              // keys per implicit item of a single-bucket phase

template <int BF>
struct VtcShape {
  static constexpr int N2 = (BF * BF + 15) / 16 * 16;   // grandchildren columns (MMA N)
  static constexpr int N1 = 16;                         // children columns
  static constexpr int kRowsB = N2 + N1;                // B rows: grandchildren, then children
  static constexpr int kAccCols = N2 + N1;
  static constexpr int kAcc = kVtcTmemCols / kAccCols;  // accumulator stages
  static constexpr int kABytes = kVtcRows * kDescBytes;
  static constexpr int kBBytes = kRowsB * kDescBytes;
  static constexpr int kBBufs = kBBytes <= 16384 ? 4 : 2;  // subtree ring depth
  static_assert(BF >= 2 && BF <= 15, "branching factor");
  static_assert(kAcc >= 2, "two accumulator stages");
};

template <int BF>
struct VtcSmem {
  using S = VtcShape<BF>;
  uint8_t a[kVtcASlots][S::kABytes];
  uint8_t b[S::kBBufs][S::kBBytes];
  int hist[kVtcLocalBins];
  unsigned long long fullA[kVtcASlots], emptyA[kVtcASlots], fullB[S::kBBufs], emptyB[S::kBBufs];
  unsigned long long accFull[S::kAcc], accEmpty[S::kAcc], mmaDone;
  uint32_t tmemBase;
  int abort;
};

// Instruction descriptor: kind::i8, D = s32, A = B = unsigned 8-bit, both K-major, M = 128.
template <int N>
__device__ __forceinline__ constexpr uint32_t vtc_idesc() {
  return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kVtcRows >> 4) << 24);
}

template <int N>
__device__ __forceinline__ void vtc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(vtc_idesc<N>()), "r"(accumulate)
      : "memory");
}

// Non-blocking test of an mbarrier phase.
__device__ __forceinline__ bool mbar_test(unsigned long long* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void vtc_cp16(uint32_t dst, const void* src, uint32_t srcBytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
}
// Raises the mbarrier's pending count by one now and arrives once every cp.async this thread has
// issued so far has completed (so the phase cannot complete before the copies have landed).
__device__ __forceinline__ void vtc_cp_arrive(unsigned long long* bar) {
  asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void vtc_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 16 TMEM columns of this warp's 32 lanes; valid after tmem_wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

// The work walk every role follows: the CTA's items (it = blockIdx.x, += gridDim.x), each cut
// into tiles of 128 keys.  The next item is loaded one item ahead (small items follow each
// other quickly).
struct VtcWalk {
  const int4* items;
  int nIt, it, t, single;
  int4 item, pre;
  // single > 0: one bucket of `single` keys, cut into items of kVtcItemKeys in order
  __device__ int4 load(int i) const {
    if (i >= nIt) return make_int4(0, 0, 0, 0);
    if (single > 0) return make_int4(0, i * kVtcItemKeys, min(kVtcItemKeys, single - i * kVtcItemKeys), 0);
    return __ldg(items + i);
  }
  __device__ bool start(const int4* its, int n, int singleN) {
    items = its;
    nIt = n;
    single = singleN;
    it = blockIdx.x;
    t = 0;
    if (it >= nIt) return false;
    item = load(it);
    pre = load(it + gridDim.x);
    return true;
  }
  __device__ bool first() const { return t == 0; }
  __device__ bool last() const { return (t + 1) * kVtcRows >= item.z; }
  // advances; returns false past the last tile
  __device__ bool next() {
    if (!last()) {
      ++t;
      return true;
    }
    it += gridDim.x;
    t = 0;
    if (it >= nIt) return false;
    item = pre;
    pre = load(it + gridDim.x);
    return true;
  }
};

// First index of the largest of v[0..BF-1] (strict '>': the first wins ties).
template <int BF>
__device__ __forceinline__ int vtc_argmax(const uint32_t* v) {
  uint32_t best = v[0];
  int bi = 0;
#pragma unroll
  for (int k = 1; k < BF; ++k)
    if (v[k] > best) {
      best = v[k];
      bi = k;
    }
  return bi;
}

template <int BF>
__global__ void __launch_bounds__(kVtcThreads, 1)
    k_vtc(VtcArgs a, const __grid_constant__ CUtensorMap tmNodes, const __grid_constant__ CUtensorMap tmKeys) {
  using S = VtcShape<BF>;
  extern __shared__ uint8_t vtcRaw[];
  VtcSmem<BF>& s = *reinterpret_cast<VtcSmem<BF>*>((reinterpret_cast<uintptr_t>(vtcRaw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nIt = a.singleN > 0 ? (a.singleN + kVtcItemKeys - 1) / kVtcItemKeys : *a.nItems;
  const bool localHist = !a.final && a.bins <= kVtcLocalBins;
  const long long lim = kWaitCycles;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kVtcASlots; ++i) {
      mbar_init(&s.fullA[i], 1);  // the producer's arrival (with a TMA's bytes, or its lanes' copies)
      mbar_init(&s.emptyA[i], 1);
    }
    for (int i = 0; i < S::kBBufs; ++i) {
      mbar_init(&s.fullB[i], 1);
      mbar_init(&s.emptyB[i], 1);
    }
    for (int i = 0; i < S::kAcc; ++i) {
      mbar_init(&s.accFull[i], 1);
      mbar_init(&s.accEmpty[i], 4);  // the four warps of the half that takes the tile
    }
    mbar_init(&s.mmaDone, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (localHist)
    for (int i = threadIdx.x; i < a.bins; i += blockDim.x) s.hist[i] = 0;
  if (warp == kVtcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmemBase)),
                 "r"(kVtcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmemBase;
  if ((tmem & 0xFFFFu) != 0 && threadIdx.x == 0) {  // 512 columns start at column 0
    atomicOr(a.err, kErrTmem);
    s.abort = 1;
  }
  __syncthreads();

  if (warp < kVtcProducers) {
    // ---------------- producers: key tiles and subtree rows (warp p takes tiles p, p + 2, ...) ----
    // Both walk every tile (the tile number gives the A slot, the item number the B buffer);
    // producer 0 also loads every item's subtree, so that one warp owns the B ring (and knows,
    // after an abort, which of its loads may still be in flight).
    if (!s.abort) {
      const int p = warp;
      VtcWalk w;
      int tn = 0, nItem = 0;
      bool armedB[S::kBBufs];  // B buffers with a TMA load this warp has not seen land (for an abort)
      uint32_t armedPar[S::kBBufs];
#pragma unroll
      for (int i = 0; i < S::kBBufs; ++i) armedB[i] = false;
      // gathered keys: the key index of each row this lane copies (row 4 i + lane / 8, chunk
      // lane % 8), -1 past the bucket; the next own tile's are loaded while this one's copies go out
      auto tile_keys = [&](const VtcWalk& v, int (&kk)[kVtcRows / 4]) {
        const int base = v.item.y + v.t * kVtcRows;
        const int cnt = min(kVtcRows, v.item.z - v.t * kVtcRows);
#pragma unroll
        for (int i = 0; i < kVtcRows / 4; ++i) {
          const int rr = 4 * i + (lane >> 3);
          kk[i] = rr < cnt ? __ldg(a.perm + base + rr) : -1;
        }
      };
      // bounded wait by lane 0, the result broadcast
      auto wait_free = [&](unsigned long long* bar, uint32_t par) -> bool {
        int okl = 1;
        if (lane == 0) okl = mbar_wait(bar, par, &s.abort, a.err, lim) ? 1 : 0;
        return __shfl_sync(0xffffffffu, okl, 0) != 0;
      };
      const bool gathered = a.perm != nullptr;
      int keysCur[kVtcRows / 4], keysNext[kVtcRows / 4];
      bool more = w.start(a.items, nIt, a.singleN);
      if (gathered) {  // the first own tile's keys
        VtcWalk v = w;
        bool m = more;
        for (int k = 0; k < p && m; ++k) m = v.next();
        if (m) tile_keys(v, keysNext);
      }
      bool ok = true;
      for (; more && ok; more = w.next(), ++tn) {
        const bool mine = (tn % kVtcProducers) == p;
        if (w.first()) {
          const int buf = nItem % S::kBBufs;
          const uint32_t use = (uint32_t)(nItem / S::kBBufs);
          ++nItem;
          if (p == 0) {
            if (!wait_free(&s.emptyB[buf], (use & 1u) ^ 1u)) break;
            if (lane == 0) {
              // subtree of the item's bucket node r: children from g1 (buffer rows N2 ..), and
              // grandchildren from g2 (buffer rows 0 .. N2 - 1)
              const long long r = a.bucketBase < 0 ? -1 : a.bucketBase + w.item.x;
              const long long g1 = (r + 1) * BF, g2 = (g1 + 1) * BF;
              const int boxes = a.levels == 2 ? S::N2 / kVtcBoxRows : 0;
              mbar_expect_tx(&s.fullB[buf], (uint32_t)((boxes + 1) * kVtcBoxRows * kDescBytes));
              tma_load_2d(s.b[buf] + S::N2 * kDescBytes, &tmNodes, &s.fullB[buf], 0, (int)g1);
              for (int x = 0; x < boxes; ++x)
                tma_load_2d(s.b[buf] + x * kVtcBoxRows * kDescBytes, &tmNodes, &s.fullB[buf], 0,
                            (int)(g2 + x * kVtcBoxRows));
            }
            armedB[buf] = true;
            armedPar[buf] = use & 1u;
          }
        }
        if (!mine) continue;
        if (gathered) {
#pragma unroll
          for (int k = 0; k < kVtcRows / 4; ++k) keysCur[k] = keysNext[k];
          VtcWalk v = w;
          bool m = true;
          for (int k = 0; k < kVtcProducers && m; ++k) m = v.next();
          if (m) tile_keys(v, keysNext);
        }
        const int slot = tn % kVtcASlots;
        const uint32_t phaseA = (uint32_t)(tn / kVtcASlots) & 1u;
        if (!wait_free(&s.emptyA[slot], phaseA ^ 1)) {
          ok = false;
          break;
        }
        if (!gathered) {
          // consecutive keys: one TMA tile (rows past the last key read as zero)
          if (lane == 0) {
            mbar_expect_tx(&s.fullA[slot], (uint32_t)S::kABytes);
            tma_load_2d(s.a[slot], &tmKeys, &s.fullA[slot], 0, w.item.y + w.t * kVtcRows);
          }
        } else {
          // eight lanes per 128-byte row, four rows per instruction; each lane's copies are
          // tracked by the slot's mbarrier, then lane 0 adds the producer's own arrival
          const uint32_t d0 = smem_u32(s.a[slot]);
          const int ch = lane & 7;
#pragma unroll
          for (int i = 0; i < kVtcRows / 4; ++i) {
            const int rr = 4 * i + (lane >> 3);
            const int key = keysCur[i];
            const uint8_t* g = a.keys + (key >= 0 ? (size_t)key * kDescBytes + 16 * ch : (size_t)0);
            vtc_cp16(d0 + (uint32_t)rr * 128u + (uint32_t)((ch ^ (rr & 7)) << 4), g, key >= 0 ? 16u : 0u);
          }
          vtc_cp_arrive(&s.fullA[slot]);
          __syncwarp();
          if (lane == 0) mbar_arrive(&s.fullA[slot]);
        }
      }
      vtc_wait_all();
      // after an abort, the TMA loads still in flight land before the CTA exits
      if (lane == 0)
        for (int i = 0; i < S::kBBufs; ++i)
          if (armedB[i]) {
            long long t0 = clock64();
            while (!mbar_try(&s.fullB[i], armedPar[i]) && clock64() - t0 < kWaitCycles) {
            }
          }
    }
  } else if (warp == kVtcMmaWarp) {
    // ---------------- MMA issuer (lane 0) ----------------
    // A tile is one chain of four dependent MMAs (K = 32 each) into its accumulator stage.  When
    // the next tile is ready as well, the two chains are issued interleaved so that the tensor
    // core overlaps them.
    if (lane == 0 && !s.abort) {
      struct Tile {
        int slot, acc, buf;
        bool last;
      };
      VtcWalk w;
      int slot = 0, acc = 0, nItem = 0, buf = 0;
      uint32_t phaseA = 0, accPhase = 0;
      bool any = false;
      // the tile at v: blocking waits (false: abort), or a non-blocking check (false: not ready)
      auto acquire = [&](const VtcWalk& v, bool block, Tile& t) -> bool {
        int b = buf;
        if (v.first()) {
          b = nItem % S::kBBufs;
          const uint32_t par = (uint32_t)(nItem / S::kBBufs) & 1u;
          if (block ? !mbar_wait(&s.fullB[b], par, &s.abort, a.err, lim) : !mbar_test(&s.fullB[b], par)) return false;
        }
        if (block ? !mbar_wait(&s.fullA[slot], phaseA, &s.abort, a.err, lim) : !mbar_test(&s.fullA[slot], phaseA))
          return false;
        if (block ? !mbar_wait(&s.accEmpty[acc], accPhase ^ 1, &s.abort, a.err, lim)
                  : !mbar_test(&s.accEmpty[acc], accPhase ^ 1))
          return false;
        if (v.first()) {
          buf = b;
          ++nItem;
        }
        t.slot = slot;
        t.acc = acc;
        t.buf = buf;
        t.last = v.last();
        if (++slot == kVtcASlots) {
          slot = 0;
          phaseA ^= 1;
        }
        if (++acc == S::kAcc) {
          acc = 0;
          accPhase ^= 1;
        }
        return true;
      };
      auto mma_k = [&](const Tile& t, int k) {
        const uint32_t aAddr = smem_u32(s.a[t.slot]), bAddr = smem_u32(s.b[t.buf]);
        const uint32_t d2 = tmem + (uint32_t)(t.acc * S::kAccCols), d1 = d2 + S::N2;
        if (a.levels == 2)  // grandchildren and children: one chain over all kRowsB rows
          vtc_mma<S::kRowsB>(d2, sdesc(aAddr + 32u * k), sdesc(bAddr + 32u * k), k > 0 ? 1u : 0u);
        else
          vtc_mma<S::N1>(d1, sdesc(aAddr + 32u * k), sdesc(bAddr + (uint32_t)(S::N2 * kDescBytes) + 32u * k),
                         k > 0 ? 1u : 0u);
      };
      auto commit = [&](const Tile& t) {
        mma_commit(&s.accFull[t.acc]);
        mma_commit(&s.emptyA[t.slot]);
        if (t.last) mma_commit(&s.emptyB[t.buf]);
      };
      bool more = w.start(a.items, nIt, a.singleN);
      while (more) {
        Tile t0, t1;
        if (!acquire(w, true, t0)) break;
        VtcWalk w1 = w;
        const bool more1 = w1.next();
        const bool pair = more1 && acquire(w1, false, t1);
        // the key rows were written by cp.async (generic proxy); the tensor core reads them
        // through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_after();
#pragma unroll
        for (int k = 0; k < kDescBytes / 32; ++k) {
          mma_k(t0, k);
          if (pair) mma_k(t1, k);
        }
        any = true;
        commit(t0);
        if (pair) {
          commit(t1);
          w = w1;
        }
        more = w.next();
      }
      if (any) {  // every MMA issued has completed before TMEM is released
        mma_commit(&s.mmaDone);
        long long t0 = clock64();
        while (!mbar_try(&s.mmaDone, 0) && clock64() - t0 < kWaitCycles) {
        }
      }
    }
  } else {
    // ---------------- epilogue: one key per thread ----------------
    const int q = warp & 3;                  // TMEM lane quadrant this warp may access
    const int half = (warp - kVtcEpiWarp0) >> 2;  // the tiles it takes: every other one
    const int row = q * 32 + lane;
    VtcWalk w;
    int acc = 0, tn = 0;
    uint32_t accPhase = 0;
    for (bool more = w.start(a.items, nIt, a.singleN); more; more = w.next(), ++tn) {
      if ((tn % kVtcEpiHalves) != half) {
        if (++acc == S::kAcc) {
          acc = 0;
          accPhase ^= 1;
        }
        continue;
      }
      // this row's key index, loaded before the wait for the accumulator
      const int pos = w.t * kVtcRows + row;
      const int key = pos < w.item.z ? (a.perm ? __ldg(a.perm + w.item.y + pos) : w.item.y + pos) : -1;
      if (!mbar_wait(&s.accFull[acc], accPhase, &s.abort, a.err, lim)) break;
      tc_fence_after();
      const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * S::kAccCols);
      uint32_t v[S::kAccCols];  // D2 in columns 0 .. N2 - 1, D1 in N2 .. N2 + 15
      if (a.levels == 2) {
#pragma unroll
        for (int c = 0; c < S::kAccCols / 32; ++c) tmem_ld32(tb + (uint32_t)(32 * c), v + 32 * c);
        if constexpr (S::kAccCols % 32 != 0) tmem_ld16(tb + (uint32_t)(S::kAccCols - 16), v + S::kAccCols - 16);
      } else {
        tmem_ld16(tb + S::N2, v + S::N2);
      }
      tmem_wait(v);
      const uint32_t* d1 = v + S::N2;
      const uint32_t* d2 = v;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s.accEmpty[acc]);
      if (++acc == S::kAcc) {
        acc = 0;
        accPhase ^= 1;
      }
      if (key < 0) continue;
      const long long r = a.bucketBase < 0 ? -1 : a.bucketBase + w.item.x;
      const long long g1 = (r + 1) * BF;
      const int c1 = vtc_argmax<BF>(d1);
      long long node = g1 + c1;
      if (a.levels == 2) {
        // the chosen child's BF children: columns BF c1 .. BF c1 + BF - 1 of D2
        uint32_t g[BF];
#pragma unroll
        for (int k = 0; k < BF; ++k) g[k] = d2[k];
#pragma unroll
        for (int c = 1; c < BF; ++c) {
          const bool p = c1 == c;
#pragma unroll
          for (int k = 0; k < BF; ++k) g[k] = p ? d2[BF * c + k] : g[k];
        }
        node = (g1 + 1) * BF + (long long)BF * c1 + vtc_argmax<BF>(g);
      }
      if (a.final) {
        a.out[key] = (int32_t)(a.idMode == V3DM_LEAF_LOCAL ? node - a.leafBase : node);
      } else {
        const int bkt = (int)(node - a.nextBase);
        a.next[key] = bkt;
        // one update per distinct bucket of the warp (keys of a tile often share buckets)
        const unsigned peers = __match_any_sync(__activemask(), bkt);
        if (lane == __ffs(peers) - 1) atomicAdd(localHist ? &s.hist[bkt] : &a.hist[bkt], __popc(peers));
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (localHist)
    for (int i = threadIdx.x; i < a.bins; i += blockDim.x)
      if (s.hist[i]) atomicAdd(&a.hist[i], s.hist[i]);
  if (warp == kVtcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kVtcTmemCols) : "memory");
}

template <int BF>
cudaError_t launch_bf(const VtcArgs& a, const CUtensorMap& m, const CUtensorMap& mk, int grid, cudaStream_t st) {
  const size_t smem = sizeof(VtcSmem<BF>) + 1024;
  static_assert(sizeof(VtcSmem<BF>) + 1024 <= 227 * 1024, "shared memory");
  cudaError_t e = cudaFuncSetAttribute(k_vtc<BF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_vtc<BF><<<grid, kVtcThreads, smem, st>>>(a, m, mk);
  return cudaGetLastError();
}

}  // namespace

bool vtc_supported(int bf) { return bf >= 2 && bf <= 15; }

cudaError_t launch_vtc(const VtcArgs& a, const CUtensorMap& m, const CUtensorMap& mk, int grid, cudaStream_t st) {
  switch (a.bf) {
    case 2: return launch_bf<2>(a, m, mk, grid, st);
    case 3: return launch_bf<3>(a, m, mk, grid, st);
    case 4: return launch_bf<4>(a, m, mk, grid, st);
    case 5: return launch_bf<5>(a, m, mk, grid, st);
    case 6: return launch_bf<6>(a, m, mk, grid, st);
    case 7: return launch_bf<7>(a, m, mk, grid, st);
    case 8: return launch_bf<8>(a, m, mk, grid, st);
    case 9: return launch_bf<9>(a, m, mk, grid, st);
    case 10: return launch_bf<10>(a, m, mk, grid, st);
    case 11: return launch_bf<11>(a, m, mk, grid, st);
    case 12: return launch_bf<12>(a, m, mk, grid, st);
    case 13: return launch_bf<13>(a, m, mk, grid, st);
    case 14: return launch_bf<14>(a, m, mk, grid, st);
    case 15: return launch_bf<15>(a, m, mk, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace v3dm
