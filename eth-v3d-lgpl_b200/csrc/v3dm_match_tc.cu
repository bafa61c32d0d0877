// v3dm_match_tc.cu -- tcgen05 matching kernel for sm_100a.
//
// Replaces cublasSgemm + the four maxima kernels of the reference
// (v3d_cudamatching.cu:529-545) with one persistent kernel whose score tiles never leave
// the SM:
//   warp 0      TMA producer: left tile A (128 descriptors x 128 bytes) once per work unit,
//               right tiles B (256 x 128 bytes) through a 4-stage ring, 128-byte swizzle;
//   warp 1      allocates 512 TMEM columns and issues tcgen05.mma.kind::i8 (u8 x u8 -> s32,
//               M=128, N=256, four K=32 steps per tile) into two 256-column accumulators;
//   warps 2-9   epilogue: tcgen05.ld 32x32b.x32 chunks, per-lane maximum of 32 scores, and
//               only when a score reaches the candidate threshold T (rare) the exact
//               per-element path: guided gates, atomicMax of both best keys, candidate
//               list append (shared-memory counter, per-CTA list segment).
// A work unit is (left block of 128 rows, range of right tiles); units are dealt to CTAs
// round-robin, every role walks the same sequence, and mbarriers order the hand-offs.
// Every mbarrier wait is bounded: on timeout the CTA raises kErrWaitTimeout, drains its
// own TMA loads and MMAs, frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <new>

#include "v3dm_device.cuh"

namespace v3dm {

namespace {

constexpr int BM = 128;          // lefts per tile (TMEM lanes)
constexpr int BN = 256;          // rights per tile (TMEM columns per accumulator)
constexpr int kStages = 4;       // right-tile ring
constexpr int kEpiWarps = 8;     // two per TMEM lane quadrant, each owning 128 columns
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr int kABytes = BM * kDescBytes;  // 16 KB
constexpr int kBBytes = BN * kDescBytes;  // 32 KB
constexpr int kTmemCols = 512;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz

struct Smem {
  uint8_t a[2][kABytes];
  uint8_t b[kStages][kBBytes];
  unsigned long long fullB[kStages], emptyB[kStages];
  unsigned long long fullA[2], emptyA[2];
  unsigned long long accFull[2], accEmpty[2];
  unsigned long long mmaDone;
  uint32_t tmemBase;
  int candCount;
  int abort;
};
constexpr size_t kSmemBytes = sizeof(Smem) + 1024;  // + alignment slack

struct TcShape {
  int nLB, nRT, nSplit, nUnits;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned long long* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity.  Returns false on timeout or when
// another role of the CTA has aborted.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, uint32_t parity, Smem& s, int* err) {
  if (mbar_try(b, parity)) return true;
  long long t0 = clock64();
  while (true) {
    if (mbar_try(b, parity)) return true;
    if (*reinterpret_cast<volatile int*>(&s.abort)) return false;
    if (clock64() - t0 > kWaitCycles) {
      atomicOr(err, kErrWaitTimeout);
      *reinterpret_cast<volatile int*>(&s.abort) = 1;
      return false;
    }
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, unsigned long long* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand stored as 128-byte rows with the
// 128-byte swizzle: 8-row core groups 1024 bytes apart (SBO), version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// Instruction descriptor: kind::i8, D = s32, A = B = unsigned 8-bit, both K-major,
// N = 256, M = 128.
constexpr uint32_t kIdesc = (2u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 consecutive 32-bit columns; thread i receives lane (base + i).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) asm volatile("" : "+r"(v[i]));  // uses stay after the wait
}

// Maximum of three non-negative int32 scores through the three-input f32 max: a
// non-negative int32 below 2^23 read as f32 is a subnormal whose order is the integer
// order, and max.f32 without .ftz keeps subnormals.
__device__ __forceinline__ uint32_t max3_bits(uint32_t a, uint32_t b, uint32_t c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(__uint_as_float(a)), "f"(__uint_as_float(b)), "f"(__uint_as_float(c)));
  return __float_as_uint(r);
}

__device__ __forceinline__ void unit_coords(const TcShape& sh, int u, int& lb, int& t0, int& t1) {
  lb = u / sh.nSplit;
  int sp = u - lb * sh.nSplit;
  t0 = (int)((long long)sp * sh.nRT / sh.nSplit);
  t1 = (int)((long long)(sp + 1) * sh.nRT / sh.nSplit);
}

__device__ __noinline__ void candidate(const MatchArgs& a, Smem& s, int l, int r, int32_t S) {
  if (a.nGates && gated_out(a, l, r)) return;
  record_best(a, l, r, S);
  int idx = atomicAdd(&s.candCount, 1);
  if (idx < a.segCap) a.cand[(long long)blockIdx.x * a.segCap + idx] = cand_pack(l, r, S);
}

__global__ void __launch_bounds__(kThreads, 1)
k_match_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TcShape sh,
           MatchArgs a) {
  extern __shared__ uint8_t smemRaw[];
  Smem& s = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&s.fullB[i], 1);
      mbar_init(&s.emptyB[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.fullA[i], 1);
      mbar_init(&s.emptyA[i], 1);
      mbar_init(&s.accFull[i], 1);
      mbar_init(&s.accEmpty[i], kEpiWarps);
    }
    mbar_init(&s.mmaDone, 1);
    s.candCount = 0;
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
    // ---------------- TMA producer ----------------
    if (lane == 0 && !s.abort) {
      int stage = 0;
      uint32_t phase = 0, aPhase = 0;
      int aBuf = 0;
      uint32_t armedPhase[kStages];
      bool armed[kStages];
      for (int i = 0; i < kStages; ++i) armed[i] = false;
      bool ok = true;
      for (int u = blockIdx.x; u < sh.nUnits && ok; u += gridDim.x) {
        int lb, t0, t1;
        unit_coords(sh, u, lb, t0, t1);
        if (!(ok = mbar_wait(&s.emptyA[aBuf], aPhase ^ 1, s, a.err))) break;
        mbar_expect_tx(&s.fullA[aBuf], kABytes);
        tma_load_2d(s.a[aBuf], &tmA, &s.fullA[aBuf], 0, lb * BM);
        for (int t = t0; t < t1; ++t) {
          if (!(ok = mbar_wait(&s.emptyB[stage], phase ^ 1, s, a.err))) break;
          mbar_expect_tx(&s.fullB[stage], kBBytes);
          tma_load_2d(s.b[stage], &tmB, &s.fullB[stage], 0, t * BN);
          armed[stage] = true;
          armedPhase[stage] = phase;
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (++aBuf == 2) {
          aBuf = 0;
          aPhase ^= 1;
        }
      }
      // Drain: every load this thread issued has landed before the CTA may exit.
      for (int i = 0; i < kStages; ++i)
        if (armed[i]) {
          long long t0c = clock64();
          while (!mbar_try(&s.fullB[i], armedPhase[i]) && clock64() - t0c < kWaitCycles) {
          }
        }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0 && !s.abort) {
      int stage = 0, acc = 0, aBuf = 0;
      uint32_t phase = 0, accPhase = 0, aPhase = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < sh.nUnits && ok; u += gridDim.x) {
        int lb, t0, t1;
        unit_coords(sh, u, lb, t0, t1);
        if (!(ok = mbar_wait(&s.fullA[aBuf], aPhase, s, a.err))) break;
        const uint32_t aAddr = smem_u32(s.a[aBuf]);
        for (int t = t0; t < t1; ++t) {
          if (!(ok = mbar_wait(&s.accEmpty[acc], accPhase ^ 1, s, a.err))) break;
          if (!(ok = mbar_wait(&s.fullB[stage], phase, s, a.err))) break;
          tc_fence_after();
          const uint32_t bAddr = smem_u32(s.b[stage]);
          const uint32_t d = tmem + (uint32_t)(acc * BN);
#pragma unroll
          for (int k = 0; k < kDescBytes / 32; ++k)
            mma_i8(d, sdesc(aAddr + 32u * k), sdesc(bAddr + 32u * k), k > 0 ? 1u : 0u);
          mma_commit(&s.emptyB[stage]);
          mma_commit(&s.accFull[acc]);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1;
          }
          if (++acc == 2) {
            acc = 0;
            accPhase ^= 1;
          }
        }
        mma_commit(&s.emptyA[aBuf]);
        if (++aBuf == 2) {
          aBuf = 0;
          aPhase ^= 1;
        }
      }
      // Every MMA this thread issued has completed before TMEM is released.
      mma_commit(&s.mmaDone);
      long long t0c = clock64();
      while (!mbar_try(&s.mmaDone, 0) && clock64() - t0c < kWaitCycles) {
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int q = warp & 3;                // TMEM lane quadrant this warp may access
    const int half = (warp - 2) >> 2;      // 0: columns 0..127, 1: columns 128..255
    int acc = 0;
    uint32_t accPhase = 0;
    bool ok = !s.abort;
    for (int u = blockIdx.x; u < sh.nUnits && ok; u += gridDim.x) {
      int lb, t0, t1;
      unit_coords(sh, u, lb, t0, t1);
      const int l = lb * BM + q * 32 + lane;
      const int32_t Tl = l < a.nL ? a.T : 0x7fffffff;
      for (int t = t0; t < t1; ++t) {
        ok = mbar_wait(&s.accFull[acc], accPhase, s, a.err);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        tc_fence_after();
        const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + half * 128);
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          uint32_t v[32];
          tmem_ld32(tbase + (uint32_t)(c * 32), v);
          uint32_t m0 = max3_bits(v[0], v[1], v[2]), m1 = max3_bits(v[3], v[4], v[5]);
          uint32_t m2 = max3_bits(v[6], v[7], v[8]), m3 = max3_bits(v[9], v[10], v[11]);
          uint32_t m4 = max3_bits(v[12], v[13], v[14]), m5 = max3_bits(v[15], v[16], v[17]);
          uint32_t m6 = max3_bits(v[18], v[19], v[20]), m7 = max3_bits(v[21], v[22], v[23]);
          uint32_t m8 = max3_bits(v[24], v[25], v[26]), m9 = max3_bits(v[27], v[28], v[29]);
          uint32_t n0 = max3_bits(m0, m1, m2), n1 = max3_bits(m3, m4, m5), n2 = max3_bits(m6, m7, m8);
          uint32_t n3 = max3_bits(m9, v[30], v[31]);
          uint32_t mx = max3_bits(n0, n1, max3_bits(n2, n3, 0u));
          if (__any_sync(0xffffffffu, (int32_t)mx >= Tl)) {
            const int col0 = t * BN + half * 128 + c * 32;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const bool p = (int32_t)v[j] >= Tl && col0 + j < a.nR;
              if (__any_sync(0xffffffffu, p)) {
                if (p) candidate(a, s, l, col0 + j, (int32_t)v[j]);
              }
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.accEmpty[acc]);
        if (++acc == 2) {
          acc = 0;
          accPhase ^= 1;
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) a.segCount[blockIdx.x] = s.candCount;
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

}  // namespace

struct TcPlan {
  int device = 0;
  int numSMs = 148;
  CUtensorMap mapA, mapB;
  int nL = 0, nR = 0;
  bool attrSet = false;
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

int tc_segments(TcPlan* p) { return p->numSMs; }

cudaError_t tc_plan_bind(TcPlan* p, const uint8_t* dL, int nL, const uint8_t* dR, int nR) {
  if (nL <= 0 || nR <= 0) return cudaSuccess;
  if (!encode_rows(&p->mapA, dL, nL, BM) || !encode_rows(&p->mapB, dR, nR, BN)) return cudaErrorInvalidValue;
  p->nL = nL;
  p->nR = nR;
  return cudaSuccess;
}

cudaError_t launch_match_tc(TcPlan* p, const MatchArgs& a, cudaStream_t st, int* launches) {
  *launches = 0;
  if (a.nL <= 0 || a.nR <= 0) return cudaSuccess;
  if (a.nL != p->nL || a.nR != p->nR) return cudaErrorInvalidValue;
  if (!p->attrSet) {
    cudaError_t e = cudaFuncSetAttribute(k_match_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    if (e != cudaSuccess) return e;
    p->attrSet = true;
  }
  TcShape sh;
  sh.nLB = (a.nL + BM - 1) / BM;
  sh.nRT = (a.nR + BN - 1) / BN;
  // Split each left block's right range so that units fill the SMs evenly: minimise the
  // makespan in tiles, counting half a tile of start-up per unit.
  double bestCost = 1e300;
  int bestSplit = 1;
  for (int sp = 1; sp <= sh.nRT; ++sp) {
    long long units = (long long)sh.nLB * sp;
    long long waves = (units + p->numSMs - 1) / p->numSMs;
    double cost = (double)waves * ((double)((sh.nRT + sp - 1) / sp) + 0.5);
    if (cost < bestCost - 1e-9) {
      bestCost = cost;
      bestSplit = sp;
    }
  }
  sh.nSplit = bestSplit;
  sh.nUnits = sh.nLB * sh.nSplit;
  int grid = std::min(p->numSMs, sh.nUnits);
  if (grid > a.nSeg) return cudaErrorInvalidValue;
  k_match_tc<<<grid, kThreads, kSmemBytes, st>>>(p->mapA, p->mapB, sh, a);
  *launches = 1;
  return cudaGetLastError();
}

}  // namespace v3dm
