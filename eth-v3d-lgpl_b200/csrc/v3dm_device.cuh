// v3dm_device.cuh -- device helpers shared by the SIMT and tcgen05 matching kernels.
#pragma once
#include "v3dm_internal.h"

namespace v3dm {

// Programmatic dependent launch: a kernel launched with launch_pdl may start while the kernel
// before it in the stream is finishing.  pdl_wait() blocks until that kernel has completed and
// its writes are visible (it returns at once for a normal launch); pdl_launch_dependents()
// lets the next kernel's blocks be scheduled.  Every kernel here calls both first thing.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

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

// A candidate (l, r, S): both best keys take it with an atomicMax whose result is unused
// (a fire-and-forget reduction, so the issuing warp does not wait for L2).
__device__ __forceinline__ void record_best(const MatchArgs& a, int l, int r, int32_t S) {
  atomicMax(&a.lBest[l], (unsigned long long)best_key(S, r));
  atomicMax(&a.rBest[r], (unsigned long long)best_key(S, l));
}

// Gate test for one (left, right) element, the reference's expressions evaluated left to
// right with one IEEE rounding per operation:
//   epipolar   (v3d_cudamatching.cu:302-308): num = (q.x*Fp.x + q.y*Fp.y + Fp.z)^2,
//              denom = Fp.x^2 + Fp.y^2 + Ftq.x^2 + Ftq.y^2, reject if num/denom > thr^2;
//   homography (v3d_cudamatching.cu:337-340): reject if |Hp - q|^2 > thr^2.
__device__ __forceinline__ bool gate_rejects(const GateParams& g, int l, int r) {
  float4 p = g.lv[l];
  float4 q = g.rv[r];
  if (g.type == 1) {
    float num = __fadd_rn(__fadd_rn(__fmul_rn(q.x, p.x), __fmul_rn(q.y, p.y)), p.z);
    num = __fmul_rn(num, num);
    float denom = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.x, p.x), __fmul_rn(p.y, p.y)), __fmul_rn(q.z, q.z)),
                            __fmul_rn(q.w, q.w));
    return __fdiv_rn(num, denom) > g.sqrThr;
  }
  float dx = __fsub_rn(p.x, q.x), dy = __fsub_rn(p.y, q.y);
  return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) > g.sqrThr;
}

__device__ __forceinline__ bool gated_out(const MatchArgs& a, int l, int r) {
  for (int g = 0; g < a.nGates; ++g)
    if (gate_rejects(a.gates[g], l, r)) return true;
  return false;
}

}  // namespace v3dm
