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

// Per-left terms of a gate from the left position p and the matrix m (row-major floats, the
// reference's double-to-float F1..F3 / H1..H3, .cu:592-595, :663-666):
//   epipolar   (.cu:293-296) Fp = F p, i.e. (Fp.x, Fp.y, Fp.z, 0);
//   homography (.cu:327-333) Hp = H p, then (Hp.x / Hp.z, Hp.y / Hp.z, Hp.z, 0).
__device__ __forceinline__ float4 gate_left_terms(int type, const float* m, float2 p) {
  float x = __fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[1], p.y)), m[2]);
  float y = __fadd_rn(__fadd_rn(__fmul_rn(m[3], p.x), __fmul_rn(m[4], p.y)), m[5]);
  const float z = __fadd_rn(__fadd_rn(__fmul_rn(m[6], p.x), __fmul_rn(m[7], p.y)), m[8]);
  if (type == 2) {
    x = __fdiv_rn(x, z);
    y = __fdiv_rn(y, z);
  }
  return make_float4(x, y, z, 0.f);
}

// Per-right terms from the right position q: epipolar (q.x, q.y, Ftq.x, Ftq.y) with Ftq = F^T q
// (.cu:302-304); homography (q.x, q.y, 0, 0).
__device__ __forceinline__ float4 gate_right_terms(int type, const float* m, float2 q) {
  if (type == 1) {
    const float fx = __fadd_rn(__fadd_rn(__fmul_rn(m[0], q.x), __fmul_rn(m[3], q.y)), m[6]);
    const float fy = __fadd_rn(__fadd_rn(__fmul_rn(m[1], q.x), __fmul_rn(m[4], q.y)), m[7]);
    return make_float4(q.x, q.y, fx, fy);
  }
  return make_float4(q.x, q.y, 0.f, 0.f);
}

// Gate test for one (left, right) element from its terms, the reference's expressions
// evaluated left to right with one IEEE rounding per operation:
//   epipolar   (v3d_cudamatching.cu:302-308): num = (q.x*Fp.x + q.y*Fp.y + Fp.z)^2,
//              denom = Fp.x^2 + Fp.y^2 + Ftq.x^2 + Ftq.y^2, reject if num/denom > thr^2;
//   homography (v3d_cudamatching.cu:337-340): reject if |Hp - q|^2 > thr^2.
__device__ __forceinline__ bool gate_rejects_terms(int type, float sqrThr, float4 p, float4 q) {
  if (type == 1) {
    float num = __fadd_rn(__fadd_rn(__fmul_rn(q.x, p.x), __fmul_rn(q.y, p.y)), p.z);
    num = __fmul_rn(num, num);
    float denom = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.x, p.x), __fmul_rn(p.y, p.y)), __fmul_rn(q.z, q.z)),
                            __fmul_rn(q.w, q.w));
    return __fdiv_rn(num, denom) > sqrThr;
  }
  float dx = __fsub_rn(p.x, q.x), dy = __fsub_rn(p.y, q.y);
  return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) > sqrThr;
}

__device__ __forceinline__ bool gate_rejects(const GateParams& g, int l, int r) {
  return gate_rejects_terms(g.type, g.sqrThr, g.lv[l], g.rv[r]);
}

// Batched guided matching: the pair of a side-pass state and its index on the A side.
// Pass A states are (pair, left) in batch order (stateA0 ascending); pass B states name their
// pair and right directly.
__device__ __forceinline__ void bgate_resolve(const BatchGateArgs& g, int aIsLeft, long long state, int* pair,
                                              int* aIdx) {
  if (aIsLeft) {
    int lo = 0, hi = g.nPairs - 1;  // last batch-order pair whose first state is <= state
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (g.stateA0[mid] <= state) lo = mid;
      else hi = mid - 1;
    }
    *pair = g.origOf[lo];
    *aIdx = (int)(state - g.stateA0[lo]);
  } else {
    *pair = g.chosenPair[state];
    *aIdx = g.chosenRight[state];
  }
}

// Gate of pair 'pair' (caller's order) for left l and right r of its images.
__device__ __forceinline__ bool bgate_rejects(const BatchGateArgs& g, int pair, int l, int r) {
  const float* m = g.gm + (size_t)pair * kBGateFloats;
  const int2 lr = g.pairLR[pair];
  const float2 p = g.pos[g.posOff[lr.x] + l];
  const float2 q = g.pos[g.posOff[lr.y] + r];
  return gate_rejects_terms(g.type, m[9], gate_left_terms(g.type, m, p), gate_right_terms(g.type, m, q));
}

__device__ __forceinline__ bool gated_out(const MatchArgs& a, int l, int r) {
  for (int g = 0; g < a.nGates; ++g)
    if (gate_rejects(a.gates[g], l, r)) return true;
  return false;
}

}  // namespace v3dm
