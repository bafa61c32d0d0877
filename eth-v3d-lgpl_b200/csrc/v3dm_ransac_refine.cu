// v3dm_ransac_refine.cu -- the RANSAC loop's selection with mode.iterativeRefinement
// (V3D/Apps/SfM/reconstruction_common.cpp:255-314): each accepted candidate's pose is refined by
// refineRelativePose (V3D/Geometry/v3d_poseutilities.cpp:1063-1101) on the inliers of the
// candidate's F, the refined F is scored over all correspondences, and the loop keeps
// min(cost, refined cost), the refined model and the refined inlier count for its budget.
//
// The refinement is a Levenberg-Marquardt loop whose accept/reject and stopping decisions can
// turn on the last bits of its sums, so this file reproduces the arithmetic of the reference's
// CPU code (ess::refine_pose restates it and matches it inside the loop on every tested pair):
//   - it is built without contraction into fused multiply-adds (the reference builds for plain
//     x86-64), see the Makefile;
//   - the sums over the inliers run in index order: the lanes of the warp compute the
//     correspondences' residuals and Jacobian rows 32 at a time, stage them in shared memory,
//     and lane q then accumulates quantity q (one of the 21 entries of J^T J, 6 of J^T e, and
//     |e|^2) over them in order -- every sum has the sequential order of the reference's loops;
//   - the rotation update's sin and cos are correctly rounded (ess::pose_update, device path).
#include <cuda_runtime.h>

#include "v3dm_essential.cuh"
#include "v3dm_internal.h"
#include "v3dm_ransac.cuh"

namespace v3dm {

namespace {

// F = (invK2^T E) invK1, the reference's product order (reconstruction_common.cpp:271).
__device__ void rs_fund(const double* invK1, const double* invK2t, const double* E, double* F) {
  double tmp[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += invK2t[3 * i + k] * E[3 * k + j];
      tmp[3 * i + j] = v;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += tmp[3 * i + k] * invK1[3 * k + j];
      F[3 * i + j] = v;
    }
}

constexpr int kRsQuant = 28;  // 21 entries of J^T J (upper triangle), 6 of J^T e, |e|^2

// One pass over the inliers of F0 (Sampson distance below thr2: the set the reference hands to
// refineRelativePose, in index order): RelativePoseMinimizer's weights at pose (Rw, Tw) (from the
// pixel positions and thr, ess::pose_weighted_residual), the weighted residuals at (R, T) and,
// with derivs, the normal equations (ess::pose_normal_equations).  Every lane gets the sums.
__device__ double rs_lm_pass(const float4* __restrict__ px, const double4* __restrict__ nm, int n, const double* F0,
                             double thr2, const double* invK1, const double* invK2t, double thr, const double* Rw,
                             const double* Tw, const double* R, const double* T, bool derivs, double* JtJ,
                             double* Jte, double (*sv)[8]) {
  const int lane = threadIdx.x & 31;
  double Ew[9], Fw[9], E[9], inner[9][6], a[3], b[2];
  ess::pose_essential(Rw, Tw, Ew);
  rs_fund(invK1, invK2t, Ew, Fw);
  ess::pose_essential(R, T, E);
  if (derivs) ess::pose_inner(E, R, inner);
  // the quantity this lane owns: JtJ[qa][qb] (qa <= qb), Jte[qa], or |e|^2
  int qa = 0, qb = 0;
  if (lane < 21) {
    int t = lane;
    while (t >= 6 - qa) {
      t -= 6 - qa;
      ++qa;
    }
    qb = qa + t;
  } else if (lane < 27) {
    qa = lane - 21;
    qb = 6;  // e
  } else {
    qa = 6;
    qb = 6;
  }
  const bool owns = lane < kRsQuant && (derivs || lane == 27);
  double acc = 0.0;
  for (int k0 = 0; k0 < n; k0 += 32) {
    const int k = k0 + lane;
    double J[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, e = 0.0;
    bool in = false;
    if (k < n) {
      const float4 c = px[k];
      in = ess::sampson(F0, c.x, c.y, c.z, c.w) < thr2;
      if (in) {
        const double4 q = nm[k];
        const double ew = ess::pose_residual(Fw, c.x, c.y, c.z, c.w, a, b);
        const double w = (fabs(ew) < thr) ? 1.0 : sqrt(thr / fabs(ew));
        e = w * (0.0 - ess::pose_residual(E, q.x, q.y, q.z, q.w, a, b));
        if (derivs) ess::pose_jacobian_row(E, inner, q.x, q.y, q.z, q.w, J);
      }
    }
    const unsigned inMask = __ballot_sync(0xffffffffu, in);
    __syncwarp();
    for (int j = 0; j < 6; ++j) sv[lane][j] = J[j];
    sv[lane][6] = e;
    __syncwarp();
    if (owns) {
      for (unsigned m = inMask; m; m &= m - 1) {  // the inliers of this chunk, in index order
        const int l = __ffs(m) - 1;
        acc += sv[l][qa] * sv[l][qb];
      }
    }
  }
  if (derivs) {
    for (int t = 0; t < 21; ++t) {
      const double v = __shfl_sync(0xffffffffu, acc, t);
      int i = 0, r = t;
      while (r >= 6 - i) {
        r -= 6 - i;
        ++i;
      }
      JtJ[6 * i + i + r] = v;
      JtJ[6 * (i + r) + i] = v;
    }
    for (int t = 0; t < 6; ++t) Jte[t] = __shfl_sync(0xffffffffu, acc, 21 + t);
  }
  return __shfl_sync(0xffffffffu, acc, 27);
}

// refineRelativePose on the inliers of F0: ess::refine_pose's Levenberg-Marquardt loop
// (SimpleLevenbergOptimizer's damping schedule and stopping rules), warp-uniform.
__device__ void rs_refine_warp(const float4* __restrict__ px, const double4* __restrict__ nm, int n, const double* F0,
                               double thr2, const double* invK1, const double* invK2t, double thr, double* R,
                               double* T, double (*sv)[8]) {
  double lambda = 1e-3, JtJ[36], Jte[6], N[36], delta[6], Rs[9], Ts[3];
  bool computeDerivatives = true;
  for (int it = 0; it < 50; ++it) {
    const double err =
        rs_lm_pass(px, nm, n, F0, thr2, invK1, invK2t, thr, R, T, R, T, computeDerivatives, JtJ, Jte, sv);
    double gmax = 0.0;
    for (int k = 0; k < 6; ++k) gmax = fmax(gmax, fabs(Jte[k]));
    if (gmax < 1e-8) return;
    if (it == 0) {
      double maxEl = -1e30;
      for (int k = 0; k < 6; ++k) maxEl = fmax(maxEl, JtJ[7 * k]);
      lambda = 1e-3 * maxEl;
    }
    for (int k = 0; k < 36; ++k) N[k] = JtJ[k];
    for (int k = 0; k < 6; ++k) N[7 * k] += lambda;
    if (!ess::cholesky_solve6(N, Jte, delta)) return;
    double dl = 0.0;
    for (int k = 0; k < 6; ++k) dl += delta[k] * delta[k];
    dl = sqrt(dl);
    if (it >= 10 && dl < 1e-8 * (4.0 + 1e-8)) return;
    for (int k = 0; k < 9; ++k) Rs[k] = R[k];
    for (int k = 0; k < 3; ++k) Ts[k] = T[k];
    ess::pose_update(Rs, Ts, delta, R, T);
    const double errNew =
        rs_lm_pass(px, nm, n, F0, thr2, invK1, invK2t, thr, Rs, Ts, R, T, false, nullptr, nullptr, sv);
    double rho = err - errNew;
    double d1 = 0.0, d2 = 0.0;
    for (int k = 0; k < 6; ++k) {
      d1 += delta[k] * delta[k];
      d2 += delta[k] * Jte[k];
    }
    rho = rho / (lambda * d1 + d2);
    if (rho > 0) {
      lambda = fmax(1e-10, lambda * 0.1);
      computeDerivatives = true;
    } else {
      for (int k = 0; k < 9; ++k) R[k] = Rs[k];
      for (int k = 0; k < 3; ++k) T[k] = Ts[k];
      lambda *= 10.0;
      computeDerivatives = false;
    }
  }
}

// sum_i min(d_i, thr2) over all correspondences in index order (the loop's sum, as k_rs_score
// forms it) and the count of d_i < thr2; every lane gets both.
__device__ void rs_cost_in_order(const float4* __restrict__ px, int n, const double* F, double thr2, double* cost,
                                 int* nIn) {
  const int lane = threadIdx.x & 31;
  double sum = 0.0;
  int cnt = 0;
  for (int k0 = 0; k0 < n; k0 += 32) {
    double t = 0.0;
    bool in = false;
    if (k0 + lane < n) {
      const float4 c = px[k0 + lane];
      t = ess::sampson_truncated(F, (double)c.x, (double)c.y, (double)c.z, (double)c.w, thr2, in);
    }
    cnt += __popc(__ballot_sync(0xffffffffu, in));
    const int m = min(32, n - k0);
    for (int l = 0; l < m; ++l) sum = ess::dadd(sum, __shfl_sync(0xffffffffu, t, l));
  }
  *cost = sum;
  *nIn = cnt;
}

// One warp per pair: the round's costs and pose flags staged in shared memory, then every lane
// walks the loop over the round's samples in order (the same decisions on every lane), and the
// warp refines each accepted pose.
__global__ void __launch_bounds__(32)
k_rs_select_refine(const int32_t* __restrict__ offsets, int nDraw, int s0, int len, const int8_t* __restrict__ counts,
                   const uint8_t* __restrict__ slotOk, const double* __restrict__ cost,
                   const double* __restrict__ slots, RsState* __restrict__ st, double* __restrict__ bestEF,
                   const float4* __restrict__ corrs, const double4* __restrict__ norm,
                   const int32_t* __restrict__ samples, const double* __restrict__ invK, double thr, double thr2,
                   double* __restrict__ bestRT) {
  const int p = blockIdx.x;
  const int lane = threadIdx.x;
  __shared__ double sCost[kRsRound * kRsMaxSol];
  __shared__ uint8_t sOk[kRsRound * kRsMaxSol];
  __shared__ int8_t sCnt[kRsRound];
  __shared__ double sv[32][8];
  RsState s = st[p];
  if (s.done) return;  // uniform over the warp
  const long long base = (long long)p * kRsRound;
  for (int j = lane; j < len; j += 32) sCnt[j] = counts[base + j];
  __syncwarp();
  for (int idx = lane; idx < len * kRsMaxSol; idx += 32) {
    const int j = idx / kRsMaxSol, r = idx - j * kRsMaxSol;
    if (r < sCnt[j]) {
      sCost[idx] = cost[base * kRsMaxSol + idx];
      sOk[idx] = slotOk[base * kRsMaxSol + idx];
    }
  }
  __syncwarp();
  const int b = offsets[p], n = offsets[p + 1] - b;
  double invK1[9], invK2t[9];
  for (int k = 0; k < 9; ++k) invK1[k] = invK[(size_t)p * 18 + k];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) invK2t[3 * i + j] = invK[(size_t)p * 18 + 9 + 3 * j + i];
  for (int j = 0; j < len; ++j) {
    if (s.drawn > s.budget) break;
    ++s.drawn;
    const int ns = sCnt[j];
    for (int r = 0; r < ns; ++r) {
      const int idx = j * kRsMaxSol + r;
      if (!(sCost[idx] < s.minError)) continue;
      if (!sOk[idx]) continue;
      double EF[kRsSlotDoubles];
      for (int k = 0; k < kRsSlotDoubles; ++k) EF[k] = slots[(base * kRsMaxSol + idx) * kRsSlotDoubles + k];
      const int32_t* smp = samples + ((long long)p * nDraw + s0 + j) * 5;
      double x1[5], y1[5], x2[5], y2[5];
      for (int k = 0; k < 5; ++k) {
        const double4 v = norm[b + smp[k]];
        x1[k] = v.x;
        y1[k] = v.y;
        x2[k] = v.z;
        y2[k] = v.w;
      }
      double R[9], T[3];
      if (!ess::essential_pose(EF, 5, x1, y1, x2, y2, R, T)) continue;  // relativePoseFromEssential
      rs_refine_warp(corrs + b, norm + b, n, EF + 9, thr2, invK1, invK2t, thr, R, T, sv);
      double Er[9], Fr[9], costR;
      int nInR;
      ess::pose_essential(R, T, Er);
      rs_fund(invK1, invK2t, Er, Fr);
      rs_cost_in_order(corrs + b, n, Fr, thr2, &costR, &nInR);
      s.minError = fmin(sCost[idx], costR);
      s.chosen = s0 + j;
      const float frac = (float)(nInR - 5) / (float)(n - 5);
      s.budget = min(s.budget, rs_budget(1.0 - (double)frac));
      double* ef = bestEF + (size_t)p * kRsSlotDoubles;
      double* rt = bestRT + (size_t)p * 12;
      if (lane < 9) {
        ef[lane] = Er[lane];
        ef[9 + lane] = Fr[lane];
        rt[lane] = R[lane];
      } else if (lane < 12) {
        rt[lane] = T[lane - 9];
      }
    }
  }
  if (lane == 0) {
    if (s.drawn > s.budget || s0 + len >= nDraw) s.done = 1;  // the next sample would end the loop
    st[p] = s;
  }
}

}  // namespace

cudaError_t launch_rs_select_refine(const int32_t* offsets, int nPairs, int nDraw, int s0, int len, const int8_t* counts,
                                    const uint8_t* slotOk, const double* cost, const double* slots, RsState* st,
                                    double* bestEF, const float4* corrs, const double4* norm, const int32_t* samples,
                                    const double* invK, double thr, double thr2, double* bestRT, cudaStream_t stream) {
  if (nPairs <= 0) return cudaSuccess;
  k_rs_select_refine<<<nPairs, 32, 0, stream>>>(offsets, nDraw, s0, len, counts, slotOk, cost, slots, st, bestEF,
                                                corrs, norm, samples, invK, thr, thr2, bestRT);
  return cudaGetLastError();
}

}  // namespace v3dm
