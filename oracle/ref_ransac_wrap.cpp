// C entry points over the reference's relative-orientation code: its five-point solver
// (computeEssentialsFromFiveCorrs, V3D/Geometry/v3d_poseutilities.cpp:1016-1060), its pose
// recovery (relativePoseFromEssential, :1264-1294) and the RANSAC loop of
// computeRobustOrientationMLE (V3D/Apps/SfM/reconstruction_common.cpp:139-340).  TEST
// INFRASTRUCTURE ONLY: the parity pin and the timed CPU baseline of the RANSAC workload.
//
// reconstruction_common.cpp itself does not build from a few files (its header needs the apps'
// SQLite database classes), so ref_ransac_mode restates its loop -- with or without
// mode.iterativeRefinement, whose refinement is the reference's own refineRelativePose -- on the
// reference's own solver, pose recovery, matrix inverse and products, with the samples given rather
// than drawn; ref_ransac is the default mode (no refinement); ref_shuffle_samples draws the samples
// the way that loop does (srand(seed), std::random_shuffle, consecutive 5-tuples).
// ref_ransac_swap runs the same loop with some of the reference's components replaced by the
// library's restatements (v3dm_essential.cuh, with the device's sin/cos): the five-point solver,
// the pose recovery, the refinement.  With all three it is the GPU's algorithm on the CPU; swapping
// one at a time attributes a difference between the GPU and the reference to one component.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#define V3DM_HOST_SINCOS_DD 1  // the restated refinement with the device's sin/cos
#include "v3dm_essential.cuh"

#include "Geometry/v3d_poseutilities.h"
#include "Math/v3d_linear.h"

using namespace V3D;

namespace {

// sampsonEpipolarError (reconstruction_common.h:589-607) for (p, q) given as floats.
double sampson(Matrix3x3d const& F, float px, float py, float qx, float qy) {
  Matrix3x3d const Ft = F.transposed();
  Vector2f p, q;
  p[0] = px;
  p[1] = py;
  q[0] = qx;
  q[1] = qy;
  Vector3d Fp, Ftq;
  multiply_A_v_affine(F, p, Fp);
  multiply_A_v_affine(Ft, q, Ftq);
  double const tmp = q[0] * Fp[0] + q[1] * Fp[1] + Fp[2];
  double const num = tmp * tmp;
  double const denom = Fp[0] * Fp[0] + Fp[1] * Fp[1] + Ftq[0] * Ftq[0] + Ftq[1] * Ftq[1];
  return num / denom;
}

// ransacNSamples (reconstruction_common.h:627-635).
int budget(int nNeeded, double outlierRatio, double wanted) {
  double const maxN = 1e8;
  if (outlierRatio >= 1.0) return int(maxN);
  double N = log(1.0 - wanted) / log(1.0 - pow((1.0 - outlierRatio), nNeeded));
  N = std::max(0.0, std::min(maxN, N));
  return (int)N;
}

Matrix3x3d mat(const double* a) {
  Matrix3x3d m;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m[r][c] = a[3 * r + c];
  return m;
}

void put(Matrix3x3d const& m, double* a) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a[3 * r + c] = m[r][c];
}

}  // namespace

extern "C" {

int ref_five_point(const double* x1, const double* y1, const double* x2, const double* y2, double* E, int* n) {
  std::vector<Matrix3x3d> Es;
  computeEssentialsFromFiveCorrs(x1, y1, x2, y2, Es);
  *n = (int)Es.size();
  for (size_t k = 0; k < Es.size() && k < 10; ++k) put(Es[k], E + 9 * k);
  return 0;
}

// 1 and (R, T) when the five correspondences agree on one pose, else 0.
int ref_pose(const double* E, const double* x1, const double* y1, const double* x2, const double* y2, double* R,
             double* T) {
  Matrix3x3d Rm;
  Vector3d t;
  const bool ok = relativePoseFromEssential(mat(E), 5, x1, y1, x2, y2, Rm, t);
  put(Rm, R);
  for (int k = 0; k < 3; ++k) T[k] = t[k];
  return ok ? 1 : 0;
}

// The samples the loop draws (reconstruction_common.cpp:110-114, 173-205): at most nSamples + 1.
int ref_shuffle_samples(int N, int nSamples, unsigned seed, int cap, int* samples, int* nDraw) {
  *nDraw = 0;
  if (N < 5) return 0;
  int const nShuffles = std::max(1, (int)((float)nSamples * (float)5 / (float)N + 0.5));
  std::vector<unsigned int> indices(N);
  for (int i = 0; i < N; ++i) indices[i] = i;
  srand(seed);
  int drawn = 0;
  for (int s = 0; s < nShuffles; ++s) {
    if (drawn > nSamples) break;
    std::random_shuffle(indices.begin(), indices.end());
    for (int j = 0; j < N - 5; j += 5) {
      if (drawn > nSamples) break;
      if (drawn < cap)
        for (int k = 0; k < 5; ++k) samples[5 * drawn + k] = (int)indices[j + k];
      ++drawn;
    }
  }
  *nDraw = std::min(drawn, cap);
  return 0;
}

// The loop of computeRobustOrientationMLE on the given samples (nDraw of them, in order), with
// (refine != 0) or without mode.iterativeRefinement (reconstruction_common.cpp:255-305: the
// accepted pose refined by refineRelativePose on the inliers of its F, then E, F, cost and inlier
// count from the refined pose).  model: E 9, F 9, R 9, T 3, error (-1 when nothing was accepted);
// *nInliers and flags (N bytes) from the chosen F; *chosen = sample * 10 + solution index, or -1.
// swap: bit 0 the restated five-point solver, bit 1 the restated pose recovery, bit 2 the restated
// refinement in place of the reference's.
constexpr int kSwapSolver = 1, kSwapPose = 2, kSwapRefine = 4;

int ref_ransac_swap(int N, const float* corrs, const double* K1, const double* K2, double inlierThreshold,
                    int nSamples, int nDraw, const int* samples, int refine, int swap, double* model, int* nInliers,
                    unsigned char* flags, int* chosen) {
  int const minSize = 5;
  double const sqrInlierThreshold = inlierThreshold * inlierThreshold;
  for (int k = 0; k < 30; ++k) model[k] = 0.0;
  model[30] = -1.0;
  *nInliers = -1;
  *chosen = -1;
  if (N < minSize) return 0;
  Matrix3x3d const invK1 = invertedMatrix(mat(K1));
  Matrix3x3d const invK2 = invertedMatrix(mat(K2));
  Matrix3x3d const invK2_t = invK2.transposed();
  std::vector<Vector2d> nl(N), nr(N);
  for (int i = 0; i < N; ++i) {
    Vector2d l, r;
    l[0] = corrs[4 * i];
    l[1] = corrs[4 * i + 1];
    r[0] = corrs[4 * i + 2];
    r[1] = corrs[4 * i + 3];
    multiply_A_v_projective(invK1, l, nl[i]);
    multiply_A_v_projective(invK2, r, nr[i]);
  }
  double minError = 1e30;
  Matrix3x3d bestF;
  int drawnSamples = 0;
  for (int s = 0; s < nDraw; ++s) {
    if (drawnSamples > nSamples) break;
    double x1[5], y1[5], x2[5], y2[5];
    for (int k = 0; k < 5; ++k) {
      const int c = samples[5 * s + k];
      x1[k] = nl[c][0];
      y1[k] = nl[c][1];
      x2[k] = nr[c][0];
      y2[k] = nr[c][1];
    }
    std::vector<Matrix3x3d> Es;
    if (swap & kSwapSolver) {
      double E10[10][9];
      const int ns = v3dm::ess::five_point(x1, y1, x2, y2, E10);
      Es.resize(ns);
      for (int k = 0; k < ns; ++k) Es[k] = mat(E10[k]);
    } else {
      computeEssentialsFromFiveCorrs(x1, y1, x2, y2, Es);
    }
    ++drawnSamples;
    for (size_t r = 0; r < Es.size(); ++r) {
      Matrix3x3d fund = invK2_t * Es[r] * invK1;
      int nIn = 0;
      double curError = 0;
      for (int i = 0; i < N; ++i) {
        double const dist = sampson(fund, corrs[4 * i], corrs[4 * i + 1], corrs[4 * i + 2], corrs[4 * i + 3]);
        curError += std::min(dist, sqrInlierThreshold);
        if (dist < sqrInlierThreshold) ++nIn;
      }
      if (curError < minError) {
        Matrix3x3d R;
        Vector3d t;
        if (swap & kSwapPose) {
          double Ef[9], Rr[9], Tt[3];
          put(Es[r], Ef);
          if (!v3dm::ess::essential_pose(Ef, 5, x1, y1, x2, y2, Rr, Tt)) continue;
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) R[a][b] = Rr[3 * a + b];
          for (int k = 0; k < 3; ++k) t[k] = Tt[k];
        } else if (!relativePoseFromEssential(Es[r], 5, x1, y1, x2, y2, R, t)) {
          continue;
        }
        if (refine) {
          std::vector<Vector2d> left, right;
          for (int i = 0; i < N; ++i)
            if (sampson(fund, corrs[4 * i], corrs[4 * i + 1], corrs[4 * i + 2], corrs[4 * i + 3]) <
                sqrInlierThreshold) {
              Vector2d l, q;
              l[0] = corrs[4 * i];
              l[1] = corrs[4 * i + 1];
              q[0] = corrs[4 * i + 2];
              q[1] = corrs[4 * i + 3];
              left.push_back(l);
              right.push_back(q);
            }
          if (swap & kSwapRefine) {
            std::vector<v3dm::ess::PoseCorr> c(left.size());
            double iK1[9], iK2[9], iK2t[9], Rr[9], Tt[3];
            put(invK1, iK1);
            put(invK2, iK2);
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) iK2t[3 * a + b] = iK2[3 * b + a];
            for (size_t i = 0; i < left.size(); ++i) {
              Vector2d nl2, nr2;
              multiply_A_v_projective(invK1, left[i], nl2);
              multiply_A_v_projective(invK2, right[i], nr2);
              c[i].lx = nl2[0];
              c[i].ly = nl2[1];
              c[i].rx = nr2[0];
              c[i].ry = nr2[1];
              c[i].plx = left[i][0];
              c[i].ply = left[i][1];
              c[i].prx = right[i][0];
              c[i].pry = right[i][1];
            }
            put(R, Rr);
            for (int k = 0; k < 3; ++k) Tt[k] = t[k];
            std::vector<double> w(c.size()), e(c.size());
            v3dm::ess::refine_pose(c.data(), (int)c.size(), iK1, iK2t, inlierThreshold, Rr, Tt, w.data(), e.data());
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) R[a][b] = Rr[3 * a + b];
            for (int k = 0; k < 3; ++k) t[k] = Tt[k];
          } else {
            refineRelativePose(left, right, mat(K1), mat(K2), R, t, inlierThreshold);
          }
          Matrix3x3d const E_refined = computeEssentialFromRelativePose(R, t);
          Matrix3x3d const F_refined = invK2_t * E_refined * invK1;
          double curError_refined = 0;
          nIn = 0;
          for (int i = 0; i < N; ++i) {
            double const dist = sampson(F_refined, corrs[4 * i], corrs[4 * i + 1], corrs[4 * i + 2], corrs[4 * i + 3]);
            curError_refined += std::min(dist, sqrInlierThreshold);
            if (dist < sqrInlierThreshold) ++nIn;
          }
          fund = F_refined;
          Es[r] = E_refined;
          curError = std::min(curError, curError_refined);
        }
        minError = curError;
        put(Es[r], model);
        put(fund, model + 9);
        put(R, model + 18);
        for (int k = 0; k < 3; ++k) model[27 + k] = t[k];
        model[30] = minError / N;
        bestF = fund;
        *chosen = s * 10 + (int)r;
        double const outlierFraction = 1.0 - float(nIn - minSize) / float(N - minSize);
        nSamples = std::min(nSamples, budget(minSize, outlierFraction, 1.0 - 10e-10));
      }
    }
  }
  if (*chosen < 0) return 0;
  int n = 0;
  for (int i = 0; i < N; ++i) {
    const bool in = sampson(bestF, corrs[4 * i], corrs[4 * i + 1], corrs[4 * i + 2], corrs[4 * i + 3]) <
                    sqrInlierThreshold;
    if (flags) flags[i] = in;
    n += in;
  }
  *nInliers = n;
  return 0;
}

// refineRelativePose(left, right, K1, K2, R, T, inlierThreshold) (v3d_poseutilities.cpp:1063-1101)
// on n pixel correspondences (left[2n], right[2n]); R (row-major) and T refined in place.
int ref_refine_pose(int n, const double* left, const double* right, const double* K1, const double* K2,
                    double inlierThreshold, double* R, double* T) {
  std::vector<Vector2d> l(n), r(n);
  for (int i = 0; i < n; ++i) {
    l[i][0] = left[2 * i];
    l[i][1] = left[2 * i + 1];
    r[i][0] = right[2 * i];
    r[i][1] = right[2 * i + 1];
  }
  Matrix3x3d Rm = mat(R);
  Vector3d t;
  for (int k = 0; k < 3; ++k) t[k] = T[k];
  refineRelativePose(l, r, mat(K1), mat(K2), Rm, t, inlierThreshold);
  put(Rm, R);
  for (int k = 0; k < 3; ++k) T[k] = t[k];
  return 0;
}

int ref_ransac(int N, const float* corrs, const double* K1, const double* K2, double inlierThreshold, int nSamples,
               int nDraw, const int* samples, double* model, int* nInliers, unsigned char* flags, int* chosen) {
  return ref_ransac_swap(N, corrs, K1, K2, inlierThreshold, nSamples, nDraw, samples, 0, 0, model, nInliers, flags,
                         chosen);
}

// The reference's own loop (no component replaced).
int ref_ransac_mode(int N, const float* corrs, const double* K1, const double* K2, double inlierThreshold,
                    int nSamples, int nDraw, const int* samples, int refine, double* model, int* nInliers,
                    unsigned char* flags, int* chosen) {
  return ref_ransac_swap(N, corrs, K1, K2, inlierThreshold, nSamples, nDraw, samples, refine, 0, model, nInliers,
                         flags, chosen);
}

}  // extern "C"
