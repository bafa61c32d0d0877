// Host build of the library's five-point solver and Sampson error (eth-v3d-lgpl_b200/csrc/
// v3dm_essential.cuh is host and device code), for the CPU parity test against the reference's
// computeEssentialsFromFiveCorrs.
#include <vector>

#include "v3dm_essential.cuh"

extern "C" int host_five_point(const double* x1, const double* y1, const double* x2, const double* y2, double* E) {
  double Es[10][9];
  const int n = v3dm::ess::five_point(x1, y1, x2, y2, Es);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < 9; ++j) E[9 * k + j] = Es[k][j];
  return n;
}

extern "C" int host_pose(const double* E, const double* x1, const double* y1, const double* x2, const double* y2,
                         double* R, double* T) {
  return v3dm::ess::essential_pose(E, 5, x1, y1, x2, y2, R, T) ? 1 : 0;
}

// The Sampson error, the truncated term and its inlier flag for n correspondences under F.
extern "C" void host_sampson(const double* F, int n, const float* c, double thr2, double* d, double* trunc,
                             unsigned char* inlier) {
  for (int i = 0; i < n; ++i) {
    d[i] = v3dm::ess::sampson(F, c[4 * i], c[4 * i + 1], c[4 * i + 2], c[4 * i + 3]);
    bool in = false;
    trunc[i] = v3dm::ess::sampson_truncated(F, c[4 * i], c[4 * i + 1], c[4 * i + 2], c[4 * i + 3], thr2, in);
    inlier[i] = in;
  }
}

// The library's restatement of refineRelativePose on n pixel correspondences (left[2n], right[2n]),
// normalised with K^-1 (invK1, invK2 row-major) as multiply_A_v_projective; R, T refined in place.
extern "C" void host_refine_pose(int n, const double* left, const double* right, const double* invK1,
                                 const double* invK2, double thr, double* R, double* T) {
  std::vector<v3dm::ess::PoseCorr> c(n);
  auto project = [](const double* A, double x, double y, double& u, double& v) {
    double w = A[8];
    w += A[6] * x;
    w += A[7] * y;
    double a = A[2], b = A[5];
    a += A[0] * x;
    a += A[1] * y;
    b += A[3] * x;
    b += A[4] * y;
    u = a / w;
    v = b / w;
  };
  for (int i = 0; i < n; ++i) {
    c[i].plx = left[2 * i];
    c[i].ply = left[2 * i + 1];
    c[i].prx = right[2 * i];
    c[i].pry = right[2 * i + 1];
    project(invK1, c[i].plx, c[i].ply, c[i].lx, c[i].ly);
    project(invK2, c[i].prx, c[i].pry, c[i].rx, c[i].ry);
  }
  double invK2t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) invK2t[3 * i + j] = invK2[3 * j + i];
  std::vector<double> w(n), e(n);
  v3dm::ess::refine_pose(c.data(), n, invK1, invK2t, thr, R, T, w.data(), e.data());
}

// The double-double sin and cos of the device rotation update, on the host.
extern "C" void host_sincos_dd(int n, const double* x, double* s, double* c) {
  for (int i = 0; i < n; ++i) v3dm::ess::sincos_dd(x[i], s + i, c + i);
}
