// Host build of the library's five-point solver and Sampson error (eth-v3d-lgpl_b200/csrc/
// v3dm_essential.cuh is host and device code), for the CPU parity test against the reference's
// computeEssentialsFromFiveCorrs.
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
