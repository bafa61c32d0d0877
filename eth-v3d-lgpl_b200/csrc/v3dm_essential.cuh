// v3dm_essential.cuh -- essential matrices from five correspondences, relative pose from an
// essential matrix and the Sampson error; host and device code (the RANSAC kernels run it on the
// GPU, the host tests run the same source on the CPU).
//
// Five-point solver: Nister's method ("An efficient solution to the five-point relative pose
// problem", PAMI 2004), the method of the reference's computeEssentialsFromFiveCorrs
// (V3D/Geometry/v3d_poseutilities.cpp:1016-1060), restated here:
//   1. E lies in the null space of the 5 x 9 epipolar constraints q^T E p = 0: a basis
//      X, Y, Z, W from a Householder QR of the transposed constraint matrix;
//   2. E = x X + y Y + z Z + W must satisfy det E = 0 and 2 E E^T E - tr(E E^T) E = 0: ten
//      cubic equations in (x, y, z) over 20 monomials, built by polynomial arithmetic;
//   3. Gauss-Jordan elimination of the first ten monomials (x^3 y^3 x^2y xy^2 x^2z x^2 y^2z y^2
//      xyz xy) leaves rows from which (row e - z row f), (row g - z row h), (row i - z row j)
//      are three equations linear in (x, y, 1) with coefficients polynomial in z;
//   4. their 3 x 3 determinant is a degree-10 polynomial in z whose real roots (bracketed by
//      the real roots of its derivatives, refined by safeguarded Newton steps) give z; x and y
//      follow from the null vector of the 3 x 3 matrix at that z.
// Convention as the reference's: q^T E p = 0 for a left point p and a right point q.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define V3DM_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define V3DM_HD inline
#endif

namespace v3dm {
namespace ess {

// Double operations with one rounding each (no contraction into fused multiply-adds), so that the
// device and the host compute the same bits.
#ifdef __CUDA_ARCH__
V3DM_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
V3DM_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
V3DM_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
V3DM_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
#else
V3DM_HD double dmul(double a, double b) { return a * b; }
V3DM_HD double dadd(double a, double b) { return a + b; }
V3DM_HD double dsub(double a, double b) { return a - b; }
V3DM_HD double ddiv(double a, double b) { return a / b; }
#endif

// Monomials of degree <= 3 in (x, y, z), in elimination order.
enum : int {
  kX3, kY3, kX2Y, kXY2, kX2Z, kX2, kY2Z, kY2, kXYZ, kXY,
  kXZ2, kXZ, kX, kYZ2, kYZ, kY, kZ3, kZ2, kZ, k1
};

V3DM_HD int mono_index(int a, int b, int c) {  // x^a y^b z^c -> monomial index (a + b + c <= 3)
  switch (a * 16 + b * 4 + c) {
    case 3 * 16: return kX3;
    case 3 * 4: return kY3;
    case 2 * 16 + 4: return kX2Y;
    case 16 + 2 * 4: return kXY2;
    case 2 * 16 + 1: return kX2Z;
    case 2 * 16: return kX2;
    case 2 * 4 + 1: return kY2Z;
    case 2 * 4: return kY2;
    case 16 + 4 + 1: return kXYZ;
    case 16 + 4: return kXY;
    case 16 + 2: return kXZ2;
    case 16 + 1: return kXZ;
    case 16: return kX;
    case 4 + 2: return kYZ2;
    case 4 + 1: return kYZ;
    case 4: return kY;
    case 3: return kZ3;
    case 2: return kZ2;
    case 1: return kZ;
    default: return k1;
  }
}

// A linear polynomial l[0] x + l[1] y + l[2] z + l[3]; a quadratic one over the monomials
// x^2 y^2 z^2 xy xz yz x y z 1 (exponents below); a cubic one over the 20 monomials above.
V3DM_HD void lin_exp(int k, int& a, int& b, int& c) {
  a = k == 0;
  b = k == 1;
  c = k == 2;
}
V3DM_HD void quad_exp(int k, int& a, int& b, int& c) {
  const int ta[10] = {2, 0, 0, 1, 1, 0, 1, 0, 0, 0};
  const int tb[10] = {0, 2, 0, 1, 0, 1, 0, 1, 0, 0};
  const int tc[10] = {0, 0, 2, 0, 1, 1, 0, 0, 1, 0};
  a = ta[k];
  b = tb[k];
  c = tc[k];
}
V3DM_HD int quad_index(int a, int b, int c) {
  for (int k = 0; k < 10; ++k) {
    int qa, qb, qc;
    quad_exp(k, qa, qb, qc);
    if (qa == a && qb == b && qc == c) return k;
  }
  return 9;
}

V3DM_HD void mul_lin_lin(const double* u, const double* v, double* q) {  // q (10) = u v
  for (int k = 0; k < 10; ++k) q[k] = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      int a1, b1, c1, a2, b2, c2;
      lin_exp(i, a1, b1, c1);
      lin_exp(j, a2, b2, c2);
      q[quad_index(a1 + a2, b1 + b2, c1 + c2)] += u[i] * v[j];
    }
}

V3DM_HD void mul_quad_lin_acc(const double* q, const double* v, double s, double* cub) {  // cub (20) += s q v
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 4; ++j) {
      int a1, b1, c1, a2, b2, c2;
      quad_exp(i, a1, b1, c1);
      lin_exp(j, a2, b2, c2);
      cub[mono_index(a1 + a2, b1 + b2, c1 + c2)] += s * q[i] * v[j];
    }
}

// Null-space basis of the 5 x 9 constraints: rows of N (4 x 9).  Householder QR of the 9 x 5
// transpose; the last four columns of Q are orthonormal and orthogonal to the constraints.
V3DM_HD void null_space(const double* x1, const double* y1, const double* x2, const double* y2, double N[4][9]) {
  double M[9][5];  // column k = constraint row of correspondence k (E entries row-major)
  for (int k = 0; k < 5; ++k) {
    M[0][k] = x2[k] * x1[k];
    M[1][k] = x2[k] * y1[k];
    M[2][k] = x2[k];
    M[3][k] = y2[k] * x1[k];
    M[4][k] = y2[k] * y1[k];
    M[5][k] = y2[k];
    M[6][k] = x1[k];
    M[7][k] = y1[k];
    M[8][k] = 1.0;
  }
  double vs[5][9];  // Householder vectors
  for (int k = 0; k < 5; ++k) {
    double nrm = 0.0;
    for (int i = k; i < 9; ++i) nrm += M[i][k] * M[i][k];
    nrm = sqrt(nrm);
    const double alpha = M[k][k] > 0 ? -nrm : nrm;
    double vn = 0.0;
    for (int i = 0; i < 9; ++i) {
      vs[k][i] = i < k ? 0.0 : M[i][k];
      if (i == k) vs[k][i] -= alpha;
      vn += vs[k][i] * vs[k][i];
    }
    if (vn > 0.0) {
      const double inv = 1.0 / sqrt(vn);
      for (int i = 0; i < 9; ++i) vs[k][i] *= inv;
    }
    for (int c = k; c < 5; ++c) {  // M <- (I - 2 v v^T) M
      double d = 0.0;
      for (int i = k; i < 9; ++i) d += vs[k][i] * M[i][c];
      for (int i = k; i < 9; ++i) M[i][c] -= 2.0 * d * vs[k][i];
    }
  }
  // Q e_j for j = 5..8: apply the reflections in reverse order to unit vectors
  for (int n = 0; n < 4; ++n) {
    double e[9];
    for (int i = 0; i < 9; ++i) e[i] = i == 5 + n ? 1.0 : 0.0;
    for (int k = 4; k >= 0; --k) {
      double d = 0.0;
      for (int i = k; i < 9; ++i) d += vs[k][i] * e[i];
      for (int i = k; i < 9; ++i) e[i] -= 2.0 * d * vs[k][i];
    }
    for (int i = 0; i < 9; ++i) N[n][i] = e[i];
  }
}

// The ten cubic constraints on (x, y, z) for E = x N0 + y N1 + z N2 + N3: A[10][20].
V3DM_HD void constraints(const double N[4][9], double A[10][20]) {
  double E[3][3][4];  // E[r][c] as a linear polynomial
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 4; ++k) E[r][c][k] = N[k][3 * r + c];
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 20; ++j) A[i][j] = 0.0;
  // det E by the first row
  double q[10];
  mul_lin_lin(E[1][1], E[2][2], q);
  mul_quad_lin_acc(q, E[0][0], 1.0, A[0]);
  mul_lin_lin(E[1][2], E[2][1], q);
  mul_quad_lin_acc(q, E[0][0], -1.0, A[0]);
  mul_lin_lin(E[1][2], E[2][0], q);
  mul_quad_lin_acc(q, E[0][1], 1.0, A[0]);
  mul_lin_lin(E[1][0], E[2][2], q);
  mul_quad_lin_acc(q, E[0][1], -1.0, A[0]);
  mul_lin_lin(E[1][0], E[2][1], q);
  mul_quad_lin_acc(q, E[0][2], 1.0, A[0]);
  mul_lin_lin(E[1][1], E[2][0], q);
  mul_quad_lin_acc(q, E[0][2], -1.0, A[0]);
  // EEt = E E^T (quadratic), trace
  double EEt[3][3][10];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      for (int k = 0; k < 10; ++k) EEt[i][j][k] = 0.0;
      for (int k = 0; k < 3; ++k) {
        mul_lin_lin(E[i][k], E[j][k], q);
        for (int m = 0; m < 10; ++m) EEt[i][j][m] += q[m];
      }
    }
  double tr[10];
  for (int m = 0; m < 10; ++m) tr[m] = EEt[0][0][m] + EEt[1][1][m] + EEt[2][2][m];
  // 2 EEt E - tr E
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double* row = A[1 + 3 * i + j];
      for (int k = 0; k < 3; ++k) mul_quad_lin_acc(EEt[i][k], E[k][j], 2.0, row);
      mul_quad_lin_acc(tr, E[i][j], -1.0, row);
    }
}

// Gauss-Jordan elimination of the first ten columns (partial pivoting).  false if singular.
V3DM_HD bool eliminate(double A[10][20]) {
  for (int c = 0; c < 10; ++c) {
    int p = c;
    double best = fabs(A[c][c]);
    for (int r = c + 1; r < 10; ++r)
      if (fabs(A[r][c]) > best) {
        best = fabs(A[r][c]);
        p = r;
      }
    if (!(best > 0.0)) return false;
    if (p != c)
      for (int j = 0; j < 20; ++j) {
        const double t = A[c][j];
        A[c][j] = A[p][j];
        A[p][j] = t;
      }
    const double inv = 1.0 / A[c][c];
    for (int j = c; j < 20; ++j) A[c][j] *= inv;
    for (int r = 0; r < 10; ++r) {
      if (r == c) continue;
      const double f = A[r][c];
      if (f == 0.0) continue;
      for (int j = c; j < 20; ++j) A[r][j] -= f * A[c][j];
    }
  }
  return true;
}

// Polynomials in z, ascending powers.
V3DM_HD void pmul(const double* a, int na, const double* b, int nb, double* c) {  // c (na + nb - 1) = a b
  for (int k = 0; k < na + nb - 1; ++k) c[k] = 0.0;
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) c[i + j] += a[i] * b[j];
}

V3DM_HD double peval(const double* a, int deg, double z) {
  double v = a[deg];
  for (int k = deg - 1; k >= 0; --k) v = v * z + a[k];
  return v;
}

// B(z): the three equations (row e - z row f) etc. as [x coefficient (cubic), y coefficient
// (cubic), constant (quartic)], ascending powers of z.
V3DM_HD void z_matrix(const double A[10][20], double Bx[3][4], double By[3][4], double B1[3][5]) {
  for (int r = 0; r < 3; ++r) {
    const double* e = A[4 + 2 * r];
    const double* f = A[5 + 2 * r];
    Bx[r][0] = e[kX];
    Bx[r][1] = e[kXZ] - f[kX];
    Bx[r][2] = e[kXZ2] - f[kXZ];
    Bx[r][3] = -f[kXZ2];
    By[r][0] = e[kY];
    By[r][1] = e[kYZ] - f[kY];
    By[r][2] = e[kYZ2] - f[kYZ];
    By[r][3] = -f[kYZ2];
    B1[r][0] = e[k1];
    B1[r][1] = e[kZ] - f[k1];
    B1[r][2] = e[kZ2] - f[kZ];
    B1[r][3] = e[kZ3] - f[kZ2];
    B1[r][4] = -f[kZ3];
  }
}

// det B(z): degree 10, 11 coefficients ascending.
V3DM_HD void z_determinant(const double Bx[3][4], const double By[3][4], const double B1[3][5], double n[11]) {
  double t1[8], t2[8], m[8], acc[11];
  for (int k = 0; k < 11; ++k) n[k] = 0.0;
  // + Bx0 (By1 B12 - B11 By2)
  pmul(By[1], 4, B1[2], 5, t1);
  pmul(B1[1], 5, By[2], 4, t2);
  for (int k = 0; k < 8; ++k) m[k] = t1[k] - t2[k];
  pmul(Bx[0], 4, m, 8, acc);
  for (int k = 0; k < 11; ++k) n[k] += acc[k];
  // - By0 (Bx1 B12 - B11 Bx2)
  pmul(Bx[1], 4, B1[2], 5, t1);
  pmul(B1[1], 5, Bx[2], 4, t2);
  for (int k = 0; k < 8; ++k) m[k] = t1[k] - t2[k];
  pmul(By[0], 4, m, 8, acc);
  for (int k = 0; k < 11; ++k) n[k] -= acc[k];
  // + B10 (Bx1 By2 - By1 Bx2)
  double s1[7], s2[7];
  pmul(Bx[1], 4, By[2], 4, s1);
  pmul(By[1], 4, Bx[2], 4, s2);
  for (int k = 0; k < 7; ++k) m[k] = s1[k] - s2[k];
  pmul(B1[0], 5, m, 7, acc);
  for (int k = 0; k < 11; ++k) n[k] += acc[k];
}

// p(z) and p'(z) by Horner.
V3DM_HD void peval2(const double* a, int deg, double z, double& p, double& dp) {
  p = a[deg];
  dp = 0.0;
  for (int k = deg - 1; k >= 0; --k) {
    dp = dp * z + p;
    p = p * z + a[k];
  }
}

// The root of a in (lo, hi) where a changes sign: Newton steps kept inside the bracket, bisection
// when a step leaves it or does not halve the bracket.
V3DM_HD double bracket_root(const double* a, int deg, double lo, double hi, double flo) {
  double x = 0.5 * (lo + hi), dxold = hi - lo, dx = dxold;
  double f, df;
  peval2(a, deg, x, f, df);
  for (int it = 0; it < 100; ++it) {
    if ((((x - hi) * df - f) * ((x - lo) * df - f) > 0.0) || (fabs(2.0 * f) > fabs(dxold * df))) {
      dxold = dx;
      dx = 0.5 * (hi - lo);
      x = lo + dx;
    } else {
      dxold = dx;
      dx = f / df;
      x -= dx;
    }
    if (fabs(dx) <= 1e-15 * fmax(1.0, fabs(x))) break;
    peval2(a, deg, x, f, df);
    if (f == 0.0) break;
    if ((f < 0.0) == (flo < 0.0)) lo = x;
    else hi = x;
  }
  return x;
}

// Real roots of the polynomial a (degree <= 10, ascending coefficients), ascending: the real roots
// of each derivative bracket those of the next lower one (all lie within the Cauchy bound of a,
// Gauss-Lucas), from the linear (deg-1)-th derivative down to a itself.  Roots of even
// multiplicity (no sign change) are not reported.  Returns the count.
V3DM_HD int real_roots(const double* a_in, int deg_in, double* roots) {
  double amax = 0.0;
  for (int k = 0; k <= deg_in; ++k) amax = fmax(amax, fabs(a_in[k]));
  if (!(amax > 0.0)) return 0;
  int deg = deg_in;
  while (deg > 0 && fabs(a_in[deg]) <= 1e-14 * amax) --deg;  // vanishing leading terms
  if (deg < 1) return 0;
  double D[11][11];  // D[k] = k-th derivative of the monic polynomial, divided by k!, degree deg - k
  for (int j = 0; j <= deg; ++j) D[0][j] = a_in[j] / a_in[deg];
  for (int k = 1; k < deg; ++k)
    for (int j = 0; j <= deg - k; ++j) D[k][j] = D[k - 1][j + 1] * (double)(j + 1) / (double)k;
  double bound = 0.0;
  for (int j = 0; j < deg; ++j) bound = fmax(bound, fabs(D[0][j]));
  bound += 1.0;
  double crit[10];
  int nc = 0;
  crit[nc++] = -D[deg - 1][0] / D[deg - 1][1];  // the linear derivative's root
  if (!(fabs(crit[0]) < bound)) nc = 0;
  for (int k = deg - 2; k >= 0; --k) {
    const double* P = D[k];
    const int dk = deg - k;
    double next[10];
    int nn = 0;
    double u = -bound, pu = peval(P, dk, u);
    for (int c = 0; c <= nc; ++c) {
      const double v = c < nc ? crit[c] : bound;
      const double pv = peval(P, dk, v);
      if (pu == 0.0) {
        if (nn < 10 && (nn == 0 || next[nn - 1] != u)) next[nn++] = u;
      } else if ((pu < 0.0) != (pv < 0.0) && pv != 0.0) {
        if (nn < 10) next[nn++] = bracket_root(P, dk, u, v, pu);
      }
      u = v;
      pu = pv;
    }
    if (pu == 0.0 && nn < 10 && (nn == 0 || next[nn - 1] != u)) next[nn++] = u;
    for (int c = 0; c < nn; ++c) crit[c] = next[c];
    nc = nn;
  }
  for (int c = 0; c < nc; ++c) roots[c] = crit[c];
  return nc;
}

// Essential matrices (row-major, up to 10) of five normalised correspondences; returns the count.
V3DM_HD int five_point(const double* x1, const double* y1, const double* x2, const double* y2, double Es[10][9]) {
  double N[4][9];
  null_space(x1, y1, x2, y2, N);
  double A[10][20];
  constraints(N, A);
  if (!eliminate(A)) return 0;
  double Bx[3][4], By[3][4], B1[3][5];
  z_matrix(A, Bx, By, B1);
  double poly[11];
  z_determinant(Bx, By, B1, poly);
  double zs[10];
  const int nz = real_roots(poly, 10, zs);
  int n = 0;
  for (int s = 0; s < nz; ++s) {
    const double z = zs[s];
    double R[3][3];
    for (int r = 0; r < 3; ++r) {
      R[r][0] = peval(Bx[r], 3, z);
      R[r][1] = peval(By[r], 3, z);
      R[r][2] = peval(B1[r], 4, z);
    }
    // null vector of R: the largest-last-component cross product of two rows
    double best[3] = {0.0, 0.0, 0.0};
    for (int pr = 0; pr < 3; ++pr) {
      const double* u = R[pr == 2 ? 1 : 0];
      const double* v = R[pr == 0 ? 1 : 2];
      const double c0 = u[1] * v[2] - u[2] * v[1];
      const double c1 = u[2] * v[0] - u[0] * v[2];
      const double c2 = u[0] * v[1] - u[1] * v[0];
      if (fabs(c2) > fabs(best[2])) {
        best[0] = c0;
        best[1] = c1;
        best[2] = c2;
      }
    }
    if (!(fabs(best[2]) > 0.0)) continue;
    const double x = best[0] / best[2], y = best[1] / best[2];
    for (int k = 0; k < 9; ++k) Es[n][k] = x * N[0][k] + y * N[1][k] + z * N[2][k] + N[3][k];
    ++n;
  }
  return n;
}

// Sampson error of a correspondence (p left, q right, pixels) under F (row-major), in the
// operation order of sampsonEpipolarError (V3D/Apps/SfM/reconstruction_common.h:589-607).
V3DM_HD double sampson(const double* F, float px, float py, float qx, float qy) {
  // F p and F^T q as multiply_A_v_affine (v3d_linearbase.h:1049-1062): the last column first
  const double p0 = px, p1 = py, q0 = qx, q1 = qy;
  const double Fp0 = dadd(dadd(F[2], dmul(F[0], p0)), dmul(F[1], p1));
  const double Fp1 = dadd(dadd(F[5], dmul(F[3], p0)), dmul(F[4], p1));
  const double Fp2 = dadd(dadd(F[8], dmul(F[6], p0)), dmul(F[7], p1));
  const double Ftq0 = dadd(dadd(F[6], dmul(F[0], q0)), dmul(F[3], q1));
  const double Ftq1 = dadd(dadd(F[7], dmul(F[1], q0)), dmul(F[4], q1));
  const double tmp = dadd(dadd(dmul(q0, Fp0), dmul(q1, Fp1)), Fp2);
  const double num = dmul(tmp, tmp);
  const double denom = dadd(dadd(dadd(dmul(Fp0, Fp0), dmul(Fp1, Fp1)), dmul(Ftq0, Ftq0)), dmul(Ftq1, Ftq1));
  return ddiv(num, denom);
}

// The truncated Sampson term min(d, thr2) of sampsonEpipolarError(corr, F) = d and whether
// d < thr2, for a correspondence given in double (the float positions converted): the division
// is skipped when num > thr2 * denom * (1 + 1e-12), where the rounded quotient is certainly >= thr2
// (the margin is far above the rounding of the comparison's product), so the result is that of
// the exact expression in every case.
V3DM_HD double sampson_truncated(const double* F, double p0, double p1, double q0, double q1, double thr2,
                                 bool& inlier) {
  const double Fp0 = dadd(dadd(F[2], dmul(F[0], p0)), dmul(F[1], p1));
  const double Fp1 = dadd(dadd(F[5], dmul(F[3], p0)), dmul(F[4], p1));
  const double Fp2 = dadd(dadd(F[8], dmul(F[6], p0)), dmul(F[7], p1));
  const double Ftq0 = dadd(dadd(F[6], dmul(F[0], q0)), dmul(F[3], q1));
  const double Ftq1 = dadd(dadd(F[7], dmul(F[1], q0)), dmul(F[4], q1));
  const double tmp = dadd(dadd(dmul(q0, Fp0), dmul(q1, Fp1)), Fp2);
  const double num = dmul(tmp, tmp);
  const double denom = dadd(dadd(dadd(dmul(Fp0, Fp0), dmul(Fp1, Fp1)), dmul(Ftq0, Ftq0)), dmul(Ftq1, Ftq1));
  if (num > thr2 * denom * (1.0 + 1e-12)) {  // denom > 0 here; the quotient is >= thr2
    inlier = false;
    return thr2;
  }
  const double d = ddiv(num, denom);
  inlier = d < thr2;
  return thr2 < d ? thr2 : d;  // std::min(d, thr2)
}

// C = A B for row-major 3 x 3 matrices, each entry summed over k = 0, 1, 2 in order.
V3DM_HD void mat3_mul(const double* A, const double* B, double* C) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      C[3 * i + j] = dadd(dadd(dmul(A[3 * i], B[j]), dmul(A[3 * i + 1], B[3 + j])), dmul(A[3 * i + 2], B[6 + j]));
}

// ---- relative pose from an essential matrix -------------------------------------------------
// relativePoseFromEssential(E, nCorrs, x1, y1, x2, y2, R, T) (v3d_poseutilities.cpp:1264-1294):
// E = U diag(1, 1, 0) V^T from cross products of E's rows (the essential-matrix SVD of Nister's
// paper, as computeEssentialSVD, :1137-1191); with D = [[0 1 0] [-1 0 0] [0 0 1]] the four
// candidate poses are (U D V^T, +-u3) and (U D^T V^T, +-u3).  Each correspondence is triangulated
// exactly against P = [U D V^T | u3] and classified into the candidate that puts it in front of
// both cameras (Nister's twisted-pair test, the decisions of getExactConfiguration, :1194-1225);
// the pose is accepted when all the correspondences agree.
V3DM_HD void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
V3DM_HD double norm3(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// U, V (row-major 3 x 3, columns are the singular vectors) of an essential matrix.
V3DM_HD void essential_svd(const double* E, double* U, double* V) {
  const double* ea = E;
  const double* eb = E + 3;
  const double* ec = E + 6;
  double ab[3], ac[3], bc[3];
  cross3(ea, eb, ab);
  cross3(ea, ec, ac);
  cross3(eb, ec, bc);
  const double* x = ab;
  const double* y = ea;
  double len = norm3(ab);
  if (norm3(ac) > len) {
    len = norm3(ac);
    x = ac;
    y = ea;
  }
  if (norm3(bc) > len) {
    len = norm3(bc);
    x = bc;
    y = eb;
  }
  double va[3], vb[3], vc[3];
  for (int k = 0; k < 3; ++k) vc[k] = x[k] / len;
  const double ny = norm3(y);
  for (int k = 0; k < 3; ++k) va[k] = y[k] / ny;
  cross3(vc, va, vb);
  double ua[3], ub[3], uc[3];
  for (int r = 0; r < 3; ++r) {
    ua[r] = E[3 * r] * va[0] + E[3 * r + 1] * va[1] + E[3 * r + 2] * va[2];
    ub[r] = E[3 * r] * vb[0] + E[3 * r + 1] * vb[1] + E[3 * r + 2] * vb[2];
  }
  const double na = norm3(ua), nb = norm3(ub);
  for (int k = 0; k < 3; ++k) {
    ua[k] /= na;
    ub[k] /= nb;
  }
  cross3(ua, ub, uc);
  for (int r = 0; r < 3; ++r) {
    V[3 * r] = va[r];
    V[3 * r + 1] = vb[r];
    V[3 * r + 2] = vc[r];
    U[3 * r] = ua[r];
    U[3 * r + 1] = ub[r];
    U[3 * r + 2] = uc[r];
  }
}

// R = U D V^T (twist 0) or U D^T V^T (twist 1).
V3DM_HD void twisted_rotation(const double* U, const double* V, int twist, double* R) {
  // D V^T rows: (v2^T, -v1^T, v3^T); D^T V^T rows: (-v2^T, v1^T, v3^T) (v_k = column k of V)
  double DVt[9];
  const double s = twist ? -1.0 : 1.0;
  for (int c = 0; c < 3; ++c) {
    DVt[c] = s * V[3 * c + 1];
    DVt[3 + c] = -s * V[3 * c];
    DVt[6 + c] = V[3 * c + 2];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[3 * i + j] = U[3 * i] * DVt[j] + U[3 * i + 1] * DVt[3 + j] + U[3 * i + 2] * DVt[6 + j];
}

// Candidate (0..3) that puts the correspondence (x1, y1) <-> (x2, y2) in front of both cameras.
V3DM_HD int pose_configuration(const double* E, const double* U, const double* V, double x1, double y1, double x2,
                               double y2) {
  const double p[3] = {x1, y1, 1.0}, q[3] = {x2, y2, 1.0};
  double R[9];
  twisted_rotation(U, V, 0, R);
  const double t[3] = {U[2], U[5], U[8]};
  // exact triangulation against P = [R | t]: c = q x (diag(1, 1, 0) E p), C = P^T c
  double e1p[3];
  e1p[0] = E[0] * p[0] + E[1] * p[1] + E[2] * p[2];
  e1p[1] = E[3] * p[0] + E[4] * p[1] + E[5] * p[2];
  e1p[2] = 0.0;
  double c[3];
  cross3(q, e1p, c);
  double C[4];
  for (int k = 0; k < 3; ++k) C[k] = R[k] * c[0] + R[3 + k] * c[1] + R[6 + k] * c[2];
  C[3] = t[0] * c[0] + t[1] * c[1] + t[2] * c[2];
  double Q[4] = {p[0] * C[3], p[1] * C[3], p[2] * C[3], -(p[0] * C[0] + p[1] * C[1] + p[2] * C[2])};
  Q[0] /= Q[3];
  Q[1] /= Q[3];
  Q[2] /= Q[3];
  Q[3] = 1.0;
  const double c1 = Q[2] * Q[3];
  const double depth2 = R[6] * Q[0] + R[7] * Q[1] + R[8] * Q[2] + t[2] * Q[3];
  const double c2 = depth2 * Q[3];
  if (c1 >= 0 && c2 >= 0) return 0;  // (R, t)
  if (c1 < 0 && c2 < 0) return 1;    // (R, -t)
  const double cc = -(2 * V[2] * Q[0] + 2 * V[5] * Q[1] + 2 * V[8] * Q[2] + Q[3]);
  if (Q[2] * cc >= 0) return 2;  // (R twisted, t)
  return 3;                      // (R twisted, -t)
}

// true and (R, T) when all n correspondences agree on one candidate.
V3DM_HD bool essential_pose(const double* E, int n, const double* x1, const double* y1, const double* x2,
                            const double* y2, double* R, double* T) {
  double U[9], V[9];
  essential_svd(E, U, V);
  const int conf0 = pose_configuration(E, U, V, x1[0], y1[0], x2[0], y2[0]);
  for (int i = 1; i < n; ++i)
    if (pose_configuration(E, U, V, x1[i], y1[i], x2[i], y2[i]) != conf0) {
      for (int k = 0; k < 9; ++k) R[k] = 0.0;
      T[0] = T[1] = T[2] = 0.0;
      return false;
    }
  twisted_rotation(U, V, conf0 >= 2, R);
  const double sgn = (conf0 == 1 || conf0 == 3) ? -1.0 : 1.0;
  double t[3] = {sgn * U[2], sgn * U[5], sgn * U[8]};
  const double nt = norm3(t);
  for (int k = 0; k < 3; ++k) T[k] = t[k] / nt;
  return true;
}


// ---- refinement of a relative pose ----------------------------------------------------------
// refineRelativePose (v3d_poseutilities.cpp:1063-1101) with its RelativePoseMinimizer (:812-1006)
// on the reference's dense Levenberg-Marquardt loop (V3D/Math/v3d_optimization.h:25-277), restated:
//   f_k = (q^T E p) / sqrt((Ep)_0^2 + (Ep)_1^2 + (E^T q)_0^2 + (E^T q)_1^2) on normalised points,
//   E = [T]x R; weights w_k = 1 if |e_k| < thr, else sqrt(thr / |e_k|), with e_k the same quantity on
//   pixel points under F = K2^-T E K1^-1; residual r = -w f; J = df/d(omega, T) (not weighted);
//   delta = (J^T J + lambda I)^-1 J^T r (Cholesky); R <- R Rodrigues(omega), T <- (T + dT) / |T + dT|;
//   lambda = 1e-3 max diag(J^T J) at the first iteration, x0.1 (at least 1e-10) after an improvement
//   (rho > 0), x10 and the step undone otherwise; stop when |J^T r|_inf < 1e-8, when (from the 10th
//   iteration) |delta| < 1e-8 (4 + 1e-8), or after 50 iterations.
struct PoseCorr {  // one correspondence: normalised and pixel positions
  double lx, ly, rx, ry;
  double plx, ply, prx, pry;
};

V3DM_HD void pose_essential(const double* R, const double* T, double* E) {  // E = [T]x R
  const double Tx[9] = {0.0, -T[2], T[1], T[2], 0.0, -T[0], -T[1], T[0], 0.0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += Tx[3 * i + k] * R[3 * k + j];
      E[3 * i + j] = v;
    }
}

// (q^T M p) / sqrt(...) of one correspondence under M (E on normalised, F on pixel points), with the
// intermediate products; M p and M^T q summed as multiply_A_v_affine (the last column first).
V3DM_HD double pose_residual(const double* M, double px, double py, double qx, double qy, double* Mp, double* Mtq) {
  Mp[0] = M[2] + M[0] * px + M[1] * py;
  Mp[1] = M[5] + M[3] * px + M[4] * py;
  Mp[2] = M[8] + M[6] * px + M[7] * py;
  Mtq[0] = M[6] + M[0] * qx + M[3] * qy;
  Mtq[1] = M[7] + M[1] * qx + M[4] * qy;
  const double num = qx * Mp[0] + qy * Mp[1] + Mp[2];
  const double denom = sqrt(Mp[0] * Mp[0] + Mp[1] * Mp[1] + Mtq[0] * Mtq[0] + Mtq[1] * Mtq[1]);
  return num / denom;
}

// sin and cos of |x| <= 1, correctly rounded (but for inputs whose exact value lies within
// about 2^-100 relative of a rounding boundary): Taylor series evaluated in double-double
// arithmetic (Dekker's exact product and Knuth's exact sum; Hida, Li and Bailey, "Library for
// double-double and quad-double arithmetic", 2001), then rounded once.  The device path of
// pose_update uses them so that the rotation update rounds as the host's C library does; the
// host path calls std::sin / std::cos.
struct DD {
  double hi, lo;
};
V3DM_HD DD dd_two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
V3DM_HD DD dd_add(DD x, DD y) {
  DD s = dd_two_sum(x.hi, y.hi);
  const double lo = s.lo + x.lo + y.lo;
  return dd_two_sum(s.hi, lo);
}
V3DM_HD DD dd_mul(DD x, DD y) {
  const double p = x.hi * y.hi;
  const double e = fma(x.hi, y.hi, -p);
  return dd_two_sum(p, e + (x.hi * y.lo + x.lo * y.hi));
}
V3DM_HD DD dd_div_int(DD x, double n) {  // x / n for an integer n below 2^53
  const double q1 = x.hi / n;
  const double p = q1 * n, pe = fma(q1, n, -p);  // q1 * n exactly
  const double r = ((x.hi - p) - pe) + x.lo;
  return dd_two_sum(q1, r / n);
}
V3DM_HD void sincos_dd(double x, double* sn, double* cs) {
  const DD x2 = dd_mul({x, 0.0}, {x, 0.0});
  DD ts = {x, 0.0}, s = ts;      // x^(2k+1) / (2k+1)!
  DD tc = {1.0, 0.0}, c = tc;    // x^(2k) / (2k)!
  for (int k = 1; k <= 16; ++k) {
    tc = dd_div_int(dd_mul(tc, x2), (double)((2 * k - 1) * (2 * k)));
    ts = dd_div_int(dd_mul(ts, x2), (double)((2 * k) * (2 * k + 1)));
    if (k & 1) {
      c = dd_add(c, {-tc.hi, -tc.lo});
      s = dd_add(s, {-ts.hi, -ts.lo});
    } else {
      c = dd_add(c, tc);
      s = dd_add(s, ts);
    }
  }
  *sn = s.hi + s.lo;
  *cs = c.hi + c.lo;
}

V3DM_HD void pose_update(const double* Rold, const double* Told, const double* delta, double* R, double* T) {
  // createRotationMatrixRodrigues(omega) (v3d_mathutilities.h:170-190), then R = Rold dR
  const double w0 = delta[0], w1 = delta[1], w2 = delta[2];
  const double theta = sqrt(w0 * w0 + w1 * w1 + w2 * w2);
  double dR[9] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};
  if (fabs(theta) > 1e-6) {
    const double J[9] = {0.0, -w2, w1, w2, 0.0, -w0, -w1, w0, 0.0};
    double J2[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double v = 0.0;
        for (int k = 0; k < 3; ++k) v += J[3 * i + k] * J[3 * k + j];
        J2[3 * i + j] = v;
      }
#if defined(__CUDA_ARCH__) || defined(V3DM_HOST_SINCOS_DD)
    double sn, cs;
    if (theta <= 1.0) {
      sincos_dd(theta, &sn, &cs);
    } else {
      sn = sin(theta);
      cs = cos(theta);
    }
#else
    const double sn = std::sin(theta), cs = std::cos(theta);
#endif
    const double c1 = sn / theta;
    const double c2 = (1 - cs) / (theta * theta);
    for (int k = 0; k < 9; ++k) dR[k] += c1 * J[k] + c2 * J2[k];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += Rold[3 * i + k] * dR[3 * k + j];
      R[3 * i + j] = v;
    }
  double t[3] = {Told[0] + delta[3], Told[1] + delta[4], Told[2] + delta[5]};
  const double nt = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  for (int k = 0; k < 3; ++k) T[k] = t[k] / nt;
}

// The weighted residual e = -w f under (R, T), with weights from the pixel positions; returns |e|^2.
V3DM_HD double pose_weighted_residual(const PoseCorr* c, int n, const double* R, const double* T,
                                      const double* invK1, const double* invK2t, double thr, double* w, double* e,
                                      bool fillWeights) {
  double E[9], tmp[9], F[9], a[3], b[2];
  pose_essential(R, T, E);
  if (fillWeights) {
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
    for (int k = 0; k < n; ++k) {
      const double ek = pose_residual(F, c[k].plx, c[k].ply, c[k].prx, c[k].pry, a, b);
      w[k] = (fabs(ek) < thr) ? 1.0 : sqrt(thr / fabs(ek));
    }
  }
  double err = 0.0;
  for (int k = 0; k < n; ++k) {
    e[k] = w[k] * (0.0 - pose_residual(E, c[k].lx, c[k].ly, c[k].rx, c[k].ry, a, b));
    err += e[k] * e[k];
  }
  return err;
}

// dE / d(omega_x, omega_y, omega_z, T_x, T_y, T_z) of E = [T]x R under the update of pose_update.
V3DM_HD void pose_inner(const double* E, const double* R, double (*inner)[6]) {
  for (int r = 0; r < 3; ++r) {
    inner[3 * r + 0][0] = 0.0;
    inner[3 * r + 1][0] = E[3 * r + 2];
    inner[3 * r + 2][0] = -E[3 * r + 1];
    inner[3 * r + 0][1] = -E[3 * r + 2];
    inner[3 * r + 1][1] = 0.0;
    inner[3 * r + 2][1] = E[3 * r + 0];
    inner[3 * r + 0][2] = E[3 * r + 1];
    inner[3 * r + 1][2] = -E[3 * r + 0];
    inner[3 * r + 2][2] = 0.0;
  }
  for (int j = 0; j < 3; ++j) {
    inner[j][3] = 0.0;
    inner[3 + j][3] = -R[6 + j];
    inner[6 + j][3] = R[3 + j];
    inner[j][4] = R[6 + j];
    inner[3 + j][4] = 0.0;
    inner[6 + j][4] = -R[j];
    inner[j][5] = -R[3 + j];
    inner[3 + j][5] = R[j];
    inner[6 + j][5] = 0.0;
  }
}

// Jacobian row of f (the normalised Sampson residual) of one correspondence (p = (lx, ly),
// q = (rx, ry)) under E, from pose_inner's dE/dx.
V3DM_HD void pose_jacobian_row(const double* E, const double (*inner)[6], double lx, double ly, double rx, double ry,
                               double* J) {
  const double p[3] = {lx, ly, 1.0}, q[3] = {rx, ry, 1.0};
  double Ep[3], Etq[2];
  pose_residual(E, p[0], p[1], q[0], q[1], Ep, Etq);  // for E p and E^T q
  const double num = q[0] * Ep[0] + q[1] * Ep[1] + Ep[2];
  const double sqrDenom = Ep[0] * Ep[0] + Ep[1] * Ep[1] + Etq[0] * Etq[0] + Etq[1] * Etq[1];
  const double denom = sqrt(sqrDenom);
  const double invDenom = 1.0 / denom;
  const double invSqrDenom = 1.0 / sqrDenom;
  double outer[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double numDer = (i < 2 ? q[i] : 1.0) * (j < 2 ? p[j] : 1.0);
      double sq = 0.0;  // d(sqrDenom)/dE_ij
      if (i < 2 && j < 2) sq = 2 * Ep[i] * p[j] + 2 * Etq[j] * q[i];
      else if (i < 2) sq = 2 * Ep[i];
      else if (j < 2) sq = 2 * Etq[j];
      outer[3 * i + j] = (numDer * denom - num * 0.5 * invDenom * sq) * invSqrDenom;
    }
  for (int col = 0; col < 6; ++col) {
    double v = 0.0;
    for (int j = 0; j < 9; ++j) v += outer[j] * inner[j][col];
    J[col] = v;
  }
}

// J^T J (6 x 6) and J^T e of f under (R, T).
V3DM_HD void pose_normal_equations(const PoseCorr* c, int n, const double* R, const double* T, const double* e,
                                   double* JtJ, double* Jte) {
  double E[9];
  pose_essential(R, T, E);
  double inner[9][6];
  pose_inner(E, R, inner);
  for (int k = 0; k < 36; ++k) JtJ[k] = 0.0;
  for (int k = 0; k < 6; ++k) Jte[k] = 0.0;
  for (int k = 0; k < n; ++k) {
    double J[6];
    pose_jacobian_row(E, inner, c[k].lx, c[k].ly, c[k].rx, c[k].ry, J);
    for (int a = 0; a < 6; ++a) {
      for (int b = 0; b < 6; ++b) JtJ[6 * a + b] += J[a] * J[b];
      Jte[a] += J[a] * e[k];
    }
  }
}

// x = N^-1 b for a symmetric positive definite 6 x 6 N (Cholesky); false if not positive definite.
V3DM_HD bool cholesky_solve6(const double* N, const double* b, double* x) {
  double L[36];
  for (int k = 0; k < 36; ++k) L[k] = 0.0;
  for (int j = 0; j < 6; ++j) {
    double d = N[6 * j + j];
    for (int k = 0; k < j; ++k) d -= L[6 * j + k] * L[6 * j + k];
    if (!(d > 0.0)) return false;
    L[6 * j + j] = sqrt(d);
    for (int i = j + 1; i < 6; ++i) {
      double v = N[6 * i + j];
      for (int k = 0; k < j; ++k) v -= L[6 * i + k] * L[6 * j + k];
      L[6 * i + j] = v / L[6 * j + j];
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= L[6 * i + k] * y[k];
    y[i] = v / L[6 * i + i];
  }
  for (int i = 5; i >= 0; --i) {
    double v = y[i];
    for (int k = i + 1; k < 6; ++k) v -= L[6 * k + i] * x[k];
    x[i] = v / L[6 * i + i];
  }
  return true;
}

// Refines (R, T) in place on n correspondences; w and e are scratch arrays of n doubles.
V3DM_HD void refine_pose(const PoseCorr* c, int n, const double* invK1, const double* invK2t, double thr, double* R,
                         double* T, double* w, double* e) {
  double lambda = 1e-3, JtJ[36], Jte[6], N[36], delta[6], Rs[9], Ts[3];
  bool computeDerivatives = true;
  for (int it = 0; it < 50; ++it) {
    const double err = pose_weighted_residual(c, n, R, T, invK1, invK2t, thr, w, e, true);
    if (computeDerivatives) pose_normal_equations(c, n, R, T, e, JtJ, Jte);
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
    if (!cholesky_solve6(N, Jte, delta)) return;
    double dl = 0.0;
    for (int k = 0; k < 6; ++k) dl += delta[k] * delta[k];
    dl = sqrt(dl);
    if (it >= 10 && dl < 1e-8 * (4.0 + 1e-8)) return;
    for (int k = 0; k < 9; ++k) Rs[k] = R[k];
    for (int k = 0; k < 3; ++k) Ts[k] = T[k];
    pose_update(Rs, Ts, delta, R, T);
    const double errNew = pose_weighted_residual(c, n, R, T, invK1, invK2t, thr, w, e, false);
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

}  // namespace ess
}  // namespace v3dm
