// fsm_numerics.h -- TEST INFRASTRUCTURE (CPU oracle only; never linked into the product).
//
// Double-precision numerical kernels that stand in for the two places where the
// freestream-milne reference calls GNU GSL:
//
//   * the 2D bicubic spline  (src/FreeStream.cpp:123-153 `gsl_spline2d_*` with
//     `gsl_interp2d_bicubic`, evaluated at src/FreeStream.cpp:240), and
//   * the real nonsymmetric 4x4 eigensolver (src/LandauMatch.cpp:215-218
//     `gsl_eigen_nonsymmv`).
//
// GSL is not available on this machine, so both are written here from the
// mathematics, not from GSL sources:
//
//   Bicubic spline.  Node derivatives come from 1D natural cubic splines
//   (second derivative zero at both ends): z_x along x for every grid row, z_y
//   along y for every grid column, and z_xy as the natural-spline x-derivative of
//   the z_y field.  (The mixed derivative is the tensor product of two linear
//   operators, so the x-then-y and y-then-x orders agree up to rounding.)  Each
//   cell is then the bicubic Hermite patch that matches z, z_x, z_y, z_xy at its
//   four corners.  The natural spline second derivatives solve the standard
//   tridiagonal system  h[i-1] M[i-1] + 2 (h[i-1]+h[i]) M[i] + h[i] M[i+1]
//   = 6 (d[i] - d[i-1]),  d[i] = (y[i+1]-y[i]) / h[i],  M[0] = M[n-1] = 0,
//   solved by Gaussian elimination without pivoting (the matrix is strictly
//   diagonally dominant).
//
//   Eigensolver.  Householder reduction to upper Hessenberg form followed by the
//   implicitly double-shifted Francis QR iteration (Golub & Van Loan, Matrix
//   Computations, 4th ed., Alg. 7.4.2 and 7.5.1-7.5.2) gives the eigenvalues;
//   2x2 diagonal blocks with a non-negative discriminant split into two real
//   eigenvalues with exactly zero imaginary part, otherwise into a complex pair.
//   The eigenvector of each real eigenvalue comes from inverse iteration on the
//   original matrix and is scaled to unit Euclidean norm (the normalisation the
//   reference's timelike test at src/LandauMatch.cpp:235 relies on).
#pragma once
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

namespace fsm_num {

// ---------------------------------------------------------------- 1D spline
// Derivative of the natural cubic spline through (x[i], y[i]) at every node.
// stride_y / stride_d allow walking rows or columns of a 2D array in place.
inline void natural_spline_node_derivs(const double* x, const double* y, size_t stride_y,
                                       size_t n, double* d, size_t stride_d) {
  if (n < 2) {
    if (n == 1) d[0] = 0.0;
    return;
  }
  std::vector<double> h(n - 1), sl(n - 1), M(n, 0.0);
  for (size_t i = 0; i + 1 < n; ++i) {
    h[i] = x[i + 1] - x[i];
    sl[i] = (y[(i + 1) * stride_y] - y[i * stride_y]) / h[i];
  }
  if (n > 2) {
    // unknowns M[1..n-2]; forward elimination then back substitution
    size_t m = n - 2;
    std::vector<double> diag(m), rhs(m);
    for (size_t k = 0; k < m; ++k) {
      size_t i = k + 1;
      diag[k] = 2.0 * (h[i - 1] + h[i]);
      rhs[k] = 6.0 * (sl[i] - sl[i - 1]);
    }
    for (size_t k = 1; k < m; ++k) {
      double f = h[k] / diag[k - 1];  // sub-diagonal entry of row k is h[k]
      diag[k] -= f * h[k];            // super-diagonal entry of row k-1 is h[k]
      rhs[k] -= f * rhs[k - 1];
    }
    M[m] = rhs[m - 1] / diag[m - 1];
    for (size_t k = m - 1; k-- > 0;) M[k + 1] = (rhs[k] - h[k + 1] * M[k + 2]) / diag[k];
  }
  for (size_t i = 0; i + 1 < n; ++i)
    d[i * stride_d] = sl[i] - h[i] * (2.0 * M[i] + M[i + 1]) / 6.0;
  d[(n - 1) * stride_d] = sl[n - 2] + h[n - 2] * (M[n - 2] + 2.0 * M[n - 1]) / 6.0;
}

// ---------------------------------------------------------------- 2D spline
// Node data for a bicubic spline on a rectilinear grid.  Array layout follows
// the reference's call (src/FreeStream.cpp:137): z[i + j*nx] = f(x[i], y[j]).
struct Bicubic {
  size_t nx = 0, ny = 0;
  std::vector<double> x, y, z, zx, zy, zxy;

  void init(const double* xa, const double* ya, const double* za, size_t nx_, size_t ny_) {
    nx = nx_;
    ny = ny_;
    x.assign(xa, xa + nx);
    y.assign(ya, ya + ny);
    z.assign(za, za + nx * ny);
    zx.assign(nx * ny, 0.0);
    zy.assign(nx * ny, 0.0);
    zxy.assign(nx * ny, 0.0);
    for (size_t j = 0; j < ny; ++j)
      natural_spline_node_derivs(x.data(), &z[j * nx], 1, nx, &zx[j * nx], 1);
    for (size_t i = 0; i < nx; ++i)
      natural_spline_node_derivs(y.data(), &z[i], nx, ny, &zy[i], nx);
    for (size_t j = 0; j < ny; ++j)
      natural_spline_node_derivs(x.data(), &zy[j * nx], 1, nx, &zxy[j * nx], 1);
  }

  // index i with a[i] <= v < a[i+1]; v == a[n-1] maps to n-2 (bisection)
  static size_t locate(const std::vector<double>& a, double v) {
    size_t lo = 0, hi = a.size() - 1;
    while (hi > lo + 1) {
      size_t mid = (lo + hi) / 2;
      if (a[mid] > v) hi = mid;
      else lo = mid;
    }
    return lo;
  }

  // Bicubic Hermite patch evaluation; caller guarantees x, y inside the grid.
  double eval(double xv, double yv) const {
    size_t i = locate(x, xv), j = locate(y, yv);
    double dx = x[i + 1] - x[i], dy = y[j + 1] - y[j];
    double t = (xv - x[i]) / dx, u = (yv - y[j]) / dy;
    double t2 = t * t, t3 = t2 * t, u2 = u * u, u3 = u2 * u;
    double H[2] = {1.0 - 3.0 * t2 + 2.0 * t3, 3.0 * t2 - 2.0 * t3};
    double G[2] = {t - 2.0 * t2 + t3, t3 - t2};
    double Hu[2] = {1.0 - 3.0 * u2 + 2.0 * u3, 3.0 * u2 - 2.0 * u3};
    double Gu[2] = {u - 2.0 * u2 + u3, u3 - u2};
    double r = 0.0;
    for (int b = 0; b < 2; ++b)
      for (int a = 0; a < 2; ++a) {
        size_t k = (i + a) + (j + b) * nx;
        r += z[k] * H[a] * Hu[b] + zx[k] * dx * G[a] * Hu[b] + zy[k] * dy * H[a] * Gu[b] +
             zxy[k] * dx * dy * G[a] * Gu[b];
      }
    return r;
  }
};

// ---------------------------------------------------------------- eigen
// Real nonsymmetric n x n (n <= 4) eigen-decomposition.  wr/wi receive the
// eigenvalues; for every real eigenvalue (wi == 0) the matching column of
// vr holds a unit-Euclidean-norm eigenvector, complex ones get zero columns.
// Returns 0 on success, -1 if the QR iteration did not converge.
inline int eig_nonsym(int n, const double* A /* row-major n*n */, double* wr, double* wi,
                      double* vr /* row-major n*n, column k = eigenvector k */) {
  double H[4][4];
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) H[r][c] = A[r * n + c];
  double anorm = 0.0;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) anorm += std::fabs(H[r][c]);

  // Householder reduction to upper Hessenberg form.
  for (int k = 0; k + 2 < n; ++k) {
    double alpha = 0.0;
    for (int r = k + 1; r < n; ++r) alpha += H[r][k] * H[r][k];
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) continue;
    if (H[k + 1][k] > 0) alpha = -alpha;
    double v[4] = {0, 0, 0, 0};
    for (int r = k + 1; r < n; ++r) v[r] = H[r][k];
    v[k + 1] -= alpha;
    double vv = 0.0;
    for (int r = k + 1; r < n; ++r) vv += v[r] * v[r];
    if (vv == 0.0) continue;
    // H <- P H P with P = I - 2 v v^T / (v^T v)
    for (int c = 0; c < n; ++c) {
      double s = 0.0;
      for (int r = k + 1; r < n; ++r) s += v[r] * H[r][c];
      s = 2.0 * s / vv;
      for (int r = k + 1; r < n; ++r) H[r][c] -= s * v[r];
    }
    for (int r = 0; r < n; ++r) {
      double s = 0.0;
      for (int c = k + 1; c < n; ++c) s += H[r][c] * v[c];
      s = 2.0 * s / vv;
      for (int c = k + 1; c < n; ++c) H[r][c] -= s * v[c];
    }
    for (int r = k + 2; r < n; ++r) H[r][k] = 0.0;
  }

  // Francis double-shift QR on the active window [lo, hi].
  const double eps = 2.220446049250313e-16;
  int hi = n - 1, its = 0, total_its = 0;
  while (hi >= 0) {
    int l = hi;
    for (; l > 0; --l) {
      double s = std::fabs(H[l - 1][l - 1]) + std::fabs(H[l][l]);
      if (s == 0.0) s = anorm;
      if (std::fabs(H[l][l - 1]) <= eps * s) {
        H[l][l - 1] = 0.0;
        break;
      }
    }
    if (l == hi) {
      wr[hi] = H[hi][hi];
      wi[hi] = 0.0;
      --hi;
      its = 0;
      continue;
    }
    if (l == hi - 1) {
      double a = H[hi - 1][hi - 1], b = H[hi - 1][hi], c = H[hi][hi - 1], d = H[hi][hi];
      double p = 0.5 * (a - d), q = p * p + b * c;
      if (q >= 0.0) {
        double zz = p + (p >= 0 ? std::sqrt(q) : -std::sqrt(q));
        double l1 = d + zz;
        double l2 = (zz != 0.0) ? d - b * c / zz : d + zz;
        wr[hi - 1] = l1;
        wr[hi] = l2;
        wi[hi - 1] = wi[hi] = 0.0;
      } else {
        double im = std::sqrt(-q);
        wr[hi - 1] = wr[hi] = d + p;
        wi[hi - 1] = im;
        wi[hi] = -im;
      }
      hi -= 2;
      its = 0;
      continue;
    }
    if (++total_its > 120) return -1;
    ++its;
    double s, t;
    if (its == 10 || its == 20) {  // exceptional shift
      double e = std::fabs(H[hi][hi - 1]) + std::fabs(H[hi - 1][hi - 2]);
      s = 1.5 * e;
      t = e * e;
    } else {
      s = H[hi - 1][hi - 1] + H[hi][hi];
      t = H[hi - 1][hi - 1] * H[hi][hi] - H[hi - 1][hi] * H[hi][hi - 1];
    }
    double x = H[l][l] * H[l][l] + H[l][l + 1] * H[l + 1][l] - s * H[l][l] + t;
    double y = H[l + 1][l] * (H[l][l] + H[l + 1][l + 1] - s);
    double zq = H[l + 1][l] * H[l + 2][l + 1];
    for (int k = l; k <= hi - 2; ++k) {
      // Householder reflector mapping (x, y, zq) onto a multiple of e1
      double nrm = std::sqrt(x * x + y * y + zq * zq);
      if (nrm != 0.0) {
        double al = (x > 0) ? -nrm : nrm;
        double v0 = x - al, v1 = y, v2 = zq;
        double vv = v0 * v0 + v1 * v1 + v2 * v2;
        if (vv != 0.0) {
          int c0 = (k > l) ? k - 1 : l;
          for (int c = c0; c <= hi; ++c) {
            double sm = 2.0 * (v0 * H[k][c] + v1 * H[k + 1][c] + v2 * H[k + 2][c]) / vv;
            H[k][c] -= sm * v0;
            H[k + 1][c] -= sm * v1;
            H[k + 2][c] -= sm * v2;
          }
          int r1 = (k + 3 < hi) ? k + 3 : hi;
          for (int r = l; r <= r1; ++r) {
            double sm = 2.0 * (H[r][k] * v0 + H[r][k + 1] * v1 + H[r][k + 2] * v2) / vv;
            H[r][k] -= sm * v0;
            H[r][k + 1] -= sm * v1;
            H[r][k + 2] -= sm * v2;
          }
        }
      }
      x = H[k + 1][k];
      y = H[k + 2][k];
      if (k < hi - 2) zq = H[k + 3][k];
    }
    // final 2-element reflector on rows/cols hi-1, hi
    {
      int k = hi - 1;
      double nrm = std::sqrt(x * x + y * y);
      if (nrm != 0.0) {
        double al = (x > 0) ? -nrm : nrm;
        double v0 = x - al, v1 = y;
        double vv = v0 * v0 + v1 * v1;
        if (vv != 0.0) {
          for (int c = k - 1; c <= hi; ++c) {
            double sm = 2.0 * (v0 * H[k][c] + v1 * H[k + 1][c]) / vv;
            H[k][c] -= sm * v0;
            H[k + 1][c] -= sm * v1;
          }
          for (int r = l; r <= hi; ++r) {
            double sm = 2.0 * (H[r][k] * v0 + H[r][k + 1] * v1) / vv;
            H[r][k] -= sm * v0;
            H[r][k + 1] -= sm * v1;
          }
        }
      }
    }
    // clean the sub-sub-diagonal the bulge chase leaves at rounding level
    for (int r = l + 2; r <= hi && r < 4; ++r)
      for (int c = l; c < r - 1 && c < 4; ++c) H[r][c] = 0.0;
  }

  // Eigenvectors of real eigenvalues by inverse iteration on the original matrix.
  for (int k = 0; k < n * n; ++k) vr[k] = 0.0;
  for (int e = 0; e < n; ++e) {
    if (wi[e] != 0.0) continue;
    double lam = wr[e];
    double pert = eps * (anorm > 0 ? anorm : 1.0) * 16.0;
    double LU[4][4];
    int piv[4];
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) LU[r][c] = A[r * n + c] - (r == c ? lam + pert : 0.0);
    // LU with partial pivoting; zero pivots replaced by a tiny value
    for (int k = 0; k < n; ++k) {
      int p = k;
      for (int r = k + 1; r < n; ++r)
        if (std::fabs(LU[r][k]) > std::fabs(LU[p][k])) p = r;
      piv[k] = p;
      if (p != k)
        for (int c = 0; c < n; ++c) std::swap(LU[k][c], LU[p][c]);
      if (LU[k][k] == 0.0) LU[k][k] = pert;
      for (int r = k + 1; r < n; ++r) {
        double f = LU[r][k] / LU[k][k];
        LU[r][k] = f;
        for (int c = k + 1; c < n; ++c) LU[r][c] -= f * LU[k][c];
      }
    }
    double v[4] = {1.0, 0.7548776662466927, 0.5698402909980532, 0.4301597090019468};
    for (int it = 0; it < 3; ++it) {
      double b[4];
      for (int r = 0; r < n; ++r) b[r] = v[r];
      for (int k = 0; k < n; ++k) std::swap(b[k], b[piv[k]]);
      for (int r = 1; r < n; ++r)
        for (int c = 0; c < r; ++c) b[r] -= LU[r][c] * b[c];
      for (int r = n - 1; r >= 0; --r) {
        for (int c = r + 1; c < n; ++c) b[r] -= LU[r][c] * b[c];
        b[r] /= LU[r][r];
      }
      double nr = 0.0;
      for (int r = 0; r < n; ++r) nr += b[r] * b[r];
      nr = std::sqrt(nr);
      if (!(nr > 0.0) || !std::isfinite(nr)) break;
      for (int r = 0; r < n; ++r) v[r] = b[r] / nr;
    }
    for (int r = 0; r < n; ++r) vr[r * n + e] = v[r];
  }
  return 0;
}

}  // namespace fsm_num
