// fsm_landau.cuh -- per-cell Landau matching, equation of state and viscous /
// baryon decomposition (replaces src/LandauMatch.cpp:145-392 and
// src/EquationOfState.cpp:5-80).  __host__ __device__ so the same algorithm can
// be unit-tested on the CPU; the product runs it only inside fsm_landau_kernel.
//
// Eigenproblem.  T^mu_nu u^nu = e u^mu with T^mu_nu = T^{mu a} g_{a nu},
// g = diag(1,-1,-1,-tau^2) (src/LandauMatch.cpp:197-214).  Because g T g is
// symmetric, T^mu_nu is self-adjoint in the Minkowski inner product, so the
// Rayleigh quotient  e(u) = (u.g.M.u)/(u.g.u)  is stationary at every
// eigenvector and Rayleigh-quotient iteration converges fast (cubically).
// The iteration starts from the energy-flux direction u0^mu = T^{mu tau}
// (timelike for any T^{mu nu} built from non-negative phase-space densities);
// each step solves (M - e I) y = u: in 3D by Gaussian elimination with partial
// pivoting (backward stable), for the 3 x 3 boost-invariant problem through
// the adjugate with FMA-exact 2 x 2 cofactors (no division, no pivoting), so
// strongly boosted cells (entries ~ gamma^2 e, eigenvalues ~ e) keep their
// accuracy either way.  The first steps run in FP32, the converging ones and
// the acceptance test in FP64.
//
// Acceptance mirrors src/LandauMatch.cpp:222-291: the eigenvalue must be real
// and positive, the eigenvector timelike and the boost factor u^tau below 100;
// otherwise e = 1e-3 and u = (1,0,0,0).  For a physical T^{mu nu} at most one
// eigenpair passes these tests, so which solver finds it does not matter.
#pragma once
#include <math.h>

#ifndef FSM_HD
#if defined(__CUDACC__)
#define FSM_HD __host__ __device__ __forceinline__
#else
#define FSM_HD inline
#endif
#endif

namespace fsm {

FSM_HD double fsm_rsqrt(double x) {
#if defined(__CUDA_ARCH__)
  return rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}
FSM_HD float fsm_rsqrt(float x) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}
template <typename R> FSM_HD R eps_of();
template <> FSM_HD double eps_of<double>() { return 2.220446049250313e-16; }
template <> FSM_HD float eps_of<float>() { return 1.1920929e-07f; }
template <typename R> FSM_HD R tiny_of();
template <> FSM_HD double tiny_of<double>() { return 1.0e-290; }
template <> FSM_HD float tiny_of<float>() { return 1.0e-36f; }

// Solve A y = b by Gaussian elimination with partial pivoting (backward
// stable).  Pivoting is a sequence of conditional row swaps with compile-time
// indices, so A stays in registers.  A pivot below eps*max|A| (the shift has
// hit the eigenvalue to rounding) is replaced by eps*max|A|, the usual inverse-
// iteration safeguard: y stays finite and only its direction is used.
template <typename R, int N>
FSM_HD void gepp_solve(R A[N][N], R b[N], R y[N]) {
  R amax = 0;
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) amax = fmax(amax, fabs(A[r][c]));
  const R tiny = fmax(eps_of<R>() * amax, tiny_of<R>());
  R inv[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int r = k + 1; r < N; ++r) {
      const bool sw = fabs(A[r][k]) > fabs(A[k][k]);
#pragma unroll
      for (int c = k; c < N; ++c) {
        const R a = A[k][c], z = A[r][c];
        A[k][c] = sw ? z : a;
        A[r][c] = sw ? a : z;
      }
      const R a = b[k], z = b[r];
      b[k] = sw ? z : a;
      b[r] = sw ? a : z;
    }
    R piv = A[k][k];
    if (fabs(piv) < tiny) piv = (piv < 0) ? -tiny : tiny;
    inv[k] = R(1) / piv;
#pragma unroll
    for (int r = k + 1; r < N; ++r) {
      const R f = A[r][k] * inv[k];
#pragma unroll
      for (int c = k + 1; c < N; ++c) A[r][c] -= f * A[k][c];
      b[r] -= f * b[k];
    }
  }
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    R s = b[k];
#pragma unroll
    for (int c = k + 1; c < N; ++c) s -= A[k][c] * y[c];
    y[k] = s * inv[k];
  }
}

// a*d - b*c with one rounding error on the result (Kahan's algorithm): the
// error of w = b*c is recovered exactly by an FMA, so the cancellation of the
// two products (large for the minors of strongly boosted cells) costs nothing.
FSM_HD double det2(double a, double b, double c, double d) {
  const double w = b * c;
  const double e = fma(-b, c, w);
  const double f = fma(a, d, -w);
  return f + e;
}
FSM_HD float det2(float a, float b, float c, float d) { return a * d - b * c; }

// y = adj(A) b = det(A) A^-1 b for 3 x 3 A: the direction an inverse-
// iteration step needs, without division or pivoting.  The cofactors are 2 x 2
// determinants (det2); near an eigenvalue adj(A) is the outer product of the
// right and left null vectors, so y keeps its direction to rounding level.
template <typename R>
FSM_HD void adj_solve3(const R A[3][3], const R b[3], R y[3]) {
  const R c00 = det2(A[1][1], A[1][2], A[2][1], A[2][2]);
  const R c01 = det2(A[1][2], A[1][0], A[2][2], A[2][0]);
  const R c02 = det2(A[1][0], A[1][1], A[2][0], A[2][1]);
  const R c10 = det2(A[0][2], A[0][1], A[2][2], A[2][1]);
  const R c11 = det2(A[0][0], A[0][2], A[2][0], A[2][2]);
  const R c12 = det2(A[0][1], A[0][0], A[2][1], A[2][0]);
  const R c20 = det2(A[0][1], A[0][2], A[1][1], A[1][2]);
  const R c21 = det2(A[0][2], A[0][0], A[1][2], A[1][0]);
  const R c22 = det2(A[0][0], A[0][1], A[1][0], A[1][1]);
  y[0] = c00 * b[0] + c10 * b[1] + c20 * b[2];
  y[1] = c01 * b[0] + c11 * b[1] + c21 * b[2];
  y[2] = c02 * b[0] + c12 * b[1] + c22 * b[2];
}

template <typename R, int N>
FSM_HD R mink_norm2(const R g[N], const R u[N]) {
  R s = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) s += g[r] * u[r] * u[r];
  return s;
}

template <typename R, int N>
FSM_HD R rayleigh(const R M[N][N], const R g[N], const R u[N]) {
  R num = 0, den = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    R mu = 0;
#pragma unroll
    for (int c = 0; c < N; ++c) mu += M[r][c] * u[c];
    num += g[r] * u[r] * mu;
    den += g[r] * u[r] * u[r];
  }
  return num / den;
}

// Rayleigh quotient of a vector already normalised to u.g.u = 1.
template <typename R, int N>
FSM_HD R rayleigh_unit(const R M[N][N], const R g[N], const R u[N]) {
  R num = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    R mu = 0;
#pragma unroll
    for (int c = 0; c < N; ++c) mu += M[r][c] * u[c];
    num += g[r] * u[r] * mu;
  }
  return num;
}

// One Rayleigh-quotient-iteration step: u <- (M - e)^-1 u, normalised to
// u.g.u = 1 with u^tau > 0, and e <- its Rayleigh quotient.  False when the
// step leaves the light cone or is not finite.
template <typename R, int N>
FSM_HD bool rqi_step(const R M[N][N], const R g[N], R u[N], R& e) {
  R A[N][N], rhs[N], y[N];
#pragma unroll
  for (int r = 0; r < N; ++r) {
    rhs[r] = u[r];
#pragma unroll
    for (int c = 0; c < N; ++c) A[r][c] = M[r][c] - (r == c ? e : R(0));
  }
  if constexpr (N == 3) adj_solve3<R>(A, rhs, y);
  else gepp_solve<R, N>(A, rhs, y);
  const R m2 = mink_norm2<R, N>(g, y);
  if (!(m2 > 0) || !isfinite(m2)) return false;
  R t = fsm_rsqrt(m2);
  if (y[0] < 0) t = -t;
#pragma unroll
  for (int r = 0; r < N; ++r) u[r] = y[r] * t;
  e = rayleigh_unit<R, N>(M, g, u);
  return true;
}

// max |M u - e u| and the scales max|M|, max|u| of a candidate eigenpair.
template <int N>
FSM_HD void eigen_residual(const double M[N][N], const double u[N], double e, double* rmax,
                           double* mmax, double* umax) {
  double rr = 0.0, mm = 0.0, uu = 0.0;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    double mu = 0.0;
#pragma unroll
    for (int c = 0; c < N; ++c) {
      mu += M[r][c] * u[c];
      mm = fmax(mm, fabs(M[r][c]));
    }
    rr = fmax(rr, fabs(mu - e * u[r]));
    uu = fmax(uu, fabs(u[r]));
  }
  *rmax = rr;
  *mmax = mm;
  *umax = uu;
}

// Timelike eigenpair of M (N = 3 for boost-invariant 2D events, whose eta row
// and column vanish identically; N = 4 in 3D).  Returns 1 and (e, u) with
// u.g.u = 1, u^tau > 0 when an acceptable pair was found.  Two FP32 RQI
// steps from the energy-flux direction bring u close to single precision (RQI
// converges cubically); FP64 steps then run until the eigen-residual is at
// rounding level, normally after one.
template <int N>
FSM_HD int landau_eigen(const double M[N][N], const double g[N], double* e_out, double u_out[N]) {
  double u[N];
  {
    float Mf[N][N], gf[N], uf[N];
#pragma unroll
    for (int r = 0; r < N; ++r) {
      gf[r] = (float)g[r];
      uf[r] = (float)M[r][0];
#pragma unroll
      for (int c = 0; c < N; ++c) Mf[r][c] = (float)M[r][c];
    }
    float n2 = mink_norm2<float, N>(gf, uf);
    bool ok = (n2 > 0.0f) && isfinite(n2);
    if (ok) {
      float s = fsm_rsqrt(n2);
      if (uf[0] < 0.0f) s = -s;
#pragma unroll
      for (int r = 0; r < N; ++r) uf[r] *= s;
      float ef = rayleigh<float, N>(Mf, gf, uf);
      float keep[N];
#pragma unroll
      for (int r = 0; r < N; ++r) keep[r] = uf[r];
      for (int it = 0; it < 2; ++it) {
        if (!rqi_step<float, N>(Mf, gf, uf, ef) || !isfinite(ef)) {
#pragma unroll
          for (int r = 0; r < N; ++r) uf[r] = keep[r];
          break;
        }
#pragma unroll
        for (int r = 0; r < N; ++r) keep[r] = uf[r];
      }
    }
#pragma unroll
    for (int r = 0; r < N; ++r) u[r] = ok ? (double)uf[r] : (double)M[r][0];
  }
  double n2 = mink_norm2<double, N>(g, u);
  if (!(n2 > 0.0) || !isfinite(n2)) {
#pragma unroll
    for (int r = 0; r < N; ++r) u[r] = (r == 0) ? 1.0 : 0.0;
    n2 = 1.0;
  }
  double s = fsm_rsqrt(n2);
  if (u[0] < 0.0) s = -s;
#pragma unroll
  for (int r = 0; r < N; ++r) u[r] *= s;
  double e = rayleigh_unit<double, N>(M, g, u);  // u.g.u = 1 up to rounding
  double rmax = 0.0, mmax = 0.0, umax = 0.0;
  bool have = false;  // the residual of the current (e, u) is at hand
  for (int it = 0; it < 12; ++it) {
    if (!rqi_step<double, N>(M, g, u, e)) break;  // a failed step leaves (e, u) unchanged
    eigen_residual<N>(M, u, e, &rmax, &mmax, &umax);
    have = true;
    if (rmax <= 1.0e-13 * mmax * umax) break;
  }
  // acceptance: a converged pair has |M u - e u| at rounding level
  if (!have) eigen_residual<N>(M, u, e, &rmax, &mmax, &umax);
  if (!(isfinite(e) && (rmax <= 1.0e-9 * mmax * umax) && (e > 0.0))) return 0;
  *e_out = e;
#pragma unroll
  for (int r = 0; r < N; ++r) u_out[r] = u[r];
  return 1;
}

// The reference's normalisation and acceptance tests on the eigenvector
// (src/LandauMatch.cpp:235-243): with v the unit-Euclidean-norm eigenvector,
// timelike iff 2 v0^2 - 1 - v3^2 (tau^2 - 1) > 0 and u = v / sqrt(v0^2 -
// (v1^2 + v2^2 + tau^2 v3^2)), where tau^2 is the float product TAU*TAU (the
// index itself was lowered with the double product).  Accept iff u^tau < 100.
// Both tests and u are invariant under a positive rescaling of v, so they are
// evaluated on w itself (multiplied through by |w|^2) without normalising it.
FSM_HD int reference_normalise(const double w[4], float TAU, double u[4]) {
  const double n2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
  if (!(n2 > 0.0)) return 0;
  const float tt = TAU * TAU;  // float product, as the reference
  if (!((2.0 * w[0] * w[0] - n2 - (w[3] * w[3] * (tt - 1.0))) > 0)) return 0;
  const double mink = w[0] * w[0] - (w[1] * w[1] + w[2] * w[2] + tt * w[3] * w[3]);
  double factor = fsm_rsqrt(mink);
  if (w[0] < 0) factor = -factor;
  if (!((w[0] * factor) < 100.0)) return 0;
  u[0] = w[0] * factor;
  u[1] = w[1] * factor;
  u[2] = w[2] * factor;
  u[3] = w[3] * factor;
  return 1;
}

// Pressure from the float energy density exactly as src/EquationOfState.cpp:5-80.
FSM_HD float eos_pressure(float e, int eos) {
  if (eos == 1) return (float)((double)e / 3.0);
  if (eos == 2) {
    const float a0 = -0.25181736420168666f, a1 = 9737.845799644809f, a2 = 1.077580993288114e6f,
                a3 = 3.1729694865420084e6f, a4 = 1.6357487344679043e6f, a5 = 334334.4309240126f,
                a6 = 41913.439282708554f, a7 = 6340.448389300905f, a8 = 141.5073484468774f,
                a9 = 0.7158279081255019f, a10 = 0.0009417586777847889f,
                a11 = 3.1188455176941583e-7f, a12 = 1.9531729608963267e-11f;
    const float b0 = 45829.44617893836f, b1 = 4.0574329080826794e6f, b2 = 2.0931169138134286e7f,
                b3 = 1.3512402226067686e7f, b4 = 1.7851642641834426e6f, b5 = 278581.2989342773f,
                b6 = 26452.34905933697f, b7 = 499.04919730607065f, b8 = 2.3405487982094204f,
                b9 = 0.002962497695527404f, b10 = 9.601103399348206e-7f,
                b11 = 5.928138360995685e-11f, b12 = 3.2581066229887368e-18f;
    float e1 = e, e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e,
          e8 = e7 * e, e9 = e8 * e, e10 = e9 * e, e11 = e10 * e, e12 = e11 * e;
    float a = fmaf(a12, e12, fmaf(a11, e11, fmaf(a10, e10, fmaf(a9, e9, fmaf(a8, e8, fmaf(a7, e7,
              fmaf(a6, e6, fmaf(a5, e5, fmaf(a4, e4, fmaf(a3, e3, fmaf(a2, e2, fmaf(a1, e1, a0))))))))))));
    float b = fmaf(b12, e12, fmaf(b11, e11, fmaf(b10, e10, fmaf(b9, e9, fmaf(b8, e8, fmaf(b7, e7,
              fmaf(b6, e6, fmaf(b5, e5, fmaf(b4, e4, fmaf(b3, e3, fmaf(b2, e2, fmaf(b1, e1, b0))))))))))));
    return a / b;
  }
  return 0.0f;  // EOS_TYPE 3: the reference's placeholder (src/EquationOfState.cpp:72-79)
}

struct CellOut {
  float e, P, Pi, u[4], pi[10], nB, V[4];
  int fallback;
};

// One cell: eigen-solve, EoS, bulk/shear (src/LandauMatch.cpp:332-367) and
// baryon density/diffusion (src/LandauMatch.cpp:370-392).  T components in
// the reference's row order; decomposition in FP64 from the float e, P, u.
template <bool k3D>
FSM_HD void landau_cell_t(const float T[10], const float J[4], int baryon, int eos, int viscous,
                          float TAU, CellOut* o) {
  double tau2 = (double)TAU * (double)TAU;
  double e = 0.0, u[4] = {0.0, 0.0, 0.0, 0.0};
  int ok;
  if constexpr (k3D) {
    double M[4][4];
    const int idx[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double gc = (c == 0) ? 1.0 : (c == 3 ? -tau2 : -1.0);
        M[r][c] = (double)T[idx[r][c]] * gc;
      }
    const double g[4] = {1.0, -1.0, -1.0, -tau2};
    double w[4];
    ok = landau_eigen<4>(M, g, &e, w) && reference_normalise(w, TAU, u);
  } else {
    double M[3][3];
    const int idx[3][3] = {{0, 1, 2}, {1, 4, 5}, {2, 5, 7}};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) M[r][c] = (double)T[idx[r][c]] * (c == 0 ? 1.0 : -1.0);
    const double g[3] = {1.0, -1.0, -1.0};
    double u3[3];
    ok = landau_eigen<3>(M, g, &e, u3);
    const double w[4] = {u3[0], u3[1], u3[2], 0.0};
    ok = ok && reference_normalise(w, TAU, u);
  }
  if (ok) {
    o->e = (float)e;
#pragma unroll
    for (int r = 0; r < 4; ++r) o->u[r] = (float)u[r];
    o->fallback = 0;
  } else {  // (src/LandauMatch.cpp:283-291)
    o->e = 1.0e-3f;
    o->u[0] = 1.0f;
    o->u[1] = o->u[2] = o->u[3] = 0.0f;
    o->fallback = 1;
  }
  o->P = eos_pressure(o->e, eos);
  double ed = o->e, Pd = o->P;
  double ud[4] = {o->u[0], o->u[1], o->u[2], o->u[3]};
  if (viscous) {
    double a = (double)T[0] - (double)T[4] - (double)T[7] - tau2 * (double)T[9];
    double Pi = (-1.0 / 3.0) * (a - ed) - Pd;
    double b = ed + Pd + Pi, c = Pd + Pi;
    o->Pi = (float)Pi;
    o->pi[0] = (float)((double)T[0] - ud[0] * ud[0] * b + c);
    o->pi[1] = (float)((double)T[1] - ud[0] * ud[1] * b);
    o->pi[2] = (float)((double)T[2] - ud[0] * ud[2] * b);
    o->pi[3] = (float)((double)T[3] - ud[0] * ud[3] * b);
    o->pi[4] = (float)((double)T[4] - ud[1] * ud[1] * b - c);
    o->pi[5] = (float)((double)T[5] - ud[1] * ud[2] * b);
    o->pi[6] = (float)((double)T[6] - ud[1] * ud[3] * b);
    o->pi[7] = (float)((double)T[7] - ud[2] * ud[2] * b - c);
    o->pi[8] = (float)((double)T[8] - ud[2] * ud[3] * b);
    o->pi[9] = (float)((double)T[9] - ud[3] * ud[3] * b - c / tau2);
  } else {
    o->Pi = 0.0f;
#pragma unroll
    for (int k = 0; k < 10; ++k) o->pi[k] = 0.0f;
  }
  if (baryon) {
    double nB = ud[0] * J[0] - ud[1] * J[1] - ud[2] * J[2] - tau2 * ud[3] * J[3];
    o->nB = (float)nB;
#pragma unroll
    for (int r = 0; r < 4; ++r) o->V[r] = (float)((double)J[r] - nB * ud[r]);
  } else {
    o->nB = 0.0f;
#pragma unroll
    for (int r = 0; r < 4; ++r) o->V[r] = 0.0f;
  }
}

// Either dimension (the device kernels instantiate each separately, so that
// each is register-allocated for its own eigenproblem).
FSM_HD void landau_cell(const float T[10], const float J[4], int is3d, int baryon, int eos,
                        int viscous, float TAU, CellOut* o) {
  if (is3d)
    landau_cell_t<true>(T, J, baryon, eos, viscous, TAU, o);
  else
    landau_cell_t<false>(T, J, baryon, eos, viscous, TAU, o);
}

}  // namespace fsm
