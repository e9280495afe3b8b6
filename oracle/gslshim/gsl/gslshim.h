// gslshim.h -- TEST INFRASTRUCTURE.  A minimal stand-in for the subset of the
// GNU GSL API that the freestream-milne reference calls, written for this
// project on top of the oracle's own numerics (../../fsm_numerics.h).  It lets
// the reference's unmodified sources compile here, where GSL is absent, so that
// the oracle restatement can be checked against the reference's own loops.
// Only the names and signatures follow GSL's public API; the numerics are this
// project's (natural-spline bicubic patches, Francis QR + inverse iteration).
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <new>

#include "../../fsm_numerics.h"

typedef struct {
  double dat[2];
} gsl_complex;
#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])

// ---------------------------------------------------------------- interp2d
typedef struct gsl_interp2d_type {
  const char* name;
} gsl_interp2d_type;
static const gsl_interp2d_type gslshim_bicubic_type = {"bicubic"};
static const gsl_interp2d_type* gsl_interp2d_bicubic = &gslshim_bicubic_type;

typedef struct gsl_interp_accel {
  size_t cache;  // unused: lookups are stateless, so sharing across threads is safe
} gsl_interp_accel;

typedef struct gsl_spline2d {
  fsm_num::Bicubic b;
} gsl_spline2d;

static inline gsl_spline2d* gsl_spline2d_alloc(const gsl_interp2d_type*, size_t, size_t) {
  return new gsl_spline2d();
}
static inline int gsl_spline2d_init(gsl_spline2d* s, const double xa[], const double ya[],
                                    const double za[], size_t nx, size_t ny) {
  s->b.init(xa, ya, za, nx, ny);
  return 0;
}
static inline double gsl_spline2d_eval(const gsl_spline2d* s, double x, double y,
                                       gsl_interp_accel*, gsl_interp_accel*) {
  if (x < s->b.x.front() || x > s->b.x.back() || y < s->b.y.front() || y > s->b.y.back()) {
    std::abort();  // GSL's default error handler aborts on a domain error
  }
  return s->b.eval(x, y);
}
static inline void gsl_spline2d_free(gsl_spline2d* s) { delete s; }
static inline gsl_interp_accel* gsl_interp_accel_alloc(void) { return new gsl_interp_accel(); }
static inline void gsl_interp_accel_free(gsl_interp_accel* a) { delete a; }

// ---------------------------------------------------------------- matrices
typedef struct gsl_matrix {
  size_t size1, size2;
  double* data;
} gsl_matrix;
typedef struct gsl_matrix_complex {
  size_t size1, size2;
  gsl_complex* data;
} gsl_matrix_complex;
typedef struct gsl_vector_complex {
  size_t size;
  gsl_complex* data;
} gsl_vector_complex;

static inline gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix* m = new gsl_matrix;
  m->size1 = n1;
  m->size2 = n2;
  m->data = new double[n1 * n2]();
  return m;
}
static inline void gsl_matrix_free(gsl_matrix* m) {
  delete[] m->data;
  delete m;
}
static inline void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x) {
  m->data[i * m->size2 + j] = x;
}
static inline int gsl_matrix_mul_elements(gsl_matrix* a, const gsl_matrix* b) {
  for (size_t k = 0; k < a->size1 * a->size2; ++k) a->data[k] *= b->data[k];
  return 0;
}
static inline gsl_matrix_complex* gsl_matrix_complex_alloc(size_t n1, size_t n2) {
  gsl_matrix_complex* m = new gsl_matrix_complex;
  m->size1 = n1;
  m->size2 = n2;
  m->data = new gsl_complex[n1 * n2]();
  return m;
}
static inline void gsl_matrix_complex_free(gsl_matrix_complex* m) {
  delete[] m->data;
  delete m;
}
static inline gsl_complex gsl_matrix_complex_get(const gsl_matrix_complex* m, size_t i, size_t j) {
  return m->data[i * m->size2 + j];
}
static inline gsl_vector_complex* gsl_vector_complex_alloc(size_t n) {
  gsl_vector_complex* v = new gsl_vector_complex;
  v->size = n;
  v->data = new gsl_complex[n]();
  return v;
}
static inline void gsl_vector_complex_free(gsl_vector_complex* v) {
  delete[] v->data;
  delete v;
}
static inline gsl_complex gsl_vector_complex_get(const gsl_vector_complex* v, size_t i) {
  return v->data[i];
}

// ---------------------------------------------------------------- eigen
typedef struct gsl_eigen_nonsymmv_workspace {
  size_t n;
} gsl_eigen_nonsymmv_workspace;
static inline gsl_eigen_nonsymmv_workspace* gsl_eigen_nonsymmv_alloc(size_t n) {
  gsl_eigen_nonsymmv_workspace* w = new gsl_eigen_nonsymmv_workspace;
  w->n = n;
  return w;
}
static inline void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace* w) { delete w; }
static inline int gsl_eigen_nonsymmv(gsl_matrix* A, gsl_vector_complex* eval,
                                     gsl_matrix_complex* evec, gsl_eigen_nonsymmv_workspace* w) {
  int n = (int)w->n;
  double wr[4], wi[4], vr[16];
  int rc = fsm_num::eig_nonsym(n, A->data, wr, wi, vr);
  for (int k = 0; k < n; ++k) {
    GSL_REAL(eval->data[k]) = wr[k];
    GSL_IMAG(eval->data[k]) = wi[k];
    for (int r = 0; r < n; ++r) {
      GSL_REAL(evec->data[r * n + k]) = vr[r * n + k];
      GSL_IMAG(evec->data[r * n + k]) = (wi[k] != 0.0) ? 1.0 : 0.0;  // complex pairs: marked non-real
    }
  }
  return rc;
}
