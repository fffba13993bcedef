/* Stand-in for the GNU Scientific Library pieces that the reference's
 * Glasma initialisation names (NEWEST5/ginit.h: gsl_integration_qag for the
 * nuclear thickness, gsl_eigen_nonsymmv in FindVar, gsl_blas_dgemm in
 * RotateTMuNu, complex vectors and matrices).  GSL is not installed in this
 * image; everything here is written from GSL's public manual, and the
 * numerical parts are ours:
 *
 *  - gsl_integration_qag: an adaptive quadrature to the requested relative
 *    tolerance.  GSL uses Gauss-Kronrod pairs; here every interval is
 *    integrated with 20-point Gauss-Legendre, whole and in halves, the
 *    difference is the interval's error estimate, and the interval with the
 *    largest estimate is bisected until the sum of estimates is within
 *    max(epsabs, epsrel |I|).  The result is the same integral to that
 *    tolerance (the reference asks for 1e-13).
 *  - gsl_eigen_nonsymmv: eigenvalues and eigenvectors of a real matrix,
 *    delegated to a callback that the harness installs (the tests give it
 *    LAPACK's dgeev through NumPy), and gsl_eigen_nonsymmv_sort by
 *    ascending modulus.  Real eigenvalues carry an exactly zero imaginary
 *    part and real eigenvectors, as in GSL.
 *
 * Test infrastructure for the oracle only.
 */
#ifndef VH_REF_SHIM_GSL_GINIT_H
#define VH_REF_SHIM_GSL_GINIT_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- matrices */
#ifndef VH_REF_SHIM_GSL_H /* gsl_multiroot_shim.h declares the same matrix */
typedef struct { size_t size1, size2; double* data; } gsl_matrix;
#endif
typedef struct { gsl_matrix matrix; } gsl_matrix_view;
static inline gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2) {
  gsl_matrix_view v;
  v.matrix.size1 = n1;
  v.matrix.size2 = n2;
  v.matrix.data = base;
  return v;
}

typedef enum { CblasNoTrans = 111, CblasTrans = 112 } CBLAS_TRANSPOSE_t;
/* C = alpha op(A) op(B) + beta C for square row-major matrices */
static inline int gsl_blas_dgemm(CBLAS_TRANSPOSE_t ta, CBLAS_TRANSPOSE_t tb, double alpha, const gsl_matrix* A,
                                 const gsl_matrix* B, double beta, gsl_matrix* C) {
  const size_t n = C->size1;
  double* out = (double*)calloc(n * n, sizeof(double));
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j < n; j++) {
      double s = 0;
      for (size_t k = 0; k < n; k++) {
        const double a = ta == CblasNoTrans ? A->data[i * n + k] : A->data[k * n + i];
        const double b = tb == CblasNoTrans ? B->data[k * n + j] : B->data[j * n + k];
        s += a * b;
      }
      out[i * n + j] = alpha * s + beta * C->data[i * n + j];
    }
  memcpy(C->data, out, n * n * sizeof(double));
  free(out);
  return 0;
}

/* ----------------------------------------------------------------- complex */
typedef struct { double dat[2]; } gsl_complex;
#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
static inline double gsl_complex_abs(gsl_complex z) { return hypot(z.dat[0], z.dat[1]); }

typedef struct { size_t size; double* data; } gsl_vector_complex;
typedef struct { size_t size1, size2; double* data; } gsl_matrix_complex;
static inline gsl_vector_complex* gsl_vector_complex_alloc(size_t n) {
  gsl_vector_complex* v = (gsl_vector_complex*)malloc(sizeof(gsl_vector_complex));
  v->size = n;
  v->data = (double*)calloc(2 * n, sizeof(double));
  return v;
}
static inline void gsl_vector_complex_free(gsl_vector_complex* v) { free(v->data); free(v); }
static inline gsl_complex gsl_vector_complex_get(const gsl_vector_complex* v, size_t i) {
  gsl_complex z;
  z.dat[0] = v->data[2 * i];
  z.dat[1] = v->data[2 * i + 1];
  return z;
}
static inline gsl_matrix_complex* gsl_matrix_complex_alloc(size_t n1, size_t n2) {
  gsl_matrix_complex* m = (gsl_matrix_complex*)malloc(sizeof(gsl_matrix_complex));
  m->size1 = n1;
  m->size2 = n2;
  m->data = (double*)calloc(2 * n1 * n2, sizeof(double));
  return m;
}
static inline void gsl_matrix_complex_free(gsl_matrix_complex* m) { free(m->data); free(m); }
static inline gsl_complex gsl_matrix_complex_get(const gsl_matrix_complex* m, size_t i, size_t j) {
  gsl_complex z;
  z.dat[0] = m->data[2 * (i * m->size2 + j)];
  z.dat[1] = m->data[2 * (i * m->size2 + j) + 1];
  return z;
}

/* ------------------------------------------------------------- eigensystem */
/* a16: the matrix row-major; wr, wi: eigenvalues; vr, vi: eigenvectors as
 * columns, row-major 4x4.  Returns 0 on success. */
typedef int (*vh_shim_eig_fn)(const double* a16, double* wr, double* wi, double* vr, double* vi);
static vh_shim_eig_fn vh_shim_eig = 0;

typedef struct { size_t n; } gsl_eigen_nonsymmv_workspace;
typedef enum { GSL_EIGEN_SORT_ABS_ASC = 2, GSL_EIGEN_SORT_ABS_DESC = 3 } gsl_eigen_sort_t;
static inline gsl_eigen_nonsymmv_workspace* gsl_eigen_nonsymmv_alloc(size_t n) {
  gsl_eigen_nonsymmv_workspace* w = (gsl_eigen_nonsymmv_workspace*)malloc(sizeof(gsl_eigen_nonsymmv_workspace));
  w->n = n;
  return w;
}
static inline void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace* w) { free(w); }
static inline int gsl_eigen_nonsymmv(gsl_matrix* A, gsl_vector_complex* eval, gsl_matrix_complex* evec,
                                     gsl_eigen_nonsymmv_workspace*) {
  double wr[4], wi[4], vr[16], vi[16];
  if (!vh_shim_eig || A->size1 != 4 || vh_shim_eig(A->data, wr, wi, vr, vi) != 0) abort();
  for (int i = 0; i < 4; i++) {
    eval->data[2 * i] = wr[i];
    eval->data[2 * i + 1] = wi[i];
    for (int j = 0; j < 4; j++) {
      evec->data[2 * (j * 4 + i)] = vr[j * 4 + i];
      evec->data[2 * (j * 4 + i) + 1] = vi[j * 4 + i];
    }
  }
  return 0;
}
/* stable insertion sort of the eigenpairs by modulus */
static inline int gsl_eigen_nonsymmv_sort(gsl_vector_complex* eval, gsl_matrix_complex* evec, gsl_eigen_sort_t t) {
  const size_t n = eval->size;
  for (size_t i = 1; i < n; i++)
    for (size_t j = i; j > 0; j--) {
      const double a = hypot(eval->data[2 * j - 2], eval->data[2 * j - 1]);
      const double b = hypot(eval->data[2 * j], eval->data[2 * j + 1]);
      const bool swap = t == GSL_EIGEN_SORT_ABS_ASC ? b < a : b > a;
      if (!swap) break;
      for (int c = 0; c < 2; c++) {
        const double s = eval->data[2 * j - 2 + c];
        eval->data[2 * j - 2 + c] = eval->data[2 * j + c];
        eval->data[2 * j + c] = s;
      }
      for (size_t r = 0; r < n; r++)
        for (int c = 0; c < 2; c++) {
          double* x = &evec->data[2 * (r * n + j - 1) + c];
          double* y = &evec->data[2 * (r * n + j) + c];
          const double s = *x;
          *x = *y;
          *y = s;
        }
    }
  return 0;
}

/* -------------------------------------------------------------- quadrature */
typedef struct {
  double (*function)(double x, void* params);
  void* params;
} gsl_function;
typedef struct { size_t limit; } gsl_integration_workspace;
#define GSL_INTEG_GAUSS61 6
static inline gsl_integration_workspace* gsl_integration_workspace_alloc(size_t n) {
  gsl_integration_workspace* w = (gsl_integration_workspace*)malloc(sizeof(gsl_integration_workspace));
  w->limit = n;
  return w;
}
static inline void gsl_integration_workspace_free(gsl_integration_workspace* w) { free(w); }

/* 20-point Gauss-Legendre nodes and weights on [-1, 1] by Newton's method on
 * the Legendre polynomial (three-term recurrence) */
static inline void vh_shim_gauss_legendre(double* x, double* w) {
  const int n = 20;
  for (int i = 0; i < n; i++) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1);
      const double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2 / ((1 - z * z) * dp * dp);
  }
}
static inline double vh_shim_gl(const gsl_function* f, double a, double b, const double* x, const double* w) {
  const double h = 0.5 * (b - a), m = 0.5 * (a + b);
  double s = 0;
  for (int i = 0; i < 20; i++) s += w[i] * f->function(m + h * x[i], f->params);
  return s * h;
}
/* one interval [l, r] into slot `at`: value from the two halves, error from
 * the difference with the whole */
static inline void vh_shim_piece(const gsl_function* f, double l, double r, size_t at, const double* x,
                                 const double* w, double* lo, double* hi, double* val, double* err) {
  const double m = 0.5 * (l + r);
  const double whole = vh_shim_gl(f, l, r, x, w);
  const double halves = vh_shim_gl(f, l, m, x, w) + vh_shim_gl(f, m, r, x, w);
  lo[at] = l;
  hi[at] = r;
  val[at] = halves;
  err[at] = fabs(halves - whole);
}
static inline int gsl_integration_qag(const gsl_function* f, double a, double b, double epsabs, double epsrel,
                                      size_t limit, int, gsl_integration_workspace*, double* result,
                                      double* abserr) {
  double x[20], w[20];
  vh_shim_gauss_legendre(x, w);
  size_t cap = limit < 2 ? 2 : limit;
  double* lo = (double*)malloc(cap * sizeof(double));
  double* hi = (double*)malloc(cap * sizeof(double));
  double* val = (double*)malloc(cap * sizeof(double));
  double* err = (double*)malloc(cap * sizeof(double));
  size_t n = 0;
  vh_shim_piece(f, a, b, n++, x, w, lo, hi, val, err);
  for (;;) {
    double tot = 0, etot = 0;
    size_t worst = 0;
    for (size_t i = 0; i < n; i++) {
      tot += val[i];
      etot += err[i];
      if (err[i] > err[worst]) worst = i;
    }
    const double tol = fmax(epsabs, epsrel * fabs(tot));
    if (etot <= tol || n >= cap) {
      *result = tot;
      *abserr = etot;
      break;
    }
    const double l = lo[worst], r = hi[worst], m = 0.5 * (l + r);
    vh_shim_piece(f, l, m, worst, x, w, lo, hi, val, err);
    vh_shim_piece(f, m, r, n++, x, w, lo, hi, val, err);
  }
  free(lo); free(hi); free(val); free(err);
  return 0;
}

#endif
