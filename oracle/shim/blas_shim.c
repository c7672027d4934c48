/*
 * Project-written level-1/level-2 BLAS routines with the Fortran ABI that the
 * reference declares in c/blas.h (dcopy_ :38, ddot_ :44, dasum_ :33,
 * daxpy_ :26, dscal_ :79, dgemv_ :131).
 *
 * TEST INFRASTRUCTURE ONLY: used to compile the unchanged reference C solvers
 * as the CPU parity oracle / CPU baseline.  Straight loops in BLAS reference
 * semantics (column-major dgemv, beta == 0 overwrites y without reading it).
 */
#include <math.h>
#include <stddef.h>

void dcopy_(int *n, double *x, int *incx, double *y, int *incy) {
  int N = *n, ix = *incx, iy = *incy;
  for (int i = 0; i < N; ++i) y[(size_t)i * iy] = x[(size_t)i * ix];
}

void dscal_(int *n, double *a, double *x, int *incx) {
  int N = *n, ix = *incx;
  double A = *a;
  for (int i = 0; i < N; ++i) x[(size_t)i * ix] *= A;
}

void daxpy_(int *n, double *alpha, double *x, int *incx, double *y, int *incy) {
  int N = *n, ix = *incx, iy = *incy;
  double a = *alpha;
  for (int i = 0; i < N; ++i) y[(size_t)i * iy] += a * x[(size_t)i * ix];
}

double ddot_(int *n, double *x, int *incx, double *y, int *incy) {
  int N = *n, ix = *incx, iy = *incy;
  double s = 0.0;
  for (int i = 0; i < N; ++i) s += x[(size_t)i * ix] * y[(size_t)i * iy];
  return s;
}

double dasum_(int *n, double *x, int *incx) {
  int N = *n, ix = *incx;
  double s = 0.0;
  for (int i = 0; i < N; ++i) s += fabs(x[(size_t)i * ix]);
  return s;
}

void dgemv_(char *trans, int *m, int *n, double *alpha, double *a, int *lda,
            double *x, int *incx, double *beta, double *y, int *incy) {
  int M = *m, N = *n, LDA = *lda, ix = *incx, iy = *incy;
  double al = *alpha, be = *beta;
  int t = (trans[0] == 'T' || trans[0] == 't' || trans[0] == 'C' || trans[0] == 'c');
  int ylen = t ? N : M;
  for (int i = 0; i < ylen; ++i) {
    if (be == 0.0) y[(size_t)i * iy] = 0.0;
    else if (be != 1.0) y[(size_t)i * iy] *= be;
  }
  if (!t) {
    for (int j = 0; j < N; ++j) {
      double tmp = al * x[(size_t)j * ix];
      const double *col = a + (size_t)j * LDA;
      for (int i = 0; i < M; ++i) y[(size_t)i * iy] += tmp * col[i];
    }
  } else {
    for (int j = 0; j < N; ++j) {
      const double *col = a + (size_t)j * LDA;
      double s = 0.0;
      for (int i = 0; i < M; ++i) s += col[i] * x[(size_t)i * ix];
      y[(size_t)j * iy] += al * s;
    }
  }
}
