/*
 * Project-written dsyrk_ (c/blas.h:107) and dposv_ (c/lapack.h:3) with the
 * Fortran ABI, for compiling the reference's leave-one-out error code
 * (c/looe_lib.c) as a CPU parity oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Straight loops in the routines' documented
 * semantics, column-major storage:
 *   dsyrk_  C := alpha op(A) op(A)^T + beta C on the `uplo` triangle
 *           (trans 'T': op(A) = A^T, A is k x n; 'N': A is n x k);
 *   dposv_  Cholesky A = L L^T ('L') or U^T U ('U') of the n x n matrix,
 *           then B := A^{-1} B for nrhs columns; info = j > 0 when the
 *           leading minor of order j is not positive definite (B untouched).
 */
#include <math.h>
#include <stddef.h>

static int is(char c, char u) { return c == u || c == u + 32; }

void dsyrk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *ldA, double *beta,
            double *C, int *ldC) {
  int N = *n, K = *k, lda = *ldA, ldc = *ldC;
  int lower = is(uplo[0], 'L'), t = is(trans[0], 'T') || is(trans[0], 'C');
  for (int j = 0; j < N; ++j) {
    int i0 = lower ? j : 0, i1 = lower ? N : j + 1;
    for (int i = i0; i < i1; ++i) {
      double s = 0.0;
      for (int p = 0; p < K; ++p) {
        double a = t ? A[(size_t)i * lda + p] : A[(size_t)p * lda + i];
        double b = t ? A[(size_t)j * lda + p] : A[(size_t)p * lda + j];
        s += a * b;
      }
      double *c = &C[(size_t)j * ldc + i];
      *c = (*beta == 0.0 ? 0.0 : *beta * *c) + *alpha * s;
    }
  }
}

void dposv_(char *uplo, int *n, int *nrhs, double *a, int *lda, double *b, int *ldb, int *info) {
  int N = *n, R = *nrhs, ld = *lda, lb = *ldb;
  int lower = is(uplo[0], 'L');
  /* L(i,j), i >= j, lives in the `uplo` triangle */
#define AL(i, j) (*(lower ? &a[(size_t)(j) * ld + (i)] : &a[(size_t)(i) * ld + (j)]))
  *info = 0;
  for (int j = 0; j < N; ++j) {
    double d = AL(j, j);
    for (int p = 0; p < j; ++p) d -= AL(j, p) * AL(j, p);
    if (!(d > 0.0)) {
      *info = j + 1;
      return;
    }
    d = sqrt(d);
    AL(j, j) = d;
    for (int i = j + 1; i < N; ++i) {
      double s = AL(i, j);
      for (int p = 0; p < j; ++p) s -= AL(i, p) * AL(j, p);
      AL(i, j) = s / d;
    }
  }
  for (int r = 0; r < R; ++r) {
    double *x = b + (size_t)r * lb;
    for (int i = 0; i < N; ++i) { /* L y = b */
      double s = x[i];
      for (int p = 0; p < i; ++p) s -= AL(i, p) * x[p];
      x[i] = s / AL(i, i);
    }
    for (int i = N - 1; i >= 0; --i) { /* L^T x = y */
      double s = x[i];
      for (int p = i + 1; p < N; ++p) s -= AL(p, i) * x[p];
      x[i] = s / AL(i, i);
    }
  }
#undef AL
}
