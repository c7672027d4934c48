/*
 * Project-written implementation of the FFTW3 calls declared in fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY: it lets the unchanged reference C solvers
 * (c/mfista_nufft_lib.c, c/mfista_fft_lib.c) be compiled as the CPU parity
 * oracle and CPU baseline.  The shipped GPU library never links it.
 *
 * Algorithm (own code): an iterative Stockham auto-sort complex FFT with
 * mixed radix (2, 3, 4, 5 and a direct DFT for any other prime factor),
 * twiddles taken from a per-length table exp(-2*pi*i*k/n) computed with
 * cos/sin of reduced angles.  The 2-D real transforms follow the usual
 * row/column decomposition:
 *   r2c: 1-D real->half-complex on every row (via a full-length complex FFT
 *        of the real row), then complex FFTs down every half-spectrum column;
 *   c2r: inverse complex FFTs down every column, then a 1-D half-complex->real
 *        transform on every row that uses only the real parts of the DC and
 *        Nyquist bins (the imaginary parts of those bins are ignored, as a
 *        half-complex input defines them to be zero).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

typedef double _Complex cplx;

typedef struct {
  int n;
  int nf;
  int fac[64];
  cplx *tw; /* tw[k] = exp(-2 pi i k / n) */
  cplx *stw[64]; /* per-stage twiddles */
} cfft_t;

struct oracle_fftw_plan_s {
  int kind; /* 0 = r2c, 1 = c2r */
  int n0, n1, nh;
  double *rbuf;
  cplx *cbuf;
  cfft_t row, col;
  cplx *work_a, *work_b;
};

static void cfft_init(cfft_t *p, int n) {
  int m = n, f;
  p->n = n;
  p->nf = 0;
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  for (f = 3; f * f <= m; f += 2)
    while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
  if (m > 1) p->fac[p->nf++] = m;
  p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
  for (int k = 0; k < n; ++k) {
    /* reduce the angle to the first octant-ish range for accuracy */
    long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
    p->tw[k] = (double)cosl(a) - I * (double)sinl(a);
  }
}

static void cfft_stage_twiddles(cfft_t *p);

static void cfft_free(cfft_t *p) {
  for (int s = 0; s < p->nf; ++s) free(p->stw[s]);
  free(p->tw);
  p->tw = NULL;
}

/* root of unity exp(sign * 2 pi i * idx / n) from the table */
static inline cplx tw_get(const cfft_t *p, long idx, int sign) {
  int n = p->n;
  long k = idx % n;
  if (k < 0) k += n;
  cplx w = p->tw[k];
  return sign < 0 ? w : conj(w);
}

/* per-stage twiddles: stw[s][k*(R-1) + (r-1)] = exp(-2 pi i k r / (Ns R)) */
static void cfft_stage_twiddles(cfft_t *p) {
  int Ns = 1;
  for (int s = 0; s < p->nf; ++s) {
    int R = p->fac[s];
    p->stw[s] = (cplx *)malloc(sizeof(cplx) * (size_t)Ns * (R - 1) + sizeof(cplx));
    long stride = p->n / (Ns * R);
    for (int k = 0; k < Ns; ++k)
      for (int r = 1; r < R; ++r)
        p->stw[s][(size_t)k * (R - 1) + (r - 1)] = p->tw[((long)k * r * stride) % p->n];
    Ns *= R;
  }
}

/* one length-n transform of x (in place), using work as scratch. */
static void cfft_exec(const cfft_t *p, cplx *x, cplx *work, int sign) {
  int n = p->n;
  if (n <= 1) return;
  cplx *src = x, *dst = work;
  int Ns = 1;
  cplx v[64], o[64];
  /* constants for the radix-3 and radix-5 butterflies (exact trig values) */
  const double c3 = -0.5, s3 = 0.86602540378443864676;
  const double c51 = 0.30901699437494742410, c52 = -0.80901699437494742410;
  const double s51 = 0.95105651629515357212, s52 = 0.58778525229247312917;
  for (int s = 0; s < p->nf; ++s) {
    int R = p->fac[s];
    int nR = n / R;
    const cplx *tws = p->stw[s];
    cplx *vv = v, *oo = o, *vbig = NULL, *obig = NULL;
    if (R > 64) {
      vbig = (cplx *)malloc(sizeof(cplx) * R);
      obig = (cplx *)malloc(sizeof(cplx) * R);
      vv = vbig; oo = obig;
    }
    double sg = (double)sign;
    for (int j = 0; j < nR; ++j) {
      int k = j % Ns;
      const cplx *tk = tws + (size_t)k * (R - 1);
      vv[0] = src[j];
      for (int r = 1; r < R; ++r) {
        cplx a = src[j + r * nR];
        if (k) a *= (sign < 0 ? tk[r - 1] : conj(tk[r - 1]));
        vv[r] = a;
      }
      if (R == 2) {
        oo[0] = vv[0] + vv[1];
        oo[1] = vv[0] - vv[1];
      } else if (R == 4) {
        cplx t0 = vv[0] + vv[2], t1 = vv[0] - vv[2];
        cplx t2 = vv[1] + vv[3], t3 = vv[1] - vv[3];
        /* t3 times exp(sign*i*pi/2) = sign*i */
        cplx t3r = sign < 0 ? (cimag(t3) - I * creal(t3)) : (-cimag(t3) + I * creal(t3));
        oo[0] = t0 + t2;
        oo[2] = t0 - t2;
        oo[1] = t1 + t3r;
        oo[3] = t1 - t3r;
      } else if (R == 3) {
        cplx t1 = vv[1] + vv[2], t2 = vv[1] - vv[2];
        cplx m1 = vv[0] + c3 * t1;
        /* exp(sign*2 pi i/3) = c3 + sign*i*s3 */
        cplx m2 = (sg * s3) * (I * t2);
        oo[0] = vv[0] + t1;
        oo[1] = m1 + m2;
        oo[2] = m1 - m2;
      } else if (R == 5) {
        cplx a1 = vv[1] + vv[4], b1 = vv[1] - vv[4];
        cplx a2 = vv[2] + vv[3], b2 = vv[2] - vv[3];
        cplx r1 = vv[0] + c51 * a1 + c52 * a2;
        cplx r2 = vv[0] + c52 * a1 + c51 * a2;
        cplx i1 = (sg * I) * (s51 * b1 + s52 * b2);
        cplx i2 = (sg * I) * (s52 * b1 - s51 * b2);
        oo[0] = vv[0] + a1 + a2;
        oo[1] = r1 + i1;
        oo[4] = r1 - i1;
        oo[2] = r2 + i2;
        oo[3] = r2 - i2;
      } else {
        long step = n / R;
        for (int q = 0; q < R; ++q) {
          cplx acc = vv[0];
          for (int r = 1; r < R; ++r)
            acc += vv[r] * tw_get(p, (long)((r * q) % R) * step, sign);
          oo[q] = acc;
        }
      }
      int base = (j / Ns) * Ns * R + k;
      for (int r = 0; r < R; ++r) dst[base + r * Ns] = oo[r];
    }
    free(vbig);
    free(obig);
    cplx *t = src; src = dst; dst = t;
    Ns *= R;
  }
  if (src != x) memcpy(x, src, sizeof(cplx) * n);
}

static fftw_plan plan_alloc(int kind, int n0, int n1) {
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  int mx = n0 > n1 ? n0 : n1;
  p->kind = kind;
  p->n0 = n0;
  p->n1 = n1;
  p->nh = n1 / 2 + 1;
  cfft_init(&p->row, n1);
  cfft_init(&p->col, n0);
  cfft_stage_twiddles(&p->row);
  cfft_stage_twiddles(&p->col);
  p->work_a = (cplx *)malloc(sizeof(cplx) * mx);
  p->work_b = (cplx *)malloc(sizeof(cplx) * mx);
  return p;
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags) {
  (void)flags;
  fftw_plan p = plan_alloc(0, n0, n1);
  p->rbuf = in;
  p->cbuf = out;
  return p;
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags) {
  (void)flags;
  fftw_plan p = plan_alloc(1, n0, n1);
  p->rbuf = out;
  p->cbuf = in;
  return p;
}

static void exec_r2c(fftw_plan p) {
  int n0 = p->n0, n1 = p->n1, nh = p->nh;
  cplx *a = p->work_a, *b = p->work_b;
  for (int i = 0; i < n0; ++i) {
    for (int j = 0; j < n1; ++j) a[j] = p->rbuf[(size_t)i * n1 + j];
    cfft_exec(&p->row, a, b, -1);
    for (int j = 0; j < nh; ++j) p->cbuf[(size_t)i * nh + j] = a[j];
  }
  for (int j = 0; j < nh; ++j) {
    for (int i = 0; i < n0; ++i) a[i] = p->cbuf[(size_t)i * nh + j];
    cfft_exec(&p->col, a, b, -1);
    for (int i = 0; i < n0; ++i) p->cbuf[(size_t)i * nh + j] = a[i];
  }
}

static void exec_c2r(fftw_plan p) {
  int n0 = p->n0, n1 = p->n1, nh = p->nh;
  cplx *a = p->work_a, *b = p->work_b;
  /* columns first; the input buffer is overwritten (FFTW may do the same) */
  for (int j = 0; j < nh; ++j) {
    for (int i = 0; i < n0; ++i) a[i] = p->cbuf[(size_t)i * nh + j];
    cfft_exec(&p->col, a, b, +1);
    for (int i = 0; i < n0; ++i) p->cbuf[(size_t)i * nh + j] = a[i];
  }
  for (int i = 0; i < n0; ++i) {
    const cplx *h = p->cbuf + (size_t)i * nh;
    for (int k = 0; k < n1; ++k) {
      if (k == 0) a[k] = creal(h[0]);
      else if (2 * k == n1) a[k] = creal(h[k]);
      else if (k < nh) a[k] = h[k];
      else a[k] = conj(h[n1 - k]);
    }
    cfft_exec(&p->row, a, b, +1);
    for (int k = 0; k < n1; ++k) p->rbuf[(size_t)i * n1 + k] = creal(a[k]);
  }
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (p->kind == 0) exec_r2c(p);
  else exec_c2r(p);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  cfft_free(&p->row);
  cfft_free(&p->col);
  free(p->work_a);
  free(p->work_b);
  free(p);
}

void *fftw_malloc(size_t n) {
  void *ptr = NULL;
  if (posix_memalign(&ptr, 64, n ? n : 64) != 0) return NULL;
  return ptr;
}

void fftw_free(void *ptr) { free(ptr); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}
