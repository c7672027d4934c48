/*
 * Project-written stand-in for the small part of the FFTW3 API that the
 * sparseimaging C solvers call (c/mfista.h:34 includes <fftw3.h>).
 *
 * TEST INFRASTRUCTURE ONLY.  This header and fftw_shim.c exist so that the
 * unchanged reference C sources can be compiled in this container (which has
 * no FFTW) and used as the parity oracle.  Nothing in the shipped library
 * includes or links it.
 *
 * Semantics follow the public FFTW3 documentation for the calls used:
 *   fftw_plan_dft_r2c_2d(n0, n1, in, out, flags): real n0 x n1 (row-major)
 *       -> complex n0 x (n1/2+1), forward sign -1, unnormalised.
 *   fftw_plan_dft_c2r_2d(n0, n1, in, out, flags): complex n0 x (n1/2+1)
 *       -> real n0 x n1, sign +1, unnormalised (may overwrite its input).
 * fftw_complex is C99 double _Complex because <complex.h> is included before
 * this header in c/mfista.h:33-34, which is FFTW's documented convention.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H

#include <stddef.h>
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fftw_complex;
typedef struct oracle_fftw_plan_s *fftw_plan;

#define FFTW_MEASURE        (0U)
#define FFTW_DESTROY_INPUT  (1U << 0)
#define FFTW_ESTIMATE       (1U << 6)

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
int  fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif
