/*
 * C ABI of libmfista_b200_cpp.so: the entry points of the reference's C++
 * build (c++/mfista.hpp:115-140), computed on the GPU by libmfista_b200.so.
 *
 * The reference ships two builds that export the same C names with
 * different numerics.  A program written against the C++ build links this
 * library instead of the reference's C++ objects; a program written
 * against the C build links libmfista_b200.so (include/mfista_b200.h).
 * struct RESULT is the one of mfista_b200.h (c/mfista.h:45-66; the C++
 * build's c++/mfista.hpp declares the same layout).
 */
#ifndef MFISTA_B200_CPP_H
#define MFISTA_B200_CPP_H

#include "mfista_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces the C++ build's mfista_imaging_core_nufft, c++/mfista.hpp:118-124
 * (implementation c++/mfista_nufft_lib.cpp:1016-1074): its NUFFT (12-tap
 * kernel, floor binning, Hermitian halos; c++/mfista_nufft_lib.cpp:85-504),
 * a backtracking factor of 10 in the first iteration (:818, :860-863),
 * RESULT filled by calc_costs_nufft (:931-998: M is the number of points).
 * As there, u_dx, v_dy, vis_r, vis_i and vis_std are sorted in place by
 * grid row of v, then of u (sort_input, :550-641), and only the TSV form
 * exists: lambda_tv != 0 prints a message and returns after filling the
 * costs at xinit. */
void mfista_imaging_core_nufft(double *u_dx, double *v_dy,
                               double *vis_r, double *vis_i, double *vis_std,
                               int M, int Nx, int Ny, int maxiter, double eps,
                               double lambda_l1, double lambda_tv, double lambda_tsv,
                               double cinit, double *xinit, double *xout,
                               int nonneg_flag, int box_flag, float *cl_box,
                               struct RESULT *mfista_result);

/* Replaces the C++ build's mfista_imaging_core_fft, c++/mfista.hpp:128-134
 * (implementation c++/mfista_fft_lib.cpp:425-485): the C library's gridded
 * TSV solve; lambda_tv != 0 prints a message and returns. */
void mfista_imaging_core_fft(int *u_idx, int *v_idx,
                             double *y_r, double *y_i, double *noise_stdev,
                             int M, int Nx, int Ny, int maxiter, double eps,
                             double lambda_l1, double lambda_tv, double lambda_tsv,
                             double cinit, double *xinit, double *xout,
                             int nonneg_flag, unsigned int fftw_plan_flag,
                             int box_flag, float *cl_box,
                             struct RESULT *mfista_result);

/* Replaces x2y_nufft, c++/mfista.hpp:136-137 (c++/mfista_nufft_lib.cpp:1076-1149):
 * y = A x with the C++ build's NUFFT. */
void x2y_nufft(double *u_dx, double *v_dy, int M, int Nx, int Ny,
               double *xin, double *y_r, double *y_i);

/* Replaces y2x_nufft, c++/mfista.hpp:139-140 (c++/mfista_nufft_lib.cpp:1151-1219):
 * x = A^H y with the C++ build's NUFFT (NUFFT2d1_sngl, :189-258). */
void y2x_nufft(double *u_dx, double *v_dy, int M, int Nx, int Ny,
               double *yin_r, double *yin_i, double *xout);

#ifdef __cplusplus
}
#endif

#endif /* MFISTA_B200_CPP_H */
