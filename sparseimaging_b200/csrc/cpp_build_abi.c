/*
 * libmfista_b200_cpp.so: the names the reference's C++ build exports
 * (include/mfista_b200_cpp.h), each forwarding to the C++-build entry of
 * libmfista_b200.so.  Status and messages of a call are those of
 * libmfista_b200.so (mfista_last_status / mfista_last_error).
 */
#include "mfista_b200_cpp.h"

void mfista_imaging_core_nufft(double *u_dx, double *v_dy, double *vis_r, double *vis_i, double *vis_std, int M,
                               int Nx, int Ny, int maxiter, double eps, double lambda_l1, double lambda_tv,
                               double lambda_tsv, double cinit, double *xinit, double *xout, int nonneg_flag,
                               int box_flag, float *cl_box, struct RESULT *mfista_result) {
  mfista_cpp_imaging_core_nufft(u_dx, v_dy, vis_r, vis_i, vis_std, M, Nx, Ny, maxiter, eps, lambda_l1, lambda_tv,
                                lambda_tsv, cinit, xinit, xout, nonneg_flag, box_flag, cl_box, mfista_result);
}

void mfista_imaging_core_fft(int *u_idx, int *v_idx, double *y_r, double *y_i, double *noise_stdev, int M, int Nx,
                             int Ny, int maxiter, double eps, double lambda_l1, double lambda_tv, double lambda_tsv,
                             double cinit, double *xinit, double *xout, int nonneg_flag,
                             unsigned int fftw_plan_flag, int box_flag, float *cl_box,
                             struct RESULT *mfista_result) {
  mfista_cpp_imaging_core_fft(u_idx, v_idx, y_r, y_i, noise_stdev, M, Nx, Ny, maxiter, eps, lambda_l1, lambda_tv,
                              lambda_tsv, cinit, xinit, xout, nonneg_flag, fftw_plan_flag, box_flag, cl_box,
                              mfista_result);
}

void x2y_nufft(double *u_dx, double *v_dy, int M, int Nx, int Ny, double *xin, double *y_r, double *y_i) {
  mfista_cpp_x2y_nufft(u_dx, v_dy, M, Nx, Ny, xin, y_r, y_i);
}

void y2x_nufft(double *u_dx, double *v_dy, int M, int Nx, int Ny, double *yin_r, double *yin_i, double *xout) {
  mfista_cpp_y2x_nufft(u_dx, v_dy, M, Nx, Ny, yin_r, yin_i, xout);
}
