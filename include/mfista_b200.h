/*
 * C ABI of the B200 MFISTA solver library (libmfista_b200.so).
 *
 * Part 1 replaces the reference's solver entry points one for one: same
 * names, same argument lists and meanings, same struct RESULT layout, so the
 * reference's command-line drivers (c/mfista_imaging_{nufft,fft,dft}.c) link
 * against this library unchanged.  Part 2 adds entry points the reference
 * does not have (batched solves, a reusable device-resident plan, operator
 * level calls); they follow the same conventions (caller-owned host arrays,
 * layouts of the reference) and return a status code.
 *
 * All computation runs on the current CUDA device of the calling thread.
 * There is no CPU fallback: without a usable GPU every entry point fails
 * (the reference-compatible ones print the error, leave their outputs as
 * the reference leaves them on error, and set mfista_last_status()).
 */
#ifndef MFISTA_B200_H
#define MFISTA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* struct RESULT exactly as c/mfista.h:45-66 (field order and types are ABI). */
struct RESULT {
  int M;
  int N;
  int NX;
  int NY;
  int N_active;
  int maxiter;
  int ITER;
  int nonneg;
  double lambda_l1;
  double lambda_tv;
  double lambda_tsv;
  double sq_error;
  double mean_sq_error;
  double l1cost;
  double tvcost;
  double tsvcost;
  double finalcost;
  double comp_time;
  double *residual;
  double Lip_const;
};

/* ------------------------------------------------------------------------
 * Part 1: drop-in replacements (FP64, one problem per call).
 * ------------------------------------------------------------------------ */

/* Replaces mfista_imaging_core_nufft, c/mfista.h:172-178
 * (implementation c/mfista_nufft_lib.c:909-957). */
void mfista_imaging_core_nufft(double *u_dx, double *v_dy,
                               double *vis_r, double *vis_i, double *vis_std,
                               int M, int NX, int NY, int maxiter, double eps,
                               double lambda_l1, double lambda_tv, double lambda_tsv,
                               double cinit, double *xinit, double *xout,
                               int nonneg_flag, int box_flag, float *cl_box,
                               struct RESULT *mfista_result);

/* Replaces mfista_imaging_core_fft, c/mfista.h:161-168
 * (implementation c/mfista_fft_lib.c:701-756).  fftw_plan_flag is accepted
 * and ignored (there is no FFTW planning on the GPU). */
void mfista_imaging_core_fft(int *u_idx, int *v_idx,
                             double *y_r, double *y_i, double *noise_stdev,
                             int M, int NX, int NY, int maxiter, double eps,
                             double lambda_l1, double lambda_tv, double lambda_tsv,
                             double cinit, double *xinit, double *xout,
                             int nonneg_flag, unsigned int fftw_plan_flag,
                             int box_flag, float *cl_box,
                             struct RESULT *mfista_result);

/* Replaces mfista_imaging_core_dft, c/mfista.h:151-157
 * (implementation c/mfista_dft_lib.c:540-589).  A is column-major M x N.
 * As in the reference, RESULT.residual is malloc'ed here ([M] doubles) and
 * owned by the caller; looe_flag is ignored (the reference's LOOE call is
 * commented out, c/mfista_dft_lib.c:508-531). */
void mfista_imaging_core_dft(double *y, double *A,
                             int *M, int *N, int NX, int NY, int maxiter, double eps,
                             double lambda_l1, double lambda_tv, double lambda_tsv,
                             double cinit, double *xinit, double *xout,
                             int nonneg_flag, int looe_flag,
                             int box_flag, float *cl_box,
                             struct RESULT *mfista_result);

/* ------------------------------------------------------------------------
 * Part 2: extensions (no counterpart in the reference unless cited).
 * ------------------------------------------------------------------------ */

enum mfista_status {
  MFISTA_OK = 0,
  MFISTA_ERR_CUDA = 1,       /* a CUDA call failed (no device, launch error ...) */
  MFISTA_ERR_ARG = 2,        /* invalid argument (sizes, flags, unsupported shape) */
  MFISTA_ERR_NOMEM = 3,      /* device allocation failed */
  MFISTA_ERR_BOTH_REG = 4,   /* lambda_tv and lambda_tsv both non-zero */
  MFISTA_ERR_NONFINITE = 5,  /* objective became NaN/Inf: problem stopped */
  MFISTA_ERR_STEPCAP = 6     /* device step budget exhausted: problem stopped */
};

/* Selects the CUDA device used by this thread's subsequent calls (the
 * library carries its own CUDA runtime, so a device chosen through another
 * runtime, e.g. a framework's, does not carry over). */
int mfista_set_device(int device);

/* Status / message of the last call made by this thread. */
int mfista_last_status(void);
const char *mfista_last_error(void);

/* mfista_imaging_core_nufft keeps the solvers of its last calls (at most 4,
 * per device): a call with the same uv points, vis_std, sizes, regulariser
 * form, FGP iterations and box mask as a kept one reuses its device buffers
 * and captured solve graph and only uploads the new visibilities.  This
 * frees them (solvers in use by another thread stay); call it before a
 * cudaDeviceReset (a kept solver found without its device memory is not
 * reused, but its addresses are not freed either).  Setting
 * MFISTA_DROPIN_CACHE=0 in the environment disables the cache. */
void mfista_release_cache(void);

/* FGP iterations used by the TV form of the drop-in entry points on this
 * thread (the reference compiles it in: FGPITER 100, c/mfista.h:38).
 * Returns the previous value; n < 1 is rejected (returns -1). */
int mfista_set_fgp_iter(int n);

/* Arithmetic of the operators (spread/interp/FFT/stencils).  The objective,
 * reductions, backtracking test and FISTA sequence are FP64 in both. */
enum mfista_precision {
  MFISTA_FP64 = 64,
  MFISTA_FP32 = 32,
  MFISTA_BF16X3 = 3,
  MFISTA_BF16X6 = 6
};
/* MFISTA_BF16X3 / MFISTA_BF16X6 (DFT operator only): A z and A^T r on the
 * tensor cores from BF16 split operands with FP32 accumulation: two planes
 * each and three products (hi*hi + hi*lo + lo*hi, ~2^-16 relative), or
 * three planes each and six products (~2^-24, FP32-like).  The solver applies
 * them to the departure from an FP64 anchor refreshed every 8 (BF16X3) or 32
 * (BF16X6) outer iterations. */

/* Per-problem parameters of a batched solve. */
struct mfista_problem {
  double lambda_l1;
  double lambda_tv;
  double lambda_tsv;
  double cinit;
  int maxiter;
  int nonneg_flag;
  /* > 0: the problem also stops as soon as its accepted objective is
   * <= target_cost (used to time solves to a given relative objective);
   * 0 keeps the reference's stopping rules only. */
  double target_cost;
};

/* Batched NUFFT solve: B problems on one Nx x Ny grid advance together on
 * the GPU, each with its own backtracking state and convergence mask.
 *   geometry: if shared_geometry != 0 all problems use the M points of
 *     u_dx/v_dy/vis_*; otherwise problem b uses points
 *     [pt_off[b], pt_off[b+1]) of the concatenated arrays (uneven M), and
 *     M is their length, or 0 to take it as pt_off[B]; pt_off must start
 *     at >= 0, never decrease and end at <= M (else MFISTA_ERR_ARG).
 *   eps is scaled per problem exactly as mfista_imaging_core_nufft does.
 *   xinit: [B*Nx*Ny] or NULL (zero start); xout: [B*Nx*Ny];
 *   results: [B] RESULT records (residual left NULL).
 *   fgp_iter: FGP iterations of the TV form (the reference uses 100). */
int mfista_nufft_batch(const double *u_dx, const double *v_dy, const double *vis_r,
                       const double *vis_i, const double *vis_std, const int *pt_off,
                       int shared_geometry, int M, int Nx, int Ny, int B,
                       const struct mfista_problem *problems, double eps, int precision,
                       int fgp_iter, const double *xinit, double *xout,
                       struct RESULT *results);

/* Movie: n_frames images of one source, solved as ONE problem
 *   min sum_b [ chi2_b(x_b)/2 + lambda_l1 |x_b|_1 + lambda_tsv TSV(x_b) ]
 *       + lambda_t sum_b |x_b - x_{b+1}|^2 / (t_{b+1} - t_b)
 * by MFISTA with one joint step size, momentum, backtracking test and
 * stopping rule (the reference's matlab/MFISTA_movie_eht.m:93-194, with
 * d_X / dt_X of matlab/lib; its NUFFT is FINUFFT, here every frame uses
 * this library's NUFFT, i.e. the C reference's gridding).  Frame b uses
 * points [pt_off[b], pt_off[b+1]).  t_list: n_frames increasing frame times,
 * or NULL for 1, 2, ...  eps is used as given (the matlab code does not
 * scale it).  xinit: one Nx*Ny image replicated to every frame, or NULL.
 * xout: [n_frames*Nx*Ny]; results: [n_frames] per-frame terms (finalcost
 * without the temporal term; ITER and Lip_const are the joint ones);
 * temporal_cost: lambda_t times the temporal sum at xout (may be NULL).
 * c_box: [Nx*Ny] pixel weights or NULL: the starting image is xinit .* c_box
 * and every thresholded image is multiplied by c_box pixel by pixel, as the
 * matlab code's c_box (MFISTA_movie_eht.m:46, :143-146; a 0/1 mask is a
 * support constraint).
 * precision: MFISTA_FP64, or MFISTA_FP32 (FP32 NUFFTs with the FP64 anchor
 * correction of mfista_nufft_batch; objective, backtracking and momentum in
 * FP64).  TSV form (the matlab code has no TV form).
 * No counterpart in the reference's C library. */
int mfista_nufft_movie(const double *u_dx, const double *v_dy, const double *vis_r, const double *vis_i,
                       const double *vis_std, const int *pt_off, int n_frames, int Nx, int Ny,
                       const double *t_list, double lambda_l1, double lambda_tsv, double lambda_t,
                       double cinit, int maxiter, double eps, int nonneg_flag, const double *c_box,
                       int precision, const double *xinit, double *xout, struct RESULT *results,
                       double *temporal_cost);

/* Batched DFT solve (B problems sharing the column-major M x N matrix A and
 * the data y, e.g. a lambda grid): A z and A^T r run as GEMMs over the
 * batch.  eps is used raw, as mfista_imaging_core_dft does.  precision: 64. */
int mfista_dft_batch(const double *y, const double *A, int M, int N, int NX, int NY, int B,
                     const struct mfista_problem *problems, double eps, int precision,
                     int fgp_iter, const double *xinit, double *xout, struct RESULT *results);

/* Batched FFT (gridded) variant: B problems sharing the gridded data of
 * mfista_imaging_core_fft (u_idx, v_idx, y_r, y_i, noise_stdev [M] on an
 * NX x NY grid, e.g. a lambda grid) advance together, each with its own
 * backtracking state and convergence mask.  eps is scaled as
 * mfista_imaging_core_fft scales it (c/mfista_fft_lib.c:715-717).
 * precision MFISTA_FP64, or MFISTA_FP32: FP32 FFTs and FGP stencils, the
 * forward spectrum corrected by the exact FP64 spectrum of an anchor image
 * refreshed every 32 outer iterations, objective / backtracking / FISTA
 * sequence in FP64.  fgp_iter: FGP iterations of the TV form (the
 * reference compiles in 100).  xinit: [B*NX*NY] or NULL; xout [B*NX*NY];
 * results [B] (may be NULL).  No counterpart in the reference. */
int mfista_fft_batch(const int *u_idx, const int *v_idx, const double *y_r, const double *y_i,
                     const double *noise_stdev, int M, int NX, int NY, int B,
                     const struct mfista_problem *problems, double eps, int precision, int fgp_iter,
                     const double *xinit, double *xout, struct RESULT *results);

/* Device-resident plan of a batched NUFFT solve.  Creation uploads the
 * geometry and visibilities once and builds the CUDA graph; mfista_plan_run
 * enqueues one whole batched solve on the plan's stream without waiting;
 * mfista_plan_fetch waits and copies results to the host. */
typedef struct mfista_plan_s *mfista_plan;
mfista_plan mfista_nufft_plan_create(const double *u_dx, const double *v_dy,
                                     const double *vis_r, const double *vis_i,
                                     const double *vis_std, const int *pt_off,
                                     int shared_geometry, int M, int Nx, int Ny, int B,
                                     int precision, int form_tv, int fgp_iter);
int mfista_plan_set_problems(mfista_plan plan, const struct mfista_problem *problems,
                             double eps, const double *xinit);
int mfista_plan_run(mfista_plan plan);
int mfista_plan_fetch(mfista_plan plan, double *xout, struct RESULT *results);
void *mfista_plan_stream(mfista_plan plan);          /* cudaStream_t */
/* Times one operator kernel of the plan in isolation on the plan's stream:
 * `reps` back-to-back launches over all B problems, CUDA events around
 * them.  kernel: 0 interpolation, 1 spreading, 2 row FFT (forward),
 * 3 column FFT (forward), 4 column FFT (inverse), 5 row FFT (inverse),
 * 6 proximal update (TSV form) or FGP (TV form).  Outputs the mean
 * milliseconds per launch and the algorithmic bytes one launch must move
 * (compulsory reads + writes).  Leaves the plan's iterates undefined: call
 * mfista_plan_set_problems again before the next run. */
int mfista_plan_profile(mfista_plan plan, int kernel, int reps, double *ms_per_launch,
                        double *bytes_per_launch);
int mfista_plan_kernel_launches(mfista_plan plan);   /* kernels per solve, last run */
/* Launch shapes of the plan's operator kernels, as int[4]:
 *   [0] interpolation points per warp (shared geometry; 1..32),
 *   [1] spreading CTAs per tile cluster (shared geometry; 1..16),
 *   [2] image rows per CTA of the row FFT passes,
 *   [3] grid columns per CTA of the column FFT passes;
 * 0 = not used by this plan's operator (get) or keep the current value
 * (set).  Rows/columns per CTA leave results bit-identical; the other two
 * regroup sums and move results by rounding only.  set_shapes captures the
 * solve graph again; an impossible shape returns MFISTA_ERR_ARG. */
int mfista_plan_get_shapes(mfista_plan plan, int *shapes);
int mfista_plan_set_shapes(mfista_plan plan, const int *shapes);
/* Autotuner: times every candidate shape of each knob above with the
 * plan's kernels in isolation (as mfista_plan_profile, `reps` launches),
 * one knob at a time, both with every problem active (t_all) and with one
 * problem active (t_one, the tail of a batched solve), keeps the shape
 * minimising t_all / min t_all + 2 t_one / min t_one, and captures the graph
 * again.  shapes_out: int[4] chosen shapes; ms_out: double[4] t_all per
 * launch of each knob's kernels at the chosen shape (0 for unused knobs).
 * Either may be NULL.  Like mfista_plan_profile, it leaves the iterates
 * undefined. */
int mfista_plan_tune(mfista_plan plan, int reps, int *shapes_out, double *ms_out);
/* Per-problem status of the last fetched solve (enum mfista_status values). */
int mfista_plan_statuses(mfista_plan plan, int *status_out);
/* 1 when the plan iterates with a device-side conditional WHILE graph node,
 * 0 when it fell back to relaunching the step graph from the host. */
int mfista_plan_device_loop(mfista_plan plan);
void mfista_plan_destroy(mfista_plan plan);

/* Operators of the NUFFT variant, as the C++ reference exports them
 * (x2y_nufft / y2x_nufft, c++/mfista.hpp:136-140), with the C gridding of
 * c/mfista_nufft_lib.c:123-243:
 *   forward: (out_r, out_i)[M] = NUFFT2d2(x)       x: [Nx*Ny]
 *   adjoint: x_out[Nx*Ny]      = NUFFT2d1(r_r, r_i) */
int mfista_nufft_forward(const double *u_dx, const double *v_dy, int M, int Nx, int Ny,
                         const double *x, double *out_r, double *out_i, int precision);
int mfista_nufft_adjoint(const double *u_dx, const double *v_dy, int M, int Nx, int Ny,
                         const double *r_r, const double *r_i, double *x_out, int precision);

/* NUFFT forward operator for callers that may not allocate GPU memory (no
 * counterpart in the reference).  Meant for hosts whose device memory is
 * owned by their own pool, or that cannot take the device-wide
 * synchronisation a cudaMalloc/cudaFree brings; mfista_nufft_forward
 * allocates its working buffers on every call.
 *   u_dx, v_dy [M], x [Nx*Ny], out_r, out_i [M]: DEVICE pointers; FP64.
 *   stream: a cudaStream_t (NULL: the default stream); the work is enqueued
 *           there and the call returns without waiting for it.
 * All intermediates live in one fixed device array of
 * MFISTA_NOALLOC_SCRATCH_BYTES, which a device holds from the first call on
 * it (earlier where CUDA loads modules eagerly) until the process exits;
 * nothing is allocated or freed.  Inputs whose working set exceeds it, and
 * Nx > 767 or Ny > 1535, are rejected with MFISTA_ERR_ARG.  The working set
 * is approximately 32*Nx*(Ny+1) + 8*Nx*Ny + 408*M bytes (each of its 13
 * pieces is rounded up to 256 bytes and the FFT twiddle tables add
 * 16*(3*Ny + 2*Nx) bytes), so inputs near the limit may be rejected.  The
 * first call on a device looks up the array's address there and keeps it:
 * make it before any stream capture, and do not call this entry point on a
 * device after a cudaDeviceReset of it (the kept address is then stale).  A
 * CUDA error already pending in the calling thread is reported as
 * MFISTA_ERR_CUDA and left pending.  Calls share the array, so calls that
 * may run at the same time on one GPU race and must be ordered by the
 * caller.  Returns an mfista_status; mfista_last_status/error are not
 * updated. */
#define MFISTA_NOALLOC_SCRATCH_BYTES (16u << 20)
int mfista_nufft_forward_noalloc(const double *u_dx, const double *v_dy, int M, int Nx, int Ny,
                                 const double *x, double *out_r, double *out_i, void *stream);

/* DFT operator alone for B vectors (dgemv "N"/"T" of c/mfista_dft_lib.c:30-66,
 * :253-278, batched): A is column-major M x N;
 *   transpose = 0: out[b][m] = sum_n A[m + n M] X[b][n]   (X [B][N], out [B][M])
 *   transpose = 1: out[b][n] = sum_m A[m + n M] X[b][m]   (X [B][M], out [B][N])
 * precision MFISTA_FP64, or MFISTA_BF16X3 / MFISTA_BF16X6 for the
 * tensor-core split-BF16 GEMM alone (no anchor: ~1e-5 / ~1e-7 relative
 * error). */
int mfista_dft_apply(const double *A, int M, int N, const double *X, int B, int transpose, int precision,
                     double *out);

/* Times one DFT operator kernel alone for a batch of B problems sharing A
 * (as mfista_plan_profile): kernel 0 = the A z GEMM, 1 = the A^T r GEMM, in
 * the given precision (MFISTA_FP64 needs B > 1: the batched GEMMs). */
int mfista_dft_profile(const double *A, int M, int N, int B, int precision, int kernel, int reps,
                       double *ms_per_launch, double *bytes_per_launch);

/* Approximate leave-one-out error (LOOE) of B solutions X [B][N] of the DFT
 * problem y [M] = A [M x N, column-major] x: the reference's
 * compute_LOOE_L1 / compute_LOOE_L1_TSV (c/looe_lib.c:190-226, :275-309;
 * its call in c/mfista_dft_lib.c:506-529 is commented out and the reference
 * does not build the file) on the GPU in FP64.  From the active set S of x:
 * H = A_S^T A_S (+ lambda_tsv[b] times the TSV Hessian diagonal 8/6/4 of
 * the NX grid), d_i = (A_S H^-1 A_S^T)_ii, t_i = (y - A x)_i / (1 - d_i);
 * looe_m[b] = mean t_i^2/2 and looe_std[b] their spread as the reference
 * forms it.  hessian_positive[b] = 0 when H is not positive definite (then
 * looe_m = looe_std = 0, the reference's -1 return).  lambda_tsv may be
 * NULL (L1 form for every solution).  Needs M >= 2. */
int mfista_dft_looe(const double *y, const double *A, int M, int N, int NX, const double *X, int B,
                    const double *lambda_tsv, double *looe_m, double *looe_std, int *hessian_positive);

/* Forward NUFFT of the reference's C++ build: x2y_nufft
 * (c++/mfista_nufft_lib.cpp:1076-1149, exported by c++/mfista.hpp:136-137)
 * with the same arguments, on the GPU in FP64: its 12-tap (MSP = 6) kernel,
 * floor binning of points flipped to v >= 0 and Hermitian halo, which differ
 * from the C library's operator (mfista_nufft_forward).  y_r, y_i: [M]. */
int mfista_cpp_x2y_nufft(const double *u_dx, const double *v_dy, int M, int Nx, int Ny, const double *xin,
                         double *y_r, double *y_i);

/* Adjoint NUFFT of the reference's C++ build: y2x_nufft
 * (c++/mfista_nufft_lib.cpp:1151-1219, NUFFT2d1_sngl :189-258, exported by
 * c++/mfista.hpp:139-140), on the GPU in FP64: the 12-tap spreading with
 * the Hermitian halo folds done as a deterministic per-cell gather, then the
 * padded inverse FFT and the C++ grid correction.  xout: [Nx*Ny]. */
int mfista_cpp_y2x_nufft(const double *u_dx, const double *v_dy, int M, int Nx, int Ny, const double *yin_r,
                         const double *yin_i, double *xout);

/* The C++ build's solver entry points (c++/mfista_nufft_lib.cpp:1016-1074,
 * c++/mfista_fft_lib.cpp:425-485) under library-specific names; the C++
 * build's own names are exported by libmfista_b200_cpp.so
 * (include/mfista_b200_cpp.h), which forwards here.  NUFFT: the C++
 * operators above, first-iteration backtracking factor 10, RESULT as its
 * calc_costs_nufft fills it, the caller's u/v/vis arrays sorted in place,
 * TSV form only.  FFT: the C library's TSV solve, no TV form. */
void mfista_cpp_imaging_core_nufft(double *u_dx, double *v_dy, double *vis_r, double *vis_i, double *vis_std,
                                   int M, int Nx, int Ny, int maxiter, double eps, double lambda_l1,
                                   double lambda_tv, double lambda_tsv, double cinit, double *xinit, double *xout,
                                   int nonneg_flag, int box_flag, float *cl_box, struct RESULT *mfista_result);
void mfista_cpp_imaging_core_fft(int *u_idx, int *v_idx, double *y_r, double *y_i, double *noise_stdev, int M,
                                 int NX, int NY, int maxiter, double eps, double lambda_l1, double lambda_tv,
                                 double lambda_tsv, double cinit, double *xinit, double *xout, int nonneg_flag,
                                 unsigned int fftw_plan_flag, int box_flag, float *cl_box,
                                 struct RESULT *mfista_result);

/* FGP TV proximal map alone (FGP_L1_box / FGP_nonneg_box,
 * c/mfista_TV_lib.c:189-384) on an NX x NY view: x_out = prox(b). */
int mfista_fgp_prox(const double *b, int NX, int NY, double lambda_l1, double lambda_tv,
                    int iters, int nonneg_flag, int box_flag, const float *cl_box,
                    double *x_out, int precision);

/* Times the FGP TV prox alone (the kernel mfista_fgp_prox runs) for B
 * problems of NX x NY in one launch, `iters` FGP iterations each, in
 * MFISTA_FP64 or MFISTA_FP32 stencil arithmetic: CUDA events around `reps`
 * launches on the library's stream.  Outputs the mean milliseconds per
 * launch and its compulsory bytes (image vectors read and written once). */
int mfista_fgp_profile(int NX, int NY, int B, int iters, int precision, int reps, double *ms_per_launch,
                       double *bytes_per_launch);

/* Power-iteration estimate of the Lipschitz constant of the chi^2 gradient
 * (largest eigenvalue of A^H W^2 A) of a NUFFT problem, for choosing cinit. */
int mfista_nufft_lipschitz(const double *u_dx, const double *v_dy, const double *vis_std,
                           int M, int Nx, int Ny, int iters, double *lip_out);

/* Learned warm start (no counterpart in the reference): a U-Net with 4
 * levels of 16-32-64-128 channels, BF16 weights and FP32 accumulation, that
 * maps a problem's dirty image and dirty beam (2 input channels, H x W, H
 * and W multiples of 8) to an initial image clamped to >= 0.  Forward,
 * backward and Adam run on the GPU (deterministic).  Arrays are host float
 * arrays: inputs [n][2][H][W], images [n][H][W], parameters in the layout
 * of csrc/unet.cu (per 3x3 layer: weights [cout][cin][3][3], bias [cout];
 * then the 1x1 head's 16 weights and bias).  Status: 0 or an mfista_status
 * (details from mfista_unet_last_error). */
void *mfista_unet_create(int H, int W, int batch_max);
void mfista_unet_destroy(void *net);
long mfista_unet_param_count(void *net);
int mfista_unet_get_params(void *net, float *out);
int mfista_unet_set_params(void *net, const float *in);
int mfista_unet_forward(void *net, const float *in, int n, float *out);
/* loss = mean squared error of the unclamped output against target;
 * grad [param_count] (may be NULL) */
int mfista_unet_grad(void *net, const float *in, const float *target, int n, float *loss, float *grad);
/* one Adam step (beta 0.9 / 0.999) with learning rate lr; reports the loss */
int mfista_unet_train_step(void *net, const float *in, const float *target, int n, float lr, float *loss);
int mfista_unet_last_status(void);
const char *mfista_unet_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MFISTA_B200_H */
