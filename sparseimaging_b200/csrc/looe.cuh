// Approximate leave-one-out error (LOOE) of DFT solutions on the GPU.
//
// The reference's c/looe_lib.c (compute_LOOE_L1 :190-226, compute_LOOE_L1_TSV
// :275-309, compute_LOOE_core :112-171; its call in c/mfista_dft_lib.c:506-529
// is commented out and its makefile does not build the file) scores a
// solution x of the DFT problem by
//   S = {j : |x_j| > 0},  A_S = A[:, S],
//   H = A_S^T A_S (+ lambda_tsv d2(j) on the diagonal, d2 = 8 / 6 / 4 inside /
//       on an edge / on a corner of the NX grid, d2_TSV :228-245),
//   d_i = (A_S H^-1 A_S^T)_ii,  t_i = (y - A x)_i / (1 - d_i),  s_i = t_i^2 / 2,
//   LOOE_m = mean s,  LOOE_std = sqrt(sum s^2 / (M-1) - LOOE_m^2 M / (M-1)),
// and reports a Hessian that is not positive definite (dposv info > 0).
//
// Here, all in FP64 on one stream, per solution:
//   Z = A_S gathered (M x n_s, column-major, coalesced column copies);
//   H = Z^T Z by a tiled FP64 GEMM (lower tiles only);
//   blocked right-looking Cholesky H = L L^T (64-wide panels: the diagonal
//   block factored in one CTA's shared memory, the panel below by one
//   thread per row, the trailing matrix by the GEMM);
//   Z <- Z L^-T block by block in the same loop, so that row i of Z ends as
//   (L^-1 a_i)^T and d_i = |row i|^2 (one triangular solve instead of the
//   reference's two: the same quantity, other rounding);
//   the residual, the t_i and the two sums with fixed-order reductions.
// A non-positive pivot sets an info word that every later kernel of the
// solution checks at entry.
#pragma once

#include "solver.cuh"

namespace mf {
namespace looe {

constexpr int kPanel = 64;  // Cholesky / triangular-solve block width
constexpr int kGT = 64;     // GEMM tile (rows and columns)
constexpr int kGK = 16;     // GEMM k step

// 8-byte asynchronous global -> shared copy; src_bytes 0 writes zeros
__device__ __forceinline__ void cp_async8_zfill(void* smem_dst, const void* gmem_src, unsigned int src_bytes) {
  const unsigned int d = (unsigned int)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(gmem_src), "r"(src_bytes) : "memory");
}

// C (m x n, ldc) = alpha op(A) op(B) + beta C, column-major; op(A)(i,p) is
// A[p + i lda] when TA, else A[i + p lda]; op(B)(p,j) is B[j + p ldb] when
// TB, else B[p + j ldb].  lower: tiles strictly above the diagonal are
// skipped (the Cholesky reads the lower triangle only).  256 threads, a
// 64 x 64 tile per CTA, 4 x 4 outputs per thread at rows tx + 16r and
// columns ty + 16c.  The k steps are double-buffered: the copies of step
// p + 1 (cp.async, element by element, zeros outside the matrices) are in
// flight while step p is multiplied.  With beta != 0 the C tile is copied
// into shared memory at the start, behind the k steps (the trailing
// updates of the factorisation are rank-64: four k steps only).
constexpr int kGLd = kGT + 1;  // shared row length (padded)
constexpr size_t kGemmSmem = sizeof(double) * (2 * 2 * kGK * kGLd + kGT * kGT);
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_looe_gemm(int m, int n, int k, double alpha, const double* __restrict__ A,
                                                   int lda, const double* __restrict__ B, int ldb, double beta,
                                                   double* __restrict__ C, int ldc, int lower,
                                                   const int* __restrict__ info) {
  if (info && *info) return;
  const int i0 = blockIdx.x * kGT, j0 = blockIdx.y * kGT;
  if (lower && i0 + kGT - 1 < j0) return;
  extern __shared__ __align__(16) double gemm_smem[];
  auto As = reinterpret_cast<double(*)[kGK][kGLd]>(gemm_smem);
  auto Bs = reinterpret_cast<double(*)[kGK][kGLd]>(gemm_smem + 2 * kGK * kGLd);
  double* Cs = gemm_smem + 4 * kGK * kGLd;  // [64 columns][64 rows]
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  if (beta != 0.0) {
    for (int e = t; e < kGT * kGT; e += 256) {
      const int i = e & (kGT - 1), j = e >> 6;
      const int gi = i0 + i, gj = j0 + j;
      const bool v = gi < m && gj < n;
      cp_async8_zfill(Cs + e, v ? C + (size_t)gi + (size_t)gj * ldc : C, v ? 8u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  auto stage = [&](int buf, int p0) {
#pragma unroll
    for (int q = 0; q < (kGT * kGK) / 256; ++q) {
      const int e = t + 256 * q;
      int i, p;
      if (TA) {
        i = e / kGK;
        p = e % kGK;
      } else {
        i = e % kGT;
        p = e / kGT;
      }
      const int gi = i0 + i, gp = p0 + p;
      const bool va = gi < m && gp < k;
      cp_async8_zfill(&As[buf][p][i], va ? (TA ? A + (size_t)gp + (size_t)gi * lda : A + (size_t)gi + (size_t)gp * lda) : A,
                      va ? 8u : 0u);
      int j;
      if (TB) {
        j = e % kGT;
        p = e / kGT;
      } else {
        j = e / kGK;
        p = e % kGK;
      }
      const int gj = j0 + j, gq = p0 + p;
      const bool vb = gj < n && gq < k;
      cp_async8_zfill(&Bs[buf][p][j], vb ? (TB ? B + (size_t)gj + (size_t)gq * ldb : B + (size_t)gq + (size_t)gj * ldb) : B,
                      vb ? 8u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
  const int nk = (k + kGK - 1) / kGK;
  // (the C group, when there is one, is older than every step's group, so
  // the waits below cover it too)
  if (nk > 0) stage(0, 0);
  for (int kt = 0; kt < nk; ++kt) {
    if (kt + 1 < nk) stage((kt + 1) & 1, (kt + 1) * kGK);
    else asm volatile("cp.async.commit_group;" ::: "memory");  // keeps one group per step
    asm volatile("cp.async.wait_group 1;" ::: "memory");       // step kt has landed (this thread)
    __syncthreads();                                           // and everyone's
    const int bf = kt & 1;
#pragma unroll
    for (int p = 0; p < kGK; ++p) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[bf][p][tx + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[bf][p][ty + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();  // buffer bf is refilled by the copies issued next step
  }
  if (beta != 0.0) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int li = tx + 16 * r, lj = ty + 16 * c;
      const int gi = i0 + li, gj = j0 + lj;
      if (gi < m && gj < n)
        C[(size_t)gi + (size_t)gj * ldc] = alpha * acc[r][c] + (beta != 0.0 ? beta * Cs[lj * kGT + li] : 0.0);
    }
}

// Z[:, j] = A[:, S_j] for the n_s active columns (M x n_s, column-major):
// one CTA per column
__global__ void k_looe_gather(const double* __restrict__ A, int M, const int* __restrict__ S,
                              double* __restrict__ Z) {
  const int j = blockIdx.x;
  const double* src = A + (size_t)S[j] * M;
  double* dst = Z + (size_t)j * M;
  for (int i = threadIdx.x; i < M; i += blockDim.x) dst[i] = src[i];
}

// r = y - A x over the active columns (x is zero elsewhere), column order
__global__ void k_looe_resid(const double* __restrict__ A, int M, const double* __restrict__ y,
                             const int* __restrict__ S, const double* __restrict__ xs, int ns,
                             double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  double s = 0.0;
  for (int j = 0; j < ns; ++j) s = fma(A[(size_t)S[j] * M + i], xs[j], s);
  r[i] = y[i] - s;
}

// H_jj += lambda_tsv d2(S_j) (TSV form)
__global__ void k_looe_tsv_diag(double* __restrict__ H, int ld, const int* __restrict__ S, int ns, int nx,
                                double lam) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const int pix = S[j], r = pix % nx, c = pix / nx;
  const bool ri = r > 0 && r < nx - 1, ci = c > 0 && c < nx - 1;
  const double d2 = ri ? (ci ? 8.0 : 6.0) : (ci ? 6.0 : 4.0);
  H[(size_t)j + (size_t)j * ld] += lam * d2;
}

// Cholesky of the nb x nb diagonal block at (k0, k0) in shared memory
// (lower triangle in and out); info = k0 + j + 1 at a pivot that is not > 0
__global__ void __launch_bounds__(256) k_looe_chol_diag(double* __restrict__ H, int ld, int k0, int nb,
                                                        int* __restrict__ info) {
  if (*info) return;
  __shared__ double a[kPanel][kPanel + 1];
  __shared__ int bad;
  const int t = threadIdx.x;
  double* blk = H + (size_t)k0 + (size_t)k0 * ld;
  for (int e = t; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    a[i][j] = i >= j ? blk[(size_t)i + (size_t)j * ld] : 0.0;
  }
  if (t == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    if (t == 0) {
      const double d = a[j][j];
      if (d > 0.0) a[j][j] = sqrt(d);
      else bad = j + 1;
    }
    __syncthreads();
    if (bad) {
      if (t == 0) *info = k0 + bad;
      return;
    }
    const double piv = a[j][j];
    for (int i = j + 1 + t; i < nb; i += blockDim.x) a[i][j] /= piv;
    __syncthreads();
    const int w = nb - j - 1;
    for (int e = t; e < w * w; e += blockDim.x) {
      const int ii = j + 1 + e % w, kk = j + 1 + e / w;
      if (ii >= kk) a[ii][kk] -= a[ii][j] * a[kk][j];
    }
    __syncthreads();
  }
  for (int e = t; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    if (i >= j) blk[(size_t)i + (size_t)j * ld] = a[i][j];
  }
}

// rows [r0, r1) of X (columns 0..nb-1, leading dimension ldx) := X L^-T,
// L the factored nb x nb diagonal block at Ld (ldl): one thread per row,
// forward substitution x_j = (x_j - sum_{p<j} x_p L_jp) / L_jj
__global__ void __launch_bounds__(256) k_looe_rowsolve(double* __restrict__ X, int ldx, int r0, int r1,
                                                       const double* __restrict__ Ld, int ldl, int nb,
                                                       const int* __restrict__ info) {
  if (*info) return;
  __shared__ double L[kPanel][kPanel + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    L[i][j] = i >= j ? Ld[(size_t)i + (size_t)j * ldl] : 0.0;
  }
  __syncthreads();
  const int i = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r1) return;
  double* row = X + i;
  for (int j = 0; j < nb; ++j) {
    double s = row[(size_t)j * ldx];
    for (int p = 0; p < j; ++p) s -= row[(size_t)p * ldx] * L[j][p];
    row[(size_t)j * ldx] = s / L[j][j];
  }
}

// per row i: d_i = |Z_i|^2 (columns in order), t = r_i / (1 - d_i),
// s = t^2 / 2; per-CTA partial sums of s and s^2
__global__ void __launch_bounds__(256) k_looe_terms(const double* __restrict__ Z, int M, int ns,
                                                    const double* __restrict__ r, double* __restrict__ part,
                                                    const int* __restrict__ info) {
  __shared__ double sh[2][256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0, s2 = 0.0;
  if (!*info && i < M) {
    double d = 0.0;
    for (int j = 0; j < ns; ++j) {
      const double z = Z[(size_t)j * M + i];
      d = fma(z, z, d);
    }
    const double tt = r[i] / (1.0 - d);
    s = tt * tt / 2;
    s2 = s * s;
  }
  sh[0][threadIdx.x] = s;
  sh[1][threadIdx.x] = s2;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sh[0][0];
    part[2 * blockIdx.x + 1] = sh[1][0];
  }
}

// out = (looe_m, looe_std, positive) from the partials, in block order
__global__ void k_looe_final(const double* __restrict__ part, int nblk, int M, const int* __restrict__ info,
                             double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (*info) {
    out[0] = 0.0;
    out[1] = 0.0;
    out[2] = 0.0;
    return;
  }
  double s = 0.0, s2 = 0.0;
  for (int b = 0; b < nblk; ++b) {
    s += part[2 * b];
    s2 += part[2 * b + 1];
  }
  const double m = s / M;
  const double var = s2 / (M - 1.0) - m * m * M / (M - 1.0);
  out[0] = m;
  out[1] = sqrt(var);
  out[2] = 1.0;
}

// Host driver: LOOE of B solutions X [B][N] of the DFT problem (y [M], A
// column-major M x N); lambda_tsv per solution (null: 0).  Kernels per
// solution: 5 (+1 TSV) + ceil(n_s/64) x (up to 5).
struct Looe {
  int M, N, NX;
  cudaStream_t s = nullptr;
  DevMem d_A, d_y, d_S, d_xs, d_r, d_Z, d_H, d_part, d_info, d_out;

  Looe(const double* y, const double* A, int M_, int N_, int NX_) : M(M_), N(N_), NX(NX_) {
    MF_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    d_A.upload(A, (size_t)M * N);
    d_y.upload(y, (size_t)M);
    d_r.alloc(sizeof(double) * M);
    d_part.alloc(sizeof(double) * 2 * (size_t)cdiv(M, 256));
    d_info.alloc(sizeof(int));
    d_out.alloc(sizeof(double) * 3);
    set_smem(k_looe_gemm<false, false>, kGemmSmem);
    set_smem(k_looe_gemm<false, true>, kGemmSmem);
    set_smem(k_looe_gemm<true, false>, kGemmSmem);
    set_smem(k_looe_gemm<true, true>, kGemmSmem);
  }
  ~Looe() {
    if (s) cudaStreamDestroy(s);
  }

  template <bool TA, bool TB>
  void gemm(int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb, double beta,
            double* C, int ldc, int lower) {
    if (m <= 0 || n <= 0) return;
    k_looe_gemm<TA, TB><<<dim3(cdiv(m, kGT), cdiv(n, kGT)), 256, kGemmSmem, s>>>(m, n, k, alpha, A, lda, B, ldb, beta,
                                                                                  C, ldc, lower, d_info.as<int>());
    MF_LAUNCH_CK();
  }

  // (looe_m, looe_std, positive) of one solution x [N]
  void one(const double* x, double lam_tsv, double out[3]) {
    std::vector<int> S;
    std::vector<double> xs;
    for (int j = 0; j < N; ++j)
      if (fabs(x[j]) > 0) {
        S.push_back(j);
        xs.push_back(x[j]);
      }
    const int ns = (int)S.size();
    if (ns > 0) {
      d_S.upload(S.data(), S.size());
      d_xs.upload(xs.data(), xs.size());
      if (d_Z.bytes < sizeof(double) * (size_t)M * ns) d_Z.alloc(sizeof(double) * (size_t)M * ns);
      if (d_H.bytes < sizeof(double) * (size_t)ns * ns) d_H.alloc(sizeof(double) * (size_t)ns * ns);
    }
    MF_CK(cudaMemsetAsync(d_info.p, 0, sizeof(int), s));
    double* Z = d_Z.as<double>();
    double* H = d_H.as<double>();
    const int* info = d_info.as<int>();
    k_looe_resid<<<cdiv(M, 256), 256, 0, s>>>(d_A.as<double>(), M, d_y.as<double>(), d_S.as<int>(),
                                                d_xs.as<double>(), ns, d_r.as<double>());
    MF_LAUNCH_CK();
    if (ns > 0) {
      k_looe_gather<<<ns, 256, 0, s>>>(d_A.as<double>(), M, d_S.as<int>(), Z);
      MF_LAUNCH_CK();
      gemm<true, false>(ns, ns, M, 1.0, Z, M, Z, M, 0.0, H, ns, 1);  // H = Z^T Z
      if (lam_tsv != 0.0) {
        k_looe_tsv_diag<<<cdiv(ns, 256), 256, 0, s>>>(H, ns, d_S.as<int>(), ns, NX, lam_tsv);
        MF_LAUNCH_CK();
      }
      for (int k0 = 0; k0 < ns; k0 += kPanel) {
        const int nb = std::min(kPanel, ns - k0), k1 = k0 + nb, rem = ns - k1;
        const double* Ld = H + k0 + (size_t)k0 * ns;
        k_looe_chol_diag<<<1, 256, 0, s>>>(H, ns, k0, nb, d_info.as<int>());
        MF_LAUNCH_CK();
        if (rem > 0) {
          k_looe_rowsolve<<<cdiv(rem, 256), 256, 0, s>>>(H + (size_t)k0 * ns, ns, k1, ns, Ld, ns, nb, info);
          MF_LAUNCH_CK();
          // trailing H22 -= L21 L21^T (lower tiles)
          gemm<false, true>(rem, rem, nb, -1.0, H + k1 + (size_t)k0 * ns, ns, H + k1 + (size_t)k0 * ns, ns, 1.0,
                            H + k1 + (size_t)k1 * ns, ns, 1);
        }
        // Z[:, k0:k1] := Z[:, k0:k1] L_kk^-T, then Z[:, k1:] -= Z[:, k0:k1] L21^T
        k_looe_rowsolve<<<cdiv(M, 256), 256, 0, s>>>(Z + (size_t)k0 * M, M, 0, M, Ld, ns, nb, info);
        MF_LAUNCH_CK();
        if (rem > 0)
          gemm<false, true>(M, rem, nb, -1.0, Z + (size_t)k0 * M, M, H + k1 + (size_t)k0 * ns, ns, 1.0,
                            Z + (size_t)k1 * M, M, 0);
      }
    }
    const int nblk = cdiv(M, 256);
    k_looe_terms<<<nblk, 256, 0, s>>>(Z, M, ns, d_r.as<double>(), d_part.as<double>(), info);
    MF_LAUNCH_CK();
    k_looe_final<<<1, 32, 0, s>>>(d_part.as<double>(), nblk, M, info, d_out.as<double>());
    MF_LAUNCH_CK();
    MF_CK(cudaMemcpyAsync(out, d_out.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
    MF_CK(cudaStreamSynchronize(s));
  }
};

}  // namespace looe
}  // namespace mf
