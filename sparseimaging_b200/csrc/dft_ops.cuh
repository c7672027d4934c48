// Operator of the DFT variant (c/mfista_dft_lib.c:30-66, :253-278): a dense
// real M x N column-major matrix A.
//   residual  r = y - A z            (calc_yAz, dgemv "N")
//   gradient  A^T r - lambda_tsv d_TSV(z)   (dF_dx, dgemv "T" with beta)
// FP64 GEMV kernels for the plain method: A z is split over column chunks
// (one CTA per 256 rows x chunk, deterministic second pass), A^T r is one
// warp per column with coalesced reads down the column.
#pragma once
#include "common.cuh"
#include "nufft_ops.cuh"  // dtsv_at / tsv_terms_at

namespace mf {

struct DftGeom {
  const double* A;   // column-major M x N (lda = M), shared by the batch
  const double* y;   // [M]
  int M, N;
  int nchunk, chunk; // column split of A z
  double* az_part;   // [B][nchunk][M]
  double* resid;     // [B][M]
};

__global__ void k_dft_az(DftGeom g, const double* __restrict__ zall, long xstride, const ProbState* __restrict__ st,
                         int gate) {
  int b = blockIdx.z;
  if (!gate_ok(st[b], gate)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  int c = blockIdx.y;
  int n0 = c * g.chunk, n1 = min(g.N, n0 + g.chunk);
  const double* z = zall + (size_t)b * xstride;
  extern __shared__ double zs[];
  for (int n = n0 + threadIdx.x; n < n1; n += blockDim.x) zs[n - n0] = z[n];
  __syncthreads();
  if (m >= g.M) return;
  double s = 0.0;
  const double* a = g.A + (size_t)n0 * g.M + m;
  for (int n = n0; n < n1; ++n, a += g.M) s += *a * zs[n - n0];
  g.az_part[((size_t)b * g.nchunk + c) * g.M + m] = s;
}

__global__ void k_dft_resid(DftGeom g, const ProbState* __restrict__ st, int gate, Partials part, int qchi,
                            int store) {
  __shared__ double sh[32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (m < g.M) {
    double s = 0.0;
    for (int c = 0; c < g.nchunk; ++c) s += g.az_part[((size_t)b * g.nchunk + c) * g.M + m];
    double r = g.y[m] - s;
    acc[0] = r * r;
    if (store) g.resid[(size_t)b * g.M + m] = r;
  }
  block_sum<1>(acc, sh);
  if (threadIdx.x == 0) part.at(qchi, b)[blockIdx.x] = acc[0];
}

// dfdx[n] = beta * dTSV(z)[n] + sum_m A[m + n M] r[m]  (beta = -lambda_tsv or 0)
__global__ void k_dft_atr(DftGeom g, double* __restrict__ dall, long xstride, const double* __restrict__ zall,
                          const ProbParams* __restrict__ prm, int tsvNX, int tsvNY, const ProbState* __restrict__ st,
                          int gate, Partials part, int qtsv) {
  __shared__ double sh[32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int n = blockIdx.x * nw + warp;
  const double* r = g.resid + (size_t)b * g.M;
  const ProbParams& pp = prm[b];
  bool fuse = zall != nullptr && pp.lambda_tsv > 0.0;
  double acc[1] = {0.0};
  if (n < g.N) {
    const double* col = g.A + (size_t)n * g.M;
    double s = 0.0;
    for (int m = lane; m < g.M; m += 32) s += col[m] * r[m];
    s = warp_sum(s);
    if (lane == 0) {
      double* d = dall + (size_t)b * xstride;
      if (fuse) {
        const double* z = zall + (size_t)b * xstride;
        d[n] = dtsv_at(z, n, tsvNX, tsvNY) * (-pp.lambda_tsv) + s;
        acc[0] = tsv_terms_at(z, n, tsvNX, tsvNY);
      } else {
        d[n] = s;
      }
    }
  }
  if (qtsv >= 0) {
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part.at(qtsv, b)[blockIdx.x] = acc[0];
  }
}

}  // namespace mf

// ===========================================================================
// Batched DFT (B problems share A): A Z and A^T R as register-blocked FP64
// GEMMs with split-K; each CTA computes a 64 x 64 (rows x problems) tile.
// Results are per-K-chunk partials summed in a fixed order afterwards, so
// the batched path is deterministic like the GEMV path.
// ===========================================================================
namespace mf {

constexpr int kGT = 64;   // tile edge (rows and problems)
constexpr int kGK = 16;   // K step staged in shared memory

// does any problem b0 .. b0 + kGT - 1 pass the gate?  (uniform over the CTA)
__device__ __forceinline__ bool tile_active(const ProbState* __restrict__ st, int gate, int b0, int B) {
  __shared__ int s_any;
  if (threadIdx.x == 0) {
    int any = 0;
    for (int i = 0; i < kGT && b0 + i < B; ++i) any |= gate_ok(st[b0 + i], gate) ? 1 : 0;
    s_any = any;
  }
  __syncthreads();
  return s_any != 0;
}

// az_part[b][chunk][m] = sum_{n in chunk} A[m + n M] z_b[n]
__global__ void __launch_bounds__(256) k_dft_az_gemm(DftGeom g, const double* __restrict__ zall, long xstride,
                                                     const ProbState* __restrict__ st, int gate, int B) {
  __shared__ double sA[kGK][kGT + 1];
  __shared__ double sZ[kGK][kGT + 1];
  const int m0 = blockIdx.x * kGT, b0 = blockIdx.z * kGT, c = blockIdx.y;
  if (!tile_active(st, gate, b0, B)) return;  // no problem of this tile: skip reading A
  const int n0 = c * g.chunk, n1 = min(g.N, n0 + g.chunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 4 x 4 outputs each
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int k0 = n0; k0 < n1; k0 += kGK) {
    for (int t = threadIdx.x; t < kGK * kGT; t += 256) {
      int kk = t / kGT, r = t - kk * kGT;
      int n = k0 + kk, m = m0 + r, b = b0 + r;
      sA[kk][r] = (n < n1 && m < g.M) ? g.A[(size_t)n * g.M + m] : 0.0;
      bool ok = n < n1 && b < B && gate_ok(st[b], gate);
      sZ[kk][r] = ok ? zall[(size_t)b * xstride + n] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      double a[4], z[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) z[j] = sZ[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * z[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int b = b0 + tx + 16 * j;
    if (b >= B || !gate_ok(st[b], gate)) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int m = m0 + ty + 16 * i;
      if (m < g.M) g.az_part[((size_t)b * g.nchunk + c) * g.M + m] = acc[i][j];
    }
  }
}

// atr_part[b][chunk][n] = sum_{m in chunk} A[m + n M] r_b[m]
__global__ void __launch_bounds__(256) k_dft_atr_gemm(DftGeom g, double* __restrict__ atr_part, int mchunk,
                                                      int nmchunk, const ProbState* __restrict__ st, int gate,
                                                      int B) {
  __shared__ double sA[kGK][kGT + 1];
  __shared__ double sR[kGK][kGT + 1];
  const int nn0 = blockIdx.x * kGT, b0 = blockIdx.z * kGT, c = blockIdx.y;
  if (!tile_active(st, gate, b0, B)) return;
  const int ms = c * mchunk, me = min(g.M, ms + mchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int k0 = ms; k0 < me; k0 += kGK) {
    // A is column-major: 16 consecutive rows of column n are contiguous
    for (int t = threadIdx.x; t < kGK * kGT; t += 256) {
      int r = t / kGK, kk = t - r * kGK;
      int m = k0 + kk, n = nn0 + r, b = b0 + r;
      sA[kk][r] = (m < me && n < g.N) ? g.A[(size_t)n * g.M + m] : 0.0;
      bool ok = m < me && b < B && gate_ok(st[b], gate);
      sR[kk][r] = ok ? g.resid[(size_t)b * g.M + m] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      double a[4], r[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) r[j] = sR[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * r[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int b = b0 + tx + 16 * j;
    if (b >= B || !gate_ok(st[b], gate)) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int n = nn0 + ty + 16 * i;
      if (n < g.N) atr_part[((size_t)b * nmchunk + c) * g.N + n] = acc[i][j];
    }
  }
}

// dfdx[n] = beta dTSV(z)[n] + sum_chunks atr_part[b][c][n]
__global__ void k_dft_atr_finish(DftGeom g, const double* __restrict__ atr_part, int nmchunk,
                                 double* __restrict__ dall, long xstride, const double* __restrict__ zall,
                                 const ProbParams* __restrict__ prm, int tsvNX, int tsvNY,
                                 const ProbState* __restrict__ st, int gate) {
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.N) return;
  double s = 0.0;
  for (int c = 0; c < nmchunk; ++c) s += atr_part[((size_t)b * nmchunk + c) * g.N + n];
  const ProbParams& pp = prm[b];
  double* d = dall + (size_t)b * xstride;
  if (zall != nullptr && pp.lambda_tsv > 0.0) {
    const double* z = zall + (size_t)b * xstride;
    d[n] = dtsv_at(z, n, tsvNX, tsvNY) * (-pp.lambda_tsv) + s;
  } else {
    d[n] = s;
  }
}

}  // namespace mf

// ===========================================================================
// Split-BF16 tensor-core form (tc::k_gemm_bf16x3) with FP64 defect
// correction: for an anchor x_a (refreshed in FP64 every few outer
// iterations) with ax_a = A x_a, r_a = y - ax_a and g_a = A^T r_a,
//   A v   = ax_a + A (v - x_a)            (tensor-core part: A (v - x_a))
//   A^T r = g_a  + A^T (r - r_a)          (tensor-core part: A^T (r - r_a))
// so the low-precision products only carry the (small) departures from the
// anchor.  Partials arrive per K split as FP32 [nsplit][bpad][rows] and are
// summed in a fixed order in FP64.
// ===========================================================================
namespace mf {

// r = y - (ax_a + sum_s part[s]) ; chi^2 partials; r stored when `store`
__global__ void k_dft_tc_resid(const float* __restrict__ part, int nsplit, int bpad, int rows,
                               const double* __restrict__ axa, DftGeom g, const ProbState* __restrict__ st, int gate,
                               Partials pq, int qchi, int store) {
  __shared__ double sh[32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (m < g.M) {
    double s = axa[(size_t)b * g.M + m];
    for (int k = 0; k < nsplit; ++k) s += (double)part[((size_t)k * bpad + b) * rows + m];
    double r = g.y[m] - s;
    acc[0] = r * r;
    if (store) g.resid[(size_t)b * g.M + m] = r;
  }
  block_sum<1>(acc, sh);
  if (threadIdx.x == 0 && qchi >= 0) pq.at(qchi, b)[blockIdx.x] = acc[0];
}

// dfdx[n] = beta dTSV(z)[n] + g_a[n] + sum_s part[s][n]   (beta = -lambda_tsv or 0)
__global__ void k_dft_tc_atr_finish(const float* __restrict__ part, int nsplit, int bpad, int rows,
                                    const double* __restrict__ ga, int N, double* __restrict__ dall, long xstride,
                                    const double* __restrict__ zall, const ProbParams* __restrict__ prm, int tsvNX,
                                    int tsvNY, const ProbState* __restrict__ st, int gate) {
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double s = ga[(size_t)b * N + n];
  for (int k = 0; k < nsplit; ++k) s += (double)part[((size_t)k * bpad + b) * rows + n];
  const ProbParams& pp = prm[b];
  double* d = dall + (size_t)b * xstride;
  if (zall != nullptr && pp.lambda_tsv > 0.0) {
    const double* z = zall + (size_t)b * xstride;
    d[n] = dtsv_at(z, n, tsvNX, tsvNY) * (-pp.lambda_tsv) + s;
  } else {
    d[n] = s;
  }
}

// anchor model from the FP64 GEMM partials: ax_a = sum_c az_part, r_a = y - ax_a
__global__ void k_dft_anchor(DftGeom g, const ProbState* __restrict__ st, int gate, double* __restrict__ axa,
                             double* __restrict__ ra) {
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= g.M) return;
  double s = 0.0;
  for (int c = 0; c < g.nchunk; ++c) s += g.az_part[((size_t)b * g.nchunk + c) * g.M + m];
  axa[(size_t)b * g.M + m] = s;
  ra[(size_t)b * g.M + m] = g.y[m] - s;
}

}  // namespace mf
