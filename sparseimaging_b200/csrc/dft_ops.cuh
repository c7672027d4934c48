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
