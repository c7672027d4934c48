// Operator of the gridded (FFT) variant (c/mfista_fft_lib.c:27-175):
//   F(x)  = 1/4 |full-plane (yf - mask .* FFT2(x)/sqrt(N))|^2
//   dF/dx = c2r(residual .* mask / (2 sqrt(N)))
// on an NX x NY image with an NX x (NY/2+1) half spectrum.  The full-plane
// norm of fft_half2full (:27-48) is evaluated on the half spectrum with
// column weights 1 (DC and Nyquist columns) and 2 (columns mirrored by it).
// NY must be even (for odd NY the reference reads unset entries of its
// full-plane buffer).
#pragma once
#include "common.cuh"
#include "fft_smem.cuh"

namespace mf {

struct FftVarGeom {
  const double* mask_h;   // [NX*NYh] per problem (stride geo_stride, 0 = shared)
  const double2* yf_h;    // [NX*NYh]
  long geo_stride;
};

// real FFT of every image row (length NY as NY/2 complex points); with
// `sub` (the FP64 anchor images of the corrected FP32 form) the rows of
// x - sub are transformed
template <typename T>
__global__ void k_fftv_rows_fwd(const double* __restrict__ xall, long xstride, cplx<T>* __restrict__ hall,
                                long hstride, int nx, int ny, FftDev<T> fh, const cplx<T>* __restrict__ tw2h,
                                const ProbState* __restrict__ st, int gate, int rows_per_cta,
                                const double* __restrict__ suball) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const int h = ny / 2, ld = h + 1, nyh = h + 1;
  cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* Bf = A + (size_t)rows_per_cta * ld;
  const double* x = xall + (size_t)b * xstride;
  cplx<T>* H = hall + (size_t)b * hstride;
  int i0 = blockIdx.x * rows_per_cta;
  int nrows = min(rows_per_cta, nx - i0);
  const double* sub = suball ? suball + (size_t)b * xstride : nullptr;
  for (int t = threadIdx.x; t < nrows * h; t += blockDim.x) {
    int rr = t / h, m = t - rr * h;
    const size_t f = (size_t)(i0 + rr) * ny + 2 * m;
    double x0 = x[f], x1 = x[f + 1];
    if (sub) {
      x0 -= sub[f];
      x1 -= sub[f + 1];
    }
    A[rr * ld + m] = mk<T>((T)x0, (T)x1);
  }
  __syncthreads();
  cplx<T>* Z = smem_fft<T>(A, Bf, fh, ld, nrows, -1);
  for (int t = threadIdx.x; t < nrows * nyh; t += blockDim.x) {
    int rr = t / nyh, k = t - rr * nyh;
    cplx<T> zk = Z[rr * ld + (k == h ? 0 : k)];
    cplx<T> zc = cconj<T>(Z[rr * ld + (k == 0 ? 0 : h - k)]);
    cplx<T> e = cadd<T>(zk, zc);
    cplx<T> wo = cmul_si<T>(cmul<T>(tw2h[k], csub<T>(zk, zc)), -1);
    H[(size_t)(i0 + rr) * nyh + k] = mk<T>(T(0.5) * (e.x + wo.x), T(0.5) * (e.y + wo.y));
  }
}

// column FFT (length NX) over the half spectrum; forward pass fuses
// calc_yAx_fft (:116-130), the weighted norm and, in gradient mode, the
// mask / (2 sqrt N) scaling of dF_dx_fft (:170).  Corrected FP32 form: the
// spectrum is base + FFT(x - x_a) with base the exact FP64 spectrum of the
// anchor (added in FP64 before the residual); raw_out (forward, qchi < 0)
// stores the FP64 spectrum itself (the anchor refresh of the exact operator).
template <typename T>
__global__ void k_fftv_cols(cplx<T>* __restrict__ hall, long hstride, int nx, int nyh, FftDev<T> fnx, int sign,
                            int cols_per_cta, FftVarGeom geo, double sqrtn, const ProbState* __restrict__ st,
                            int gate, Partials part, int qchi, int store_grad, const double2* __restrict__ base,
                            double2* __restrict__ raw_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sh[32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const int ld = nx + 1;
  cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* Bf = A + (size_t)cols_per_cta * ld;
  cplx<T>* H = hall + (size_t)b * hstride;
  int c0 = blockIdx.x * cols_per_cta;
  int nc = min(cols_per_cta, nyh - c0);
  for (int t = threadIdx.x; t < nx * cols_per_cta; t += blockDim.x) {
    int r = t / cols_per_cta, cc = t - r * cols_per_cta;
    if (cc >= nc) continue;
    A[cc * ld + r] = H[(size_t)r * nyh + c0 + cc];
  }
  __syncthreads();
  cplx<T>* R = smem_fft<T>(A, Bf, fnx, ld, nc, sign);
  double acc[1] = {0.0};
  const double* mask = geo.mask_h + (size_t)b * geo.geo_stride;
  const double2* yf = geo.yf_h + (size_t)b * geo.geo_stride;
  for (int t = threadIdx.x; t < nx * cols_per_cta; t += blockDim.x) {
    int r = t / cols_per_cta, cc = t - r * cols_per_cta;
    if (cc >= nc) continue;
    int k = c0 + cc;
    size_t e = (size_t)r * nyh + k;
    cplx<T> v = R[cc * ld + r];
    if (raw_out) {
      raw_out[(size_t)b * hstride + e] = make_double2((double)v.x, (double)v.y);
    } else if (qchi >= 0) {
      double mk_ = mask[e];
      double2 y = yf[e];
      double vx = (double)v.x, vy = (double)v.y;
      if (base) {
        const double2 a = base[(size_t)b * hstride + e];
        vx += a.x;
        vy += a.y;
      }
      double rr = y.x - mk_ * vx / sqrtn;
      double ri = y.y - mk_ * vy / sqrtn;
      double w = (k == 0 || k == nyh - 1) ? 1.0 : 2.0;
      acc[0] += w * (rr * rr + ri * ri);
      if (store_grad) {
        double s = mk_ / (2 * sqrtn);
        H[e] = mk<T>((T)(rr * s), (T)(ri * s));
      }
    } else {
      H[e] = v;
    }
  }
  if (qchi >= 0) {
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part.at(qchi, b)[blockIdx.x] = acc[0];
  }
}

// half-complex -> real FFT of every row (c2r, unnormalised) to dfdx, with
// the TSV gradient of z folded in (c/mfista_fft_lib.c:504-511)
template <typename T>
__global__ void k_fftv_rows_inv(const cplx<T>* __restrict__ hall, long hstride, double* __restrict__ dall,
                                long xstride, int nx, int ny, FftDev<T> fh, const cplx<T>* __restrict__ tw2h,
                                const double* __restrict__ zall, const ProbParams* __restrict__ prm,
                                int tsvNX, int tsvNY, Partials part, int qtsv, const ProbState* __restrict__ st,
                                int gate, int rows_per_cta);

}  // namespace mf

#include "nufft_ops.cuh"  // dtsv_at / tsv_terms_at

namespace mf {

template <typename T>
__global__ void k_fftv_rows_inv(const cplx<T>* __restrict__ hall, long hstride, double* __restrict__ dall,
                                long xstride, int nx, int ny, FftDev<T> fh, const cplx<T>* __restrict__ tw2h,
                                const double* __restrict__ zall, const ProbParams* __restrict__ prm,
                                int tsvNX, int tsvNY, Partials part, int qtsv, const ProbState* __restrict__ st,
                                int gate, int rows_per_cta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sh[32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const int h = ny / 2, ld = h + 1, nyh = h + 1;
  cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* Bf = A + (size_t)rows_per_cta * ld;
  const cplx<T>* H = hall + (size_t)b * hstride;
  double* dfdx = dall + (size_t)b * xstride;
  int i0 = blockIdx.x * rows_per_cta;
  int nrows = min(rows_per_cta, nx - i0);
  for (int t = threadIdx.x; t < nrows * h; t += blockDim.x) {
    int rr = t / h, k = t - rr * h;
    const cplx<T>* hr = H + (size_t)(i0 + rr) * nyh;
    cplx<T> xk = hr[k];
    cplx<T> xc = hr[h - k];
    if (k == 0) {
      xk.y = 0;
      xc.y = 0;
    }
    xc = cconj<T>(xc);
    cplx<T> e = cadd<T>(xk, xc);
    cplx<T> o = cmul_si<T>(cmul<T>(cconj<T>(tw2h[k]), csub<T>(xk, xc)), 1);
    A[rr * ld + k] = cadd<T>(e, o);
  }
  __syncthreads();
  cplx<T>* Z = smem_fft<T>(A, Bf, fh, ld, nrows, +1);
  const ProbParams& pp = prm[b];
  bool fuse = zall != nullptr && pp.lambda_tsv > 0.0;
  const double* z = fuse ? zall + (size_t)b * xstride : nullptr;
  double acc[1] = {0.0};
  for (int t = threadIdx.x; t < nrows * ny; t += blockDim.x) {
    int rr = t / ny, j = t - rr * ny;
    cplx<T> zc = Z[rr * ld + (j >> 1)];
    double d = (double)((j & 1) ? zc.y : zc.x);
    int f = (i0 + rr) * ny + j;
    if (fuse) {
      d = d + dtsv_at(z, f, tsvNX, tsvNY) * (-pp.lambda_tsv);
      acc[0] += tsv_terms_at(z, f, tsvNX, tsvNY);
    }
    dfdx[f] = d;
  }
  if (qtsv >= 0) {
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part.at(qtsv, b)[blockIdx.x] = acc[0];
  }
}

}  // namespace mf
