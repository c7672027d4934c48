// Forward NUFFT of the reference's C++ build (x2y_nufft, c++/mfista_nufft_lib.cpp:1076-1149).
//
// It differs from the C library's operator in its kernel and binning
// (c++/mfista.hpp:32-35, preNUFFT :85-187): MSP = 6, so 12 taps per axis;
// points with v < 0 are flipped to (-u, -v) and their result conjugated;
// m = floor(u 2N / 2 pi); one Gaussian width tau = MSP / Nx^2 for both
// axes; the E3 factor folded into E2; E4 centred on (Nx/2, Ny/2) with
// coefficient Nx Ny pi / MSP.  The padding (small2large :46-77) is the C
// library's centring, so the row and column FFT passes of NufftOp serve
// with this E4.  NUFFT2d2 (:440-504) then reads a half-plane buffer whose
// ky < 0 halo rows are the Hermitian images of ky > 0 for kx in
// [1 - Nx, Nx - 1], with everything else outside the half plane zero; here
// those rules are applied per tap instead of filling a buffer.
#pragma once

#include "solver.cuh"

namespace mf {
namespace cppnufft {

constexpr int kMSP = 6;
constexpr int kW = 2 * kMSP;  // taps per axis

// preNUFFT of the C++ build, on the host in FP64 (same expressions)
struct Prep {
  std::vector<int> mx, my, yneg;
  std::vector<double> e1, e2x, e2y, e4;  // e2*: [M][12]
  Prep(const double* u, const double* v, int M, int Nx, int Ny)
      : mx(M), my(M), yneg(M), e1(M), e2x((size_t)M * kW), e2y((size_t)M * kW), e4((size_t)Nx * Ny) {
    const double pi = M_PI;
    const double mrx = 2.0 * Nx, mry = 2.0 * Ny;
    const double tau = (double)kMSP / (double)(Nx * Nx);
    const double coeff = (double)(Nx * Ny) * pi / (double)kMSP;
    const double t3x = (pi * pi) / (mrx * mrx * tau), t3y = (pi * pi) / (mry * mry * tau);
    double c[kW];
    for (int j = 0; j < kW; ++j) c[j] = (double)(j - kMSP + 1);
    for (int k = 0; k < M; ++k) {
      double uk = u[k], vk = v[k];
      yneg[k] = v[k] >= 0 ? 0 : 1;
      if (yneg[k]) {
        uk *= -1.0;
        vk *= -1.0;
      }
      const double fx = floor(uk * mrx / (2.0 * pi)), fy = floor(vk * mry / (2.0 * pi));
      mx[k] = (int)fx;
      my[k] = (int)fy;
      const double xix = (2.0 * pi * fx) / mrx, xiy = (2.0 * pi * fy) / mry;
      e1[k] = exp(-((uk - xix) * (uk - xix)) / (4.0 * tau) - ((vk - xiy) * (vk - xiy)) / (4.0 * tau));
      const double t4x = pi * (uk - xix) / (mrx * tau), t4y = pi * (vk - xiy) / (mry * tau);
      for (int j = 0; j < kW; ++j) {
        e2x[(size_t)k * kW + j] = exp(c[j] * (t4x - c[j] * t3x));
        e2y[(size_t)k * kW + j] = exp(c[j] * (t4y - c[j] * t3y));
      }
    }
    for (int i = 0; i < Nx; ++i) {
      const double ti = (double)(i - Nx / 2), tx = tau * ti * ti;
      for (int j = 0; j < Ny; ++j) {
        const double tj = (double)(j - Ny / 2);
        e4[(size_t)i * Ny + j] = coeff * exp(tx + tau * tj * tj);
      }
    }
  }
};

// One warp per point, 144 taps over the lanes; G is the half-plane grid
// [2Nx][Ny+1] (row kx mod 2Nx, column ky).  F = conj(E1 s) scale, conjugated
// once more for flipped points.
__global__ void __launch_bounds__(256) k_cpp_interp(const cplx<double>* __restrict__ G, int nx, int ny,
                                                    const int* __restrict__ mx, const int* __restrict__ my,
                                                    const int* __restrict__ yneg, const double* __restrict__ e1,
                                                    const double* __restrict__ e2x, const double* __restrict__ e2y,
                                                    int M, double scale, double* __restrict__ out_r,
                                                    double* __restrict__ out_i) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (k >= M) return;
  const int mxk = mx[k], myk = my[k];
  double sr = 0.0, si = 0.0;
  for (int t = lane; t < kW * kW; t += 32) {
    const int a = t / kW, b = t - a * kW;  // a: y tap, b: x tap
    const int kx = mxk + b - (kMSP - 1), ky = myk + a - (kMSP - 1);
    double gr = 0.0, gi = 0.0;
    if (ky >= 0 && ky <= ny && kx >= -nx && kx < nx) {
      const cplx<double> g = G[(size_t)(kx < 0 ? kx + 2 * nx : kx) * (ny + 1) + ky];
      gr = g.x;
      gi = g.y;
    } else if (ky < 0 && kx >= 1 - nx && kx <= nx - 1) {  // Hermitian halo
      const int rx = -kx;
      const cplx<double> g = G[(size_t)(rx < 0 ? rx + 2 * nx : rx) * (ny + 1) + (-ky)];
      gr = g.x;
      gi = -g.y;
    }
    const double w = e2y[(size_t)k * kW + a] * e2x[(size_t)k * kW + b];
    sr += w * gr;
    si += w * gi;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o);
    si += __shfl_xor_sync(0xffffffffu, si, o);
  }
  if (lane == 0) {
    const double f = e1[k] * scale;
    out_r[k] = sr * f;
    out_i[k] = (yneg[k] ? si : -si) * f;
  }
}

}  // namespace cppnufft
}  // namespace mf
