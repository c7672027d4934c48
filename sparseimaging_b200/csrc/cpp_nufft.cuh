// NUFFT operators of the reference's C++ build: forward x2y_nufft
// (c++/mfista_nufft_lib.cpp:1076-1149, NUFFT2d2 :440-504) and adjoint
// y2x_nufft (:1151-1219, NUFFT2d1_sngl :189-258), and an Op for the solver.
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


// ---------------------------------------------------------------------------
// Adjoint (NUFFT2d1_sngl, :189-258) as a deterministic gather.
//
// The reference scatters v0 E2x E2y over each point's 12 x 12 block of a
// buffer with MSP-wide halos, then folds the halos back:
//   (a) taps at ky < 0 land, conjugated, on (-kx, -ky) -- kx = -Nx maps to
//       itself (:220-228);
//   (b) on the ky = 0 and ky = Ny columns, kx and -kx (kx != 0, -Nx) receive
//       each other's conjugate (:231-245);
//   (c) the DC cell is doubled (:248);
// and taps with kx outside [-Nx, Nx) or ky > Ny are dropped.  Here every
// cell of the [2Nx][Ny+1] half-plane grid sums, over the points binned to
// its 16 x 16 tile in increasing point order, the direct tap and the folded
// ones that reach it.  v0 = E1 (y_neg ? y : conj y) / (8 Nx Ny).
// ---------------------------------------------------------------------------
constexpr int kGTile = 16;

// tiles of the gather grid touched by point k's direct and folded taps
inline void bin_gather(const Prep& pr, int M, int nx, int ny, std::vector<int>& ptr, std::vector<int>& pts) {
  const int ntr = (2 * nx + kGTile - 1) / kGTile, ntc = (ny + 1 + kGTile - 1) / kGTile;
  std::vector<std::vector<int>> lists((size_t)ntr * ntc);
  std::vector<int> ids;
  auto add = [&](int kx, int ky) {
    const int r = kx < 0 ? kx + 2 * nx : kx;
    ids.push_back((r / kGTile) * ntc + ky / kGTile);
  };
  for (int k = 0; k < M; ++k) {
    ids.clear();
    for (int a = 0; a < kW; ++a) {
      const int ky = pr.my[k] + a - (kMSP - 1);
      if (ky > ny) continue;
      for (int b = 0; b < kW; ++b) {
        const int kx = pr.mx[k] + b - (kMSP - 1);
        if (kx < -nx || kx >= nx) continue;
        if (ky >= 0) {
          add(kx, ky);
          if ((ky == 0 || ky == ny) && kx != 0 && kx != -nx) add(-kx, ky);
        } else {
          add(kx == -nx ? -nx : -kx, -ky);
        }
      }
    }
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    for (int t : ids) lists[t].push_back(k);
  }
  ptr.assign(1, 0);
  pts.clear();
  for (auto& l : lists) {
    pts.insert(pts.end(), l.begin(), l.end());
    ptr.push_back((int)pts.size());
  }
}

// grid: (tiles, B); 256 threads, one cell each.  y: [B][ystride] complex
// visibilities (the weighted residual in the solver)
__global__ void __launch_bounds__(256) k_cpp_gather(
    cplx<double>* __restrict__ gall, long gstride, int nx, int ny, const int* __restrict__ tptr,
    const int* __restrict__ tpts, const int* __restrict__ mx, const int* __restrict__ my,
    const int* __restrict__ yneg, const double* __restrict__ e1, const double* __restrict__ e2x,
    const double* __restrict__ e2y, const double2* __restrict__ yall, long ystride, double scale,
    const ProbState* __restrict__ st, int gate) {
  const int b = blockIdx.y;
  if (st && !gate_ok(st[b], gate)) return;
  const int ntc = (ny + 1 + kGTile - 1) / kGTile;
  const int t = blockIdx.x;
  const int r = (t / ntc) * kGTile + (threadIdx.x >> 4);
  const int Y = (t % ntc) * kGTile + (threadIdx.x & 15);
  if (r >= 2 * nx || Y > ny) return;
  const int X = r < nx ? r : r - 2 * nx;
  const double2* y = yall + (size_t)b * ystride;
  const bool colfold = (Y == 0 || Y == ny) && X != 0 && X != -nx;
  const bool mirror = Y >= 1 && Y <= kMSP - 1;
  const int Xm = X == -nx ? -nx : -X;
  double ar = 0.0, ai = 0.0;
  for (int q = tptr[t]; q < tptr[t + 1]; ++q) {
    const int k = tpts[q];
    const int mxk = mx[k], myk = my[k];
    const double2 f = y[k];
    const double s = e1[k] * scale;
    // v0 = s * (y_neg ? y : conj y)
    const double vr = s * f.x, vi = s * (yneg[k] ? f.y : -f.y);
    const double* ex = e2x + (size_t)k * kW;
    const double* ey = e2y + (size_t)k * kW;
    const int ay = Y - myk + (kMSP - 1);
    if (ay >= 0 && ay < kW) {
      const int bx = X - mxk + (kMSP - 1);
      if (bx >= 0 && bx < kW) {
        double w = ex[bx] * ey[ay];
        if (X == 0 && Y == 0) w *= 2.0;
        ar += vr * w;
        ai += vi * w;
      }
      if (colfold) {
        const int bx2 = -X - mxk + (kMSP - 1);
        if (bx2 >= 0 && bx2 < kW) {
          const double w = ex[bx2] * ey[ay];
          ar += vr * w;
          ai -= vi * w;
        }
      }
    }
    if (mirror) {
      const int ay3 = -Y - myk + (kMSP - 1), bx3 = Xm - mxk + (kMSP - 1);
      if (ay3 >= 0 && ay3 < kW && bx3 >= 0 && bx3 < kW) {
        const double w = ex[bx3] * ey[ay3];
        ar += vr * w;
        ai -= vi * w;
      }
    }
  }
  gall[(size_t)b * gstride + (size_t)r * (ny + 1) + Y] = mk<double>(ar, ai);
}

// Forward with the solver's residual (calc_F_part_nufft :506-531): one warp
// per point; r = (vis - A x) w, chi^2 partials |r|^2 per CTA (8 points, in
// warp order) into part[qchi]; with `y2` the adjoint's input r w
// (dF_dx_nufft :533-548) is stored [B][M].
__global__ void __launch_bounds__(256) k_cpp_interp_resid(
    const cplx<double>* __restrict__ gall, long gstride, int nx, int ny, const int* __restrict__ mx,
    const int* __restrict__ my, const int* __restrict__ yneg, const double* __restrict__ e1,
    const double* __restrict__ e2x, const double* __restrict__ e2y, int M, double scale,
    const double* __restrict__ vis_r, const double* __restrict__ vis_i, const double* __restrict__ wgt,
    const ProbState* __restrict__ st, int gate, Partials part, int qchi, double2* __restrict__ y2) {
  __shared__ double sh[8];
  const int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = blockIdx.x * 8 + warp;
  const cplx<double>* G = gall + (size_t)b * gstride;
  double chi = 0.0;
  if (k < M) {
    const int mxk = mx[k], myk = my[k];
    double sr = 0.0, si = 0.0;
    for (int t = lane; t < kW * kW; t += 32) {
      const int a = t / kW, c = t - a * kW;
      const int kx = mxk + c - (kMSP - 1), ky = myk + a - (kMSP - 1);
      double gr = 0.0, gi = 0.0;
      if (ky >= 0 && ky <= ny && kx >= -nx && kx < nx) {
        const cplx<double> g = G[(size_t)(kx < 0 ? kx + 2 * nx : kx) * (ny + 1) + ky];
        gr = g.x;
        gi = g.y;
      } else if (ky < 0 && kx >= 1 - nx && kx <= nx - 1) {
        const int rx = -kx;
        const cplx<double> g = G[(size_t)(rx < 0 ? rx + 2 * nx : rx) * (ny + 1) + (-ky)];
        gr = g.x;
        gi = -g.y;
      }
      const double w = e2y[(size_t)k * kW + a] * e2x[(size_t)k * kW + c];
      sr += w * gr;
      si += w * gi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    const double f = e1[k] * scale;
    const double fr = sr * f, fi = (yneg[k] ? si : -si) * f;
    const double w = wgt[k];
    const double rr = (vis_r[k] - fr) * w, ri = (vis_i[k] - fi) * w;
    chi = rr * rr + ri * ri;
    if (y2 && lane == 0) y2[(size_t)b * M + k] = make_double2(rr * w, ri * w);
  }
  if (lane == 0) sh[warp] = chi;
  __syncthreads();
  if (threadIdx.x == 0 && qchi >= 0) {
    double s = 0.0;
    for (int q = 0; q < 8; ++q) s += sh[q];
    part.at(qchi, b)[blockIdx.x] = s;
  }
}

// The C++ build's operator for the solver (FP64; B problems sharing the
// points, e.g. a lambda grid).  The padded FFT passes are NufftOp's (same
// centring, small2large :46-77 / large2small :18-44) with the C++ E4.
struct CppNufftOp : Op {
  Ctx& c;
  int nx, ny, M, B;
  std::unique_ptr<NufftOp<double>> fft;  // grid, FFT plans and launch shapes
  DevMem d_mx, d_my, d_yn, d_e1, d_e2x, d_e2y, d_e4, d_vr, d_vi, d_w, d_y2, d_tptr, d_tpts;
  int ntiles = 0;
  double scale_fwd = 0, scale_adj = 0;

  CppNufftOp(Ctx& ctx, const double* u, const double* v, const double* vis_r, const double* vis_i,
             const double* vis_std, int M_, int Nx, int Ny)
      : c(ctx), nx(Nx), ny(Ny), M(M_), B(ctx.B) {
    if (M < 1 || nx < 12 || ny < 12) throw Error(MFISTA_ERR_ARG, "the C++-build NUFFT needs M >= 1, Nx, Ny >= 12");
    Prep pr(u, v, M, nx, ny);
    std::vector<double> zero(M, 0.0), one(M, 1.0);
    NufftInput in{u, v, zero.data(), zero.data(), one.data(), nullptr, 1, M, nx, ny};
    fft.reset(new NufftOp<double>(ctx, in));
    d_e4.upload(pr.e4.data(), pr.e4.size());
    d_mx.upload(pr.mx.data(), M);
    d_my.upload(pr.my.data(), M);
    d_yn.upload(pr.yneg.data(), M);
    d_e1.upload(pr.e1.data(), M);
    d_e2x.upload(pr.e2x.data(), pr.e2x.size());
    d_e2y.upload(pr.e2y.data(), pr.e2y.size());
    std::vector<double> w(M);
    for (int k = 0; k < M; ++k) w[k] = 1.0 / vis_std[k];
    d_vr.upload(vis_r, M);
    d_vi.upload(vis_i, M);
    d_w.upload(w.data(), M);
    d_y2.alloc(sizeof(double2) * (size_t)B * M);
    std::vector<int> ptr, pts;
    bin_gather(pr, M, nx, ny, ptr, pts);
    ntiles = (int)ptr.size() - 1;
    d_tptr.upload(ptr.data(), ptr.size());
    d_tpts.upload(pts.data(), std::max<size_t>(pts.size(), 1));
    scale_fwd = 1.0 / (4.0 * (double)nx * (double)ny);
    scale_adj = 1.0 / (8.0 * (double)nx * (double)ny);
    MF_CK(cudaDeviceSynchronize());
  }

  double2* y2() { return d_y2.as<double2>(); }

  // grid of B problems: rows pass (pad, C++ E4) and forward columns
  void grid_forward(cudaStream_t s, const double* src, int gate) {
    k_nufft_rows_fwd<double><<<dim3(cdiv(nx, fft->rpc), B), 256, fft->smem_rows, s>>>(
        src, c.xstride, d_e4.as<double>(), fft->d_grid.as<cplx<double>>(), fft->gstride, nx, ny, fft->fh.dev,
        fft->tw2h.as<cplx<double>>(), c.st, gate, fft->rpc, nullptr, DynUnits{nullptr, 0});
    MF_LAUNCH_CK();
    fft->launch_cols_fwd(s, gate);
  }

  void forward(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    grid_forward(s, src, gate);
    k_cpp_interp_resid<<<dim3(cdiv(M, 8), B), 256, 0, s>>>(
        fft->d_grid.as<cplx<double>>(), fft->gstride, nx, ny, d_mx.as<int>(), d_my.as<int>(), d_yn.as<int>(),
        d_e1.as<double>(), d_e2x.as<double>(), d_e2y.as<double>(), M, scale_fwd, d_vr.as<double>(),
        d_vi.as<double>(), d_w.as<double>(), c.st, gate, c.part, qchi, store ? y2() : nullptr);
    MF_LAUNCH_CK();
  }

  // gather of y2 into the grid, inverse columns, rows c2r (unpad, C++ E4;
  // the reference's large2small applies E4 without further scaling)
  void adjoint_into(cudaStream_t s, double* dst, const double* z_tsv, int qtsv, int gate) {
    cplx<double>* g = fft->d_grid.as<cplx<double>>();
    k_cpp_gather<<<dim3(ntiles, B), 256, 0, s>>>(g, fft->gstride, nx, ny, d_tptr.as<int>(), d_tpts.as<int>(),
                                                d_mx.as<int>(), d_my.as<int>(), d_yn.as<int>(), d_e1.as<double>(),
                                                d_e2x.as<double>(), d_e2y.as<double>(), y2(), M, scale_adj, c.st,
                                                gate);
    MF_LAUNCH_CK();
    k_nufft_cols<double><<<dim3(cdiv(ny + 1, fft->cpc), B), 256, fft->smem_cols, s>>>(
        g, fft->gstride, nx, ny, fft->fcol.dev, +1, fft->cpc, 0, 1, c.st, gate, DynUnits{nullptr, 0});
    MF_LAUNCH_CK();
    TsvFuse tf{z_tsv, c.prm, c.tsvNX, c.tsvNY};
    k_nufft_rows_inv<double><<<dim3(cdiv(nx, fft->rpc), B), 256, fft->smem_rows, s>>>(
        g, fft->gstride, dst, c.xstride, d_e4.as<double>(), nx, ny, 1.0, fft->fh.dev, fft->tw2h.as<cplx<double>>(),
        tf, c.part, qtsv, c.st, gate, fft->rpc, DynUnits{nullptr, 0});
    MF_LAUNCH_CK();
  }

  void adjoint(cudaStream_t s, const double* z_tsv, int qtsv) override {
    adjoint_into(s, c.dfdx, z_tsv, qtsv, kGateGrad);
  }

  int chi_slots() const override { return cdiv(M, 8); }
  int tsv_slots() const override { return std::max(fft->tsv_slots(), cdiv(nx, fft->rpc)); }
  double fscale() const override { return 0.5; }
  int launches_forward() const override { return 3; }
  int launches_adjoint() const override { return 3; }
};

}  // namespace cppnufft
}  // namespace mf
