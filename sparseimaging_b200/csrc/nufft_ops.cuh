// Gaussian-gridding NUFFT kernels (forward A x and adjoint A^H r) of the
// reference's NUFFT variant (c/mfista_nufft_lib.c:27-304), restructured for
// the GPU:
//   * preNUFFT's per-point factors are computed once per solve on the device
//     and folded into two 24-tap weight vectors per point (wx, wy*E1);
//   * the centred zero padding and the E4 grid correction are fused into the
//     first (row) pass of the r2c FFT and the last (row) pass of the c2r FFT,
//     and both column passes skip the all-zero half of the padded image;
//   * interpolation (NUFFT2d2) is one warp per uv point, 576 taps over the 32
//     lanes, complex grid cells read as one 8/16-byte vector;
//   * spreading (NUFFT2d1) is output-stationary: every CTA owns a tile of
//     the half-plane grid and gathers the taps of the points binned to it, so
//     there are no atomics and the result is deterministic.
#pragma once
#include <cooperative_groups.h>
#include "common.cuh"
#include "fft_smem.cuh"

namespace mf {

namespace cg = cooperative_groups;

// Geometry of a batch of NUFFT problems (points concatenated).
template <typename T> struct NufftGeom {
  const int* mx;          // [Mtot]
  const int* my;          // [Mtot]
  const T* wx;            // [Mtot*24]  E2x * E3x
  const T* wy;            // [Mtot*24]  E1 * E2y * E3y
  const double* vis_r;    // [Mtot]
  const double* vis_i;    // [Mtot]
  const double* weight;   // [Mtot]  1 / vis_std
  const int* pt_lo;       // [B] first point of problem b
  const int* pt_hi;       // [B] one past its last point
  const int* tile_ptr;    // CSR over (geometry, tile): [ngeo*ntiles + 1]
  const int* tile_pts;    // point indices (global) binned to each tile
  const int* tile_order;  // shared geometry: tiles by falling point count (launch order), or null
  int tile_bstride;       // ntiles, or 0 when all problems share one geometry
  long y2_bstride;        // per-problem offset of the residual, 0 if not shared
  const double* e4;       // [Nx*Ny] grid correction (shared by all problems)
  const int* act_lists;   // this step's gate lists (device loop), or null (active_chunk)
};

// m2mr (c/mfista_nufft_lib.c:42-48)
__host__ __device__ __forceinline__ int centre_index(int id, int n) { return id < n / 2 ? id + (3 * n) / 2 : id - n / 2; }

// inverse of centre_index over [0, 2n): image index or -1 for padding
__host__ __device__ __forceinline__ int uncentre_index(int c, int n) {
  if (c < n - n / 2) return c + n / 2;
  if (c >= (3 * n) / 2 && c < (3 * n) / 2 + n / 2) return c - (3 * n) / 2;
  return -1;
}

// idx_fftw (c/mfista_nufft_lib.c:32-40) for the x axis: m in [-n, n) -> row,
// anything else is outside the reference's array (dropped: -1).
__host__ __device__ __forceinline__ int wrap_row(int m, int nx) {
  if (m >= 0 && m < nx) return m;
  if (m >= -nx && m < 0) return m + 2 * nx;
  return -1;
}
// y axis as the reference filters it (idx_fftw(m, 2Ny) < Ny+1, :156/:218)
__host__ __device__ __forceinline__ int half_col(int m, int ny) {
  if (m >= 0 && m < ny) return m;
  if (m == -ny) return ny;
  return -1;
}

// ---------------------------------------------------------------------------
// per-point factors (preNUFFT, c/mfista_nufft_lib.c:50-121)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_nufft_prep_points(const double* __restrict__ u, const double* __restrict__ v,
                                    const int* __restrict__ mx, const int* __restrict__ my, int mtot, int nx,
                                    int ny, T* __restrict__ wx, T* __restrict__ wy) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= mtot) return;
  const double pi = 3.14159265358979323846;
  double mrx = 2.0 * nx, mry = 2.0 * ny;
  double taux = 12.0 / (double)(nx * nx), tauy = 12.0 / (double)(ny * ny);
  double e3x_c = (pi / mrx) * (pi / mrx) / taux;
  double e3y_c = (pi / mry) * (pi / mry) / tauy;
  double xix = (2 * pi * (double)mx[k]) / mrx;
  double xiy = (2 * pi * (double)my[k]) / mry;
  double du = u[k] - xix, dv = v[k] - xiy;
  double e1 = exp(-(du * du) / (4 * taux) + -(dv * dv) / (4 * tauy));
  double ax = pi * du / (mrx * taux), ay = pi * dv / (mry * tauy);
  for (int j = 0; j < kTaps; ++j) {
    double pw = (double)(j - (kMSP - 1));
    int l = j - (kMSP - 1);
    l = l < 0 ? -l : l;
    double e3x = exp(-e3x_c * (double)(l * l));
    double e3y = exp(-e3y_c * (double)(l * l));
    wx[(size_t)k * kTaps + j] = (T)(exp(pw * ax) * e3x);
    wy[(size_t)k * kTaps + j] = (T)(e1 * exp(pw * ay) * e3y);
  }
}

static __global__ void k_nufft_prep_e4(double* __restrict__ e4, int nx, int ny) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny) return;
  int i = t / ny, j = t - i * ny;
  const double pi = 3.14159265358979323846;
  double taux = 12.0 / (double)(nx * nx), tauy = 12.0 / (double)(ny * ny);
  double coeff = pi / sqrt(taux * tauy);
  double ti = (double)(i - nx / 2), tj = (double)(j - nx / 2);  // reference uses Nx/2 for both (:78,:82)
  e4[t] = coeff * exp(taux * ti * ti + tauy * tj * tj);
}

// Work of a CTA of the FFT passes.  Normally CTA (x, y) transforms units
// (rows or columns) [x u, x u + u) of problem y, if y passes the gate.
// Inside the device loop, with few problems active (this step's list for
// the launch's gate holds at most kDynFew), the launch's CTAs are instead
// spread over the active problems only, each taking fewer units (halving
// from `small` up to u until the grid holds the work), so that the few
// transforms left run on many SMs.  A row's or column's transform is the
// same arithmetic whatever the units per CTA, so the results do not change.
constexpr int kDynFew = 4;
struct DynUnits {
  const int* list;  // this step's gate list (count, then problem indices), or null (fixed mapping)
  int small;
};
struct FftWork {
  int b, u0, units;
};
__device__ __forceinline__ bool fft_work(const DynUnits& d, const ProbState* __restrict__ st, int gate, int n,
                                         int units, FftWork& w) {
  if (d.list && d.list[0] <= kDynFew) {
    const int nact = d.list[0];
    const int cap = (int)(gridDim.x * gridDim.y);
    int u = d.small;
    while (u < units && nact * ((n + u - 1) / u) > cap) u = min(2 * u, units);
    const int nseg = (n + u - 1) / u;
    const int idx = (int)(blockIdx.y * gridDim.x + blockIdx.x);
    if (idx >= nact * nseg) return false;
    w.b = d.list[1 + idx / nseg];
    w.u0 = (idx % nseg) * u;
    w.units = u;
    return true;
  }
  w.b = blockIdx.y;
  if (!gate_ok(st[w.b], gate)) return false;
  w.u0 = blockIdx.x * units;
  w.units = units;
  return w.u0 < n;
}

// ---------------------------------------------------------------------------
// forward, pass 1: pad + E4 + real FFT of every image row (rows of the
// 2Nx x 2Ny padded grid that hold image data), written to the half grid.
//   Row length n1 = 2Ny is transformed as a complex FFT of length h = Ny.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_nufft_rows_fwd(const double* __restrict__ xall, long xstride, const double* __restrict__ e4,
                                 cplx<T>* __restrict__ gall, long gstride, int nx, int ny, FftDev<T> fh,
                                 const cplx<T>* __restrict__ tw2h, const ProbState* __restrict__ st, int gate,
                                 int rows_per_cta, const double* __restrict__ suball, DynUnits dyn) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FftWork w;
  if (!fft_work(dyn, st, gate, nx, rows_per_cta, w)) return;
  const int b = w.b;
  const int h = ny;
  const int ld = h + 1;
  cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* Bf = A + (size_t)rows_per_cta * ld;
  const double* x = xall + (size_t)b * xstride;
  // defect correction: transform x - x_anchor (the anchor's model is added
  // back in FP64 at the interpolation)
  const double* sub = suball ? suball + (size_t)b * xstride : nullptr;
  cplx<T>* g = gall + (size_t)b * gstride;
  int i0 = w.u0;
  int nrows = min(w.units, nx - i0);
  const int lh = ((h & (h - 1)) == 0) ? __ffs(h) - 1 : -1;  // power-of-two rows: shifts
  for (int t = threadIdx.x; t < nrows * h; t += blockDim.x) {
    int rr = lh >= 0 ? t >> lh : t / h, m = t - rr * h;
    int i = i0 + rr;
    int j0 = uncentre_index(2 * m, ny), j1 = uncentre_index(2 * m + 1, ny);
    T a = 0, c = 0;
    if (j0 >= 0) {
      size_t f = (size_t)i * ny + j0;
      a = (T)((sub ? x[f] - sub[f] : x[f]) * e4[f]);
    }
    if (j1 >= 0) {
      size_t f = (size_t)i * ny + j1;
      c = (T)((sub ? x[f] - sub[f] : x[f]) * e4[f]);
    }
    A[rr * ld + m] = mk<T>(a, c);
  }
  __syncthreads();
  cplx<T>* Z = smem_fft<T>(A, Bf, fh, ld, nrows, -1);
  // X[k] = 1/2[(Z_k + conj Z_{h-k}) - i W^k (Z_k - conj Z_{h-k})], W = exp(-2 pi i / 2h)
  // a warp per row, lanes along its h + 1 outputs (no division by h + 1)
  for (int rr = (int)(threadIdx.x >> 5); rr < nrows; rr += (int)(blockDim.x >> 5))
    for (int k = (int)(threadIdx.x & 31); k <= h; k += 32) {
    cplx<T> zk = Z[rr * ld + (k == h ? 0 : k)];
    cplx<T> zc = cconj<T>(Z[rr * ld + (k == 0 ? 0 : h - k)]);
    cplx<T> e = cadd<T>(zk, zc);
    cplx<T> o = csub<T>(zk, zc);
    cplx<T> wo = cmul_si<T>(cmul<T>(tw2h[k], o), -1);
    cplx<T> X = mk<T>(T(0.5) * (e.x + wo.x), T(0.5) * (e.y + wo.y));
    int row = centre_index(i0 + rr, nx);
    g[(size_t)row * (ny + 1) + k] = X;
  }
}

// ---------------------------------------------------------------------------
// column passes: complex FFT of length 2Nx down groups of half-grid columns.
//   load_pruned: rows of the padded grid that hold no image data are zero and
//                are not read (forward).
//   store_pruned: only rows that map back to image rows are written (inverse).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_nufft_cols(cplx<T>* __restrict__ gall, long gstride, int nx, int ny, FftDev<T> f2x, int sign,
                             int cols_per_cta, int load_pruned, int store_pruned,
                             const ProbState* __restrict__ st, int gate, DynUnits dyn) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FftWork w;
  if (!fft_work(dyn, st, gate, ny + 1, cols_per_cta, w)) return;
  const int b = w.b;
  const int n0 = 2 * nx, ncol = ny + 1;
  const int ld = n0 + 1;
  cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* Bf = A + (size_t)cols_per_cta * ld;
  cplx<T>* g = gall + (size_t)b * gstride;
  const int cpc = w.units;
  int c0 = w.u0;
  int nc = min(cpc, ncol - c0);
  // columns per CTA a power of two (every shape the tuner offers): shifts
  const int lc = ((cpc & (cpc - 1)) == 0) ? __ffs(cpc) - 1 : -1;
  for (int t = threadIdx.x; t < n0 * cpc; t += blockDim.x) {
    int r = lc >= 0 ? t >> lc : t / cpc, cc = t - r * cpc;
    if (cc >= nc) continue;
    cplx<T> v = mk<T>(0, 0);
    if (!load_pruned || uncentre_index(r, nx) >= 0) v = g[(size_t)r * ncol + c0 + cc];
    A[cc * ld + r] = v;
  }
  __syncthreads();
  cplx<T>* R = smem_fft<T>(A, Bf, f2x, ld, nc, sign);
  for (int t = threadIdx.x; t < n0 * cpc; t += blockDim.x) {
    int r = lc >= 0 ? t >> lc : t / cpc, cc = t - r * cpc;
    if (cc >= nc) continue;
    if (store_pruned && uncentre_index(r, nx) < 0) continue;
    g[(size_t)r * ncol + c0 + cc] = R[cc * ld + r];
  }
}

// ---------------------------------------------------------------------------
// forward, pass 3: interpolation at the uv points (NUFFT2d2 :212-241) fused
// with the weighted residual and chi^2 (calc_yAx_nufft / calc_F_part_nufft,
// :245-285).  In gradient mode the residual weighted once more (dF_dx_nufft
// :296-299) is stored for the adjoint.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_nufft_interp(NufftGeom<T> geo, const cplx<T>* __restrict__ gall, long gstride, int nx, int ny,
                               double inv_mm, const ProbState* __restrict__ st, int gate, Partials part, int qchi,
                               cplx<T>* __restrict__ y2, const double2* __restrict__ ax_base,
                               double2* __restrict__ ax_out) {
  __shared__ double sh[32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const cplx<T>* g = gall + (size_t)b * gstride;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  int p0 = geo.pt_lo[b], p1 = geo.pt_hi[b];
  int k = p0 + blockIdx.x * nwarp + warp;
  double chi[1] = {0.0};
  if (k < p1) {
    int mxk = geo.mx[k], myk = geo.my[k];
    const T* wxk = geo.wx + (size_t)k * kTaps;
    const T* wyk = geo.wy + (size_t)k * kTaps;
    T accr = 0, acci = 0;
#pragma unroll 6
    for (int s = 0; s < (kTaps * kTaps) / 32; ++s) {
      int t = lane + 32 * s;
      int lx = t / kTaps, ly = t - lx * kTaps;
      int m = myk + ly - (kMSP - 1);
      int mxm = mxk + lx - (kMSP - 1);
      int col = half_col(m, ny), row;
      T sgn;
      if (col >= 0) {
        row = wrap_row(mxm, nx);
        sgn = T(-1);  // NU_SIGN
      } else {
        col = half_col(-m, ny);
        row = wrap_row(-mxm, nx);
        sgn = T(1);
      }
      if (col >= 0 && row >= 0) {
        cplx<T> gv = g[(size_t)row * (ny + 1) + col];
        T w = wyk[ly] * wxk[lx];
        accr += gv.x * w;
        acci += sgn * gv.y * w;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      accr += __shfl_xor_sync(0xffffffffu, accr, o);
      acci += __shfl_xor_sync(0xffffffffu, acci, o);
    }
    if (lane == 0) {
      double fr = (double)accr * inv_mm, fi = (double)acci * inv_mm;
      const size_t e = b * geo.y2_bstride + k;
      if (ax_base) {
        fr += ax_base[e].x;
        fi += ax_base[e].y;
      }
      if (ax_out) ax_out[e] = make_double2(fr, fi);
      double w = geo.weight[k];
      double rr = (geo.vis_r[k] - fr) * w;
      double ri = (geo.vis_i[k] - fi) * w;
      chi[0] = rr * rr + ri * ri;
      if (y2) y2[e] = mk<T>((T)(rr * w), (T)(ri * w));
    }
  }
  block_sum<1>(chi, sh);
  if (threadIdx.x == 0 && qchi >= 0) part.at(qchi, b)[blockIdx.x] = chi[0];
}

// ---------------------------------------------------------------------------
// adjoint, pass 1: spreading (NUFFT2d1 :140-171), output-stationary.
// One thread per half-grid cell of a TR x TC tile; points of the tile's bin
// are staged through shared memory in chunks.
// ---------------------------------------------------------------------------
template <typename T> struct SpreadChunk {
  static constexpr int P = sizeof(T) == 8 ? 32 : 64;
};

template <typename T>
__global__ void k_nufft_spread(NufftGeom<T> geo, const cplx<T>* __restrict__ y2, cplx<T>* __restrict__ gall,
                               long gstride, int nx, int ny, int tile_r, int tile_c, int ntiles,
                               const ProbState* __restrict__ st, int gate) {
  constexpr int P = SpreadChunk<T>::P;
  __shared__ int s_mx[P], s_my[P];
  __shared__ T s_vr[P], s_vi[P];
  __shared__ T s_wx[P][kTaps], s_wy[P][kTaps];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  cplx<T>* g = gall + (size_t)b * gstride;
  int tile = blockIdx.x;
  int ntc = (ny + 1 + tile_c - 1) / tile_c;
  int tr = tile / ntc, tc = tile - tr * ntc;
  int ty = threadIdx.x / tile_c, tx = threadIdx.x - ty * tile_c;
  int row = tr * tile_r + ty, col = tc * tile_c + tx;
  bool valid = ty < tile_r && row < 2 * nx && col <= ny;
  int mrow = row < nx ? row : row - 2 * nx;  // x index m with wrap_row(m) == row
  int mcol = col < ny ? col : -ny;          // y index m with half_col(m) == col
  T ar = 0, ai = 0;
  int beg = geo.tile_ptr[(size_t)b * geo.tile_bstride + tile];
  int end = geo.tile_ptr[(size_t)b * geo.tile_bstride + tile + 1];
  const cplx<T>* yb = y2 + b * geo.y2_bstride;
  for (int c0 = beg; c0 < end; c0 += P) {
    int np = min(P, end - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < np; t += blockDim.x) {
      int k = geo.tile_pts[c0 + t];
      s_mx[t] = geo.mx[k];
      s_my[t] = geo.my[k];
      cplx<T> r = yb[k];
      s_vr[t] = r.x;
      s_vi[t] = -r.y;  // NU_SIGN * Fin_i
    }
    for (int t = threadIdx.x; t < np * kTaps; t += blockDim.x) {
      int pp = t / kTaps, j = t - pp * kTaps;
      int k = geo.tile_pts[c0 + pp];
      s_wx[pp][j] = geo.wx[(size_t)k * kTaps + j];
      s_wy[pp][j] = geo.wy[(size_t)k * kTaps + j];
    }
    __syncthreads();
    if (valid) {
      for (int pp = 0; pp < np; ++pp) {
        int mx = s_mx[pp], my = s_my[pp];
        int lxd = mrow - mx + (kMSP - 1), lyd = mcol - my + (kMSP - 1);
        int lxm = -mrow - mx + (kMSP - 1), lym = -mcol - my + (kMSP - 1);
        bool d = (unsigned)lxd < (unsigned)kTaps && (unsigned)lyd < (unsigned)kTaps;
        bool mi = (unsigned)lxm < (unsigned)kTaps && (unsigned)lym < (unsigned)kTaps;
        if (!(d || mi)) continue;
        T vr = s_vr[pp], vi = s_vi[pp];
        // the reference adds the two contributions of one point in ly order
        // (direct first on a tie), which is kept here
        if (d && (!mi || lyd <= lym)) {
          const T hw = s_wy[pp][lyd] * s_wx[pp][lxd] * T(0.5);
          ar += vr * hw;
          ai += vi * hw;
          d = false;
        }
        if (mi) {
          const T hw = s_wy[pp][lym] * s_wx[pp][lxm] * T(0.5);
          ar += vr * hw;
          ai += -vi * hw;
        }
        if (d) {
          const T hw = s_wy[pp][lyd] * s_wx[pp][lxd] * T(0.5);
          ar += vr * hw;
          ai += vi * hw;
        }
      }
    }
  }
  if (valid) g[(size_t)row * (ny + 1) + col] = mk<T>(ar, ai);
}

// ---------------------------------------------------------------------------
// adjoint, last pass: half-complex -> real FFT of the rows that map to image
// rows, unpad, E4/MM (:175-183), and — for the TSV form — the TSV gradient of
// z folded in (dfdx -= lambda_tsv * d_TSV(z), c/mfista_nufft_lib.c:674-681)
// together with TSV(z).
// ---------------------------------------------------------------------------
struct TsvFuse {
  const double* z;     // per-problem z (stride xstride) or null
  const ProbParams* prm;
  int NX, NY;          // TSV view (reference's TSV(NX, NY, x))
};

__device__ __forceinline__ double dtsv_at(const double* __restrict__ x, int f, int NX, int NY) {
  int i = f % NX, j = f / NX;
  double xf = x[f];
  double d = (i < NX - 1) ? 2 * (xf - x[f + 1]) : 0.0;
  if (i >= 1) d += 2 * (xf - x[f - 1]);
  if (j < NY - 1) d += 2 * (xf - x[f + NX]);
  if (j >= 1) d += 2 * (xf - x[f - NX]);
  return d;
}

__device__ __forceinline__ double tsv_terms_at(const double* __restrict__ x, int f, int NX, int NY) {
  int i = f % NX, j = f / NX;
  double xf = x[f], s = 0.0;
  if (i < NX - 1) {
    double d = xf - x[f + 1];
    s += d * d;
  }
  if (j < NY - 1) {
    double d = xf - x[f + NX];
    s += d * d;
  }
  return s;
}

template <typename T>
__global__ void k_nufft_rows_inv(const cplx<T>* __restrict__ gall, long gstride, double* __restrict__ dall,
                                 long xstride, const double* __restrict__ e4, int nx, int ny, double inv_mm,
                                 FftDev<T> fh, const cplx<T>* __restrict__ tw2h, TsvFuse tf, Partials part,
                                 int qtsv, const ProbState* __restrict__ st, int gate, int rows_per_cta,
                                 DynUnits dyn) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sh[32];
  FftWork w;
  if (!fft_work(dyn, st, gate, nx, rows_per_cta, w)) return;
  const int b = w.b;
  const int h = ny, ld = h + 1;
  cplx<T>* A = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* Bf = A + (size_t)rows_per_cta * ld;
  const cplx<T>* g = gall + (size_t)b * gstride;
  double* dfdx = dall + (size_t)b * xstride;
  // (the spread mapping only without TSV partials: their slots are the grid's x)
  int i0 = w.u0;
  int nrows = min(w.units, nx - i0);
  // Z[k] = (X_k + conj X_{h-k}) + i conj(W^k) (X_k - conj X_{h-k}); DC/Nyquist real parts only
  const int lh = ((h & (h - 1)) == 0) ? __ffs(h) - 1 : -1;  // power-of-two rows: shifts
  for (int t = threadIdx.x; t < nrows * h; t += blockDim.x) {
    int rr = lh >= 0 ? t >> lh : t / h, k = t - rr * h;
    const cplx<T>* grow = g + (size_t)centre_index(i0 + rr, nx) * (ny + 1);
    cplx<T> xk = grow[k];
    cplx<T> xc = grow[h - k];
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
  const ProbParams& pp = tf.prm[b];
  bool fuse = tf.z != nullptr && pp.lambda_tsv > 0.0;
  const double* z = fuse ? tf.z + (size_t)b * xstride : nullptr;
  double acc[1] = {0.0};
  for (int t = threadIdx.x; t < nrows * ny; t += blockDim.x) {
    int rr = lh >= 0 ? t >> lh : t / ny, j = t - rr * ny;
    int i = i0 + rr;
    int c = centre_index(j, ny);
    cplx<T> zc = Z[rr * ld + (c >> 1)];
    double val = (double)((c & 1) ? zc.y : zc.x);
    int f = i * ny + j;
    double d = val * e4[f] * inv_mm;
    if (fuse) {
      d = d + dtsv_at(z, f, tf.NX, tf.NY) * (-pp.lambda_tsv);
      acc[0] += tsv_terms_at(z, f, tf.NX, tf.NY);
    }
    dfdx[f] = d;
  }
  if (qtsv >= 0) {
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) part.at(qtsv, b)[blockIdx.x] = acc[0];
  }
}

}  // namespace mf

// ===========================================================================
// Shared-geometry batch (every problem of the batch uses the same uv points,
// e.g. a lambda grid).  The tap geometry of a point is computed once and
// applied to a chunk of problems; grids stay problem-major.
// ===========================================================================
namespace mf {

template <typename T> struct SharedChunk;
template <> struct SharedChunk<float> {
  static constexpr int kInterp = 16;  // problems per interpolation CTA
  static constexpr int kSpread = 16;  // problems per spreading CTA
  static constexpr int kInterpMinBlocks = 3;
  static constexpr int kInterpPts = 1;  // default points per warp (what the autotuner picks on the lambda grid)
  static constexpr int kSpreadMinBlocks = 3;
};
template <> struct SharedChunk<double> {
  static constexpr int kInterp = 8;
  static constexpr int kSpread = 8;
  static constexpr int kInterpMinBlocks = 2;
  static constexpr int kInterpPts = 8;
  static constexpr int kSpreadMinBlocks = 3;
};

// interpolation: one warp per point, lanes over the 576 taps (18 each) with
// cell and weight held in registers, looping over the CTA's problem chunk;
// each warp takes `ppw` consecutive points (a launch-shape choice: the
// per-point arithmetic does not depend on it, the grouping of the chi^2
// partial sums does).  kActiveChunks: chunk y holds the y-th PB of the
// batch's active problems (active_chunk) instead of problems [y PB, y PB + PB).

template <typename T, bool kActiveChunks = false>
__global__ void __launch_bounds__(256, SharedChunk<T>::kInterpMinBlocks) k_nufft_interp_shared(NufftGeom<T> geo, const cplx<T>* __restrict__ gall,
                                                             long gstride, int nx, int ny, double inv_mm,
                                                             const ProbState* __restrict__ st, int gate,
                                                             Partials part, int qchi, cplx<T>* __restrict__ y2,
                                                             int B, const double2* __restrict__ ax_base,
                                                             double2* __restrict__ ax_out, int ppw) {
  constexpr int PB = SharedChunk<T>::kInterp;
  constexpr int NT = (kTaps * kTaps) / 32;
  __shared__ double s_chi[8][PB];
  __shared__ int s_act[PB];
  __shared__ int s_prob[PB];  // problem of chunk slot i
  if (kActiveChunks) {
    __shared__ int s_cnt[8];
    const int n = active_chunk<PB>(st, gate, B, blockIdx.y, s_prob, s_cnt, geo.act_lists);
    if (threadIdx.x < PB) s_act[threadIdx.x] = threadIdx.x < n ? 1 : 0;
  } else if (threadIdx.x < PB) {
    const int b = blockIdx.y * PB + threadIdx.x;
    s_prob[threadIdx.x] = b;
    s_act[threadIdx.x] = (b < B && gate_ok(st[b], gate)) ? 1 : 0;
  }
  __syncthreads();
  int any = 0;
#pragma unroll
  for (int i = 0; i < PB; ++i) any |= s_act[i];
  if (!any) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mtot = geo.pt_hi[0];
  if (lane < PB) s_chi[warp][lane] = 0.0;
  __syncwarp();
  for (int q = 0; q < ppw; ++q) {
    const int k = (blockIdx.x * 8 + warp) * ppw + q;
    if (k >= mtot) break;
    int cell[NT];
    T wgt[NT];
    const int mxk = geo.mx[k], myk = geo.my[k];
    const T* wxk = geo.wx + (size_t)k * kTaps;
    const T* wyk = geo.wy + (size_t)k * kTaps;
#pragma unroll
    for (int s = 0; s < NT; ++s) {
      int t = lane + 32 * s;
      int lx = t / kTaps, ly = t - lx * kTaps;
      int m = myk + ly - (kMSP - 1);
      int mxm = mxk + lx - (kMSP - 1);
      int col = half_col(m, ny), row, mirror = 0;
      if (col >= 0) {
        row = wrap_row(mxm, nx);
      } else {
        col = half_col(-m, ny);
        row = wrap_row(-mxm, nx);
        mirror = 1;
      }
      if (col >= 0 && row >= 0) {
        cell[s] = (row * (ny + 1) + col) | (mirror << 30);
        wgt[s] = wyk[ly] * wxk[lx];
      } else {
        cell[s] = -1;
        wgt[s] = 0;
      }
    }
    const double w = geo.weight[k];
    const double vr = geo.vis_r[k], vi = geo.vis_i[k];
#pragma unroll 1
    for (int i = 0; i < PB; ++i) {
      if (!s_act[i]) continue;
      const int b = s_prob[i];
      const cplx<T>* g = gall + (size_t)b * gstride;
      T accr = 0, acci = 0;
#pragma unroll
      for (int s = 0; s < NT; ++s) {
        int cc = cell[s];
        if (cc >= 0) {
          cplx<T> gv = g[cc & 0x3fffffff];
          accr += gv.x * wgt[s];
          // NU_SIGN on the imaginary part of direct taps, + on mirrored ones
          acci += ((cc >> 30) ? gv.y : -gv.y) * wgt[s];
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        accr += __shfl_xor_sync(0xffffffffu, accr, o);
        acci += __shfl_xor_sync(0xffffffffu, acci, o);
      }
      if (lane == 0) {
        double fr = (double)accr * inv_mm, fi = (double)acci * inv_mm;
        const size_t e = (size_t)b * geo.y2_bstride + k;
        if (ax_base) {
          fr += ax_base[e].x;
          fi += ax_base[e].y;
        }
        if (ax_out) ax_out[e] = make_double2(fr, fi);
        double rr = (vr - fr) * w;
        double ri = (vi - fi) * w;
        s_chi[warp][i] += rr * rr + ri * ri;
        if (y2) y2[e] = mk<T>((T)(rr * w), (T)(ri * w));
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < PB && s_act[threadIdx.x] && qchi >= 0) {
    double c = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) c += s_chi[w][threadIdx.x];
    part.at(qchi, s_prob[threadIdx.x])[blockIdx.x] = c;
  }
}

// Grouped interpolation: the same warp-per-point tap layout as
// k_nufft_interp_shared, but the CTA's active problems (compacted into a
// list) are taken G at a time with the G accumulator pairs held together,
// so the tap loop issues G independent loads per tap and each tap's address
// and weight serve G problems; G is 8, 4, 2 or 1 as the number of remaining
// active problems allows (FP32 only: 2G double sums do not fit the register
// budget, and FP64 plans use k_nufft_interp_shared).  Points whose 576 taps are all
// direct and inside the grid (the usual case; warp-uniform) take a loop
// without per-tap flag tests that adds the same products in the same order
// as the general loop.  The 2G sums are reduced over the warp by a
// transposing butterfly: at each of the first log2(2G) levels a lane keeps
// half of its values and receives the partner's copy of that half, so
// 2G - 1 shuffles (plus 5 - log2(2G) plain levels) leave lane L with value
// L >> (5 - log2(2G)); real parts sit in lanes 0-15, imaginary parts in
// lanes 16-31, and one lane per problem finishes the G problems in
// parallel.  Each level adds a lane's partial to that of lane L ^ off, the
// same pairs in the same order as the plain butterfly (offsets 16, 8, 4, 2,
// 1) of k_nufft_interp_shared, so a point's value does not depend on G and
// equals that kernel's to the bit.  Partial chi^2 sums are kept per (warp,
// problem) in point order, as in k_nufft_interp_shared.
template <typename T> struct GroupChunk;
template <> struct GroupChunk<float> {
  static constexpr int kGmax = 8;  // 16 float sums per lane
  static constexpr int kMinBlocks = 2;
};

// transposing warp reduction of 2^V values (V <= 5): afterwards every lane
// holds the warp-wide sum of value (lane >> (5 - V)) in v[0]
template <int V, typename T> __device__ __forceinline__ void transpose_reduce(T (&v)[1 << V], int lane) {
#pragma unroll
  for (int lvl = 0; lvl < V; ++lvl) {
    const int half = (1 << V) >> (lvl + 1);  // values kept after this level
    const int off = 16 >> lvl;
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const T send = upper ? v[j] : v[j + half];
      const T keep = upper ? v[j + half] : v[j];
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
#pragma unroll
  for (int off = 16 >> V; off > 0; off >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], off);
}

// per-point data of one interpolation pass
template <typename T> struct InterpPoint {
  static constexpr int NT = (kTaps * kTaps) / 32;
  int cell[NT];  // grid index | mirrored << 30, or -1
  T wgt[NT];
  bool plain;    // every tap of the warp direct and inside the grid
  int k;
  double w, vr, vi;
};

// G problems of the CTA's active list starting at list[pos]
template <typename T, int G>
__device__ __forceinline__ void interp_group(const InterpPoint<T>& P, const cplx<T>* __restrict__ gall, long gstride,
                                             const int* list, int pos, int lane, double inv_mm,
                                             const NufftGeom<T>& geo, const double2* __restrict__ ax_base,
                                             double2* __restrict__ ax_out, cplx<T>* __restrict__ y2,
                                             double* s_chi_w) {
  constexpr int V = (G == 8) ? 4 : (G == 4) ? 3 : (G == 2) ? 2 : 1;  // 2G = 2^V sums
  constexpr int NT = InterpPoint<T>::NT;
  const cplx<T>* g[G];
#pragma unroll
  for (int i = 0; i < G; ++i) g[i] = gall + (size_t)list[pos + i] * gstride;
  T acc[2 * G];
#pragma unroll
  for (int i = 0; i < 2 * G; ++i) acc[i] = 0;
  if (P.plain) {
#pragma unroll
    for (int s = 0; s < NT; ++s) {
      const int cc = P.cell[s];
#pragma unroll
      for (int i = 0; i < G; ++i) {
        const cplx<T> gv = g[i][cc];
        acc[i] += gv.x * P.wgt[s];
        acc[G + i] += (-gv.y) * P.wgt[s];  // NU_SIGN: direct taps only
      }
    }
  } else {
#pragma unroll
    for (int s = 0; s < NT; ++s) {
      const int cc = P.cell[s];
      if (cc >= 0) {
        const bool mir = (cc >> 30) != 0;
#pragma unroll
        for (int i = 0; i < G; ++i) {
          const cplx<T> gv = g[i][cc & 0x3fffffff];
          acc[i] += gv.x * P.wgt[s];
          // NU_SIGN on the imaginary part of direct taps, + on mirrored ones
          acc[G + i] += (mir ? gv.y : -gv.y) * P.wgt[s];
        }
      }
    }
  }
  transpose_reduce<V>(acc, lane);
  const T im = __shfl_xor_sync(0xffffffffu, acc[0], 16);
  const int fin = lane >> (5 - V);
  if (lane < 16 && (lane & ((1 << (5 - V)) - 1)) == 0) {
    const int slot = pos + fin;
    const int b = list[slot];
    double fr = (double)acc[0] * inv_mm, fi = (double)im * inv_mm;
    const size_t e = (size_t)b * geo.y2_bstride + P.k;
    if (ax_base) {
      fr += ax_base[e].x;
      fi += ax_base[e].y;
    }
    if (ax_out) ax_out[e] = make_double2(fr, fi);
    const double rr = (P.vr - fr) * P.w;
    const double ri = (P.vi - fi) * P.w;
    s_chi_w[slot] += rr * rr + ri * ri;
    if (y2) y2[e] = mk<T>((T)(rr * P.w), (T)(ri * P.w));
  }
}

template <typename T>
__global__ void __launch_bounds__(256, GroupChunk<T>::kMinBlocks) k_nufft_interp_group(
    NufftGeom<T> geo, const cplx<T>* __restrict__ gall, long gstride, int nx, int ny, double inv_mm,
    const ProbState* __restrict__ st, int gate, Partials part, int qchi, cplx<T>* __restrict__ y2, int B,
    const double2* __restrict__ ax_base, double2* __restrict__ ax_out, int ppw) {
  constexpr int PB = SharedChunk<T>::kInterp;
  constexpr int GM = GroupChunk<T>::kGmax;
  constexpr int NT = InterpPoint<T>::NT;
  __shared__ double s_chi[8][PB];  // per warp, per list slot
  __shared__ int s_list[PB];
  __shared__ int s_cnt[8];
  const int nact = active_chunk<PB>(st, gate, B, blockIdx.y, s_list, s_cnt, geo.act_lists);
  if (nact == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mtot = geo.pt_hi[0];
  if (lane < PB) s_chi[warp][lane] = 0.0;
  __syncwarp();
  for (int q = 0; q < ppw; ++q) {
    InterpPoint<T> P;
    P.k = (blockIdx.x * 8 + warp) * ppw + q;
    if (P.k >= mtot) break;
    const int k = P.k;
    bool plain = true;
    const int mxk = geo.mx[k], myk = geo.my[k];
    const T* wxk = geo.wx + (size_t)k * kTaps;
    const T* wyk = geo.wy + (size_t)k * kTaps;
#pragma unroll
    for (int s = 0; s < NT; ++s) {
      const int t = lane + 32 * s;
      const int lx = t / kTaps, ly = t - lx * kTaps;
      const int m = myk + ly - (kMSP - 1);
      const int mxm = mxk + lx - (kMSP - 1);
      int col = half_col(m, ny), row, mirror = 0;
      if (col >= 0) {
        row = wrap_row(mxm, nx);
      } else {
        col = half_col(-m, ny);
        row = wrap_row(-mxm, nx);
        mirror = 1;
      }
      if (col >= 0 && row >= 0) {
        P.cell[s] = (row * (ny + 1) + col) | (mirror << 30);
        P.wgt[s] = wyk[ly] * wxk[lx];
        plain = plain && !mirror;
      } else {
        P.cell[s] = -1;
        P.wgt[s] = 0;
        plain = false;
      }
    }
    P.plain = __all_sync(0xffffffffu, plain);
    P.w = geo.weight[k];
    P.vr = geo.vis_r[k];
    P.vi = geo.vis_i[k];
    int pos = 0;
    while (pos < nact) {
      const int rem = nact - pos;
      if (GM >= 8 && rem >= 8) {
        interp_group<T, (GM >= 8 ? 8 : 1)>(P, gall, gstride, s_list, pos, lane, inv_mm, geo, ax_base, ax_out,
                                           y2, s_chi[warp]);
        pos += 8;
      } else if (GM >= 4 && rem >= 4) {
        interp_group<T, (GM >= 4 ? 4 : 1)>(P, gall, gstride, s_list, pos, lane, inv_mm, geo, ax_base, ax_out, y2, s_chi[warp]);
        pos += 4;
      } else if (rem >= 2) {
        interp_group<T, 2>(P, gall, gstride, s_list, pos, lane, inv_mm, geo, ax_base, ax_out, y2, s_chi[warp]);
        pos += 2;
      } else {
        interp_group<T, 1>(P, gall, gstride, s_list, pos, lane, inv_mm, geo, ax_base, ax_out, y2, s_chi[warp]);
        pos += 1;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < nact && qchi >= 0) {
    double c = 0.0;
#pragma unroll
    for (int wp = 0; wp < 8; ++wp) c += s_chi[wp][threadIdx.x];
    part.at(qchi, s_list[threadIdx.x])[blockIdx.x] = c;
  }
}

// The same grouped interpolation with the taps formed on the fly instead of
// held in registers: a lane walks its 18 taps t = lane + 32 s as (lx, ly)
// pairs, takes the weight wy[ly] wx[lx] from the warp's copy of the point's
// 48 tap factors in shared memory, and the cell from (mx, my) (a direct,
// inside point, the usual case, needs no per-tap tests: its rows only wrap
// at kx = 0).  Far fewer registers per thread (more warps per SM to hide
// the gathers) for a little more arithmetic per tap; the products and their
// order are those of k_nufft_interp_group, so results are bit-identical.
template <typename T> struct TapPoint {
  int k, mx0, my0;  // point, mx - 11, my - 11
  bool plain;       // every tap direct and inside the grid
  double w, vr, vi;
};

template <typename T, int G>
__device__ __forceinline__ void interp_group_fly(const TapPoint<T>& P, const T* __restrict__ swx,
                                                 const T* __restrict__ swy, const cplx<T>* __restrict__ gall,
                                                 long gstride, const int* list, int pos, int lane, int nx, int ny,
                                                 double inv_mm, const NufftGeom<T>& geo,
                                                 const double2* __restrict__ ax_base, double2* __restrict__ ax_out,
                                                 cplx<T>* __restrict__ y2, double* s_chi_w) {
  constexpr int V = (G == 8) ? 4 : (G == 4) ? 3 : (G == 2) ? 2 : 1;
  constexpr int NT = (kTaps * kTaps) / 32;
  const cplx<T>* g[G];
#pragma unroll
  for (int i = 0; i < G; ++i) g[i] = gall + (size_t)list[pos + i] * gstride;
  T acc[2 * G];
#pragma unroll
  for (int i = 0; i < 2 * G; ++i) acc[i] = 0;
  int lx = lane / kTaps, ly = lane - (lane / kTaps) * kTaps;
  if (P.plain) {
#pragma unroll 2
    for (int s = 0; s < NT; ++s) {
      const int kx = P.mx0 + lx;
      const int cc = (kx + (kx < 0 ? 2 * nx : 0)) * (ny + 1) + P.my0 + ly;
      const T wg = swy[ly] * swx[lx];
#pragma unroll
      for (int i = 0; i < G; ++i) {
        const cplx<T> gv = g[i][cc];
        acc[i] += gv.x * wg;
        acc[G + i] += (-gv.y) * wg;  // NU_SIGN: direct taps only
      }
      ly += 32 - kTaps;  // t += 32 = one row of 24 taps and 8 more
      lx += 1;
      if (ly >= kTaps) {
        ly -= kTaps;
        lx += 1;
      }
    }
  } else {
#pragma unroll 1
    for (int s = 0; s < NT; ++s) {
      const int m = P.my0 + ly, mxm = P.mx0 + lx;
      int col = half_col(m, ny), row;
      bool mir = false;
      if (col >= 0) {
        row = wrap_row(mxm, nx);
      } else {
        col = half_col(-m, ny);
        row = wrap_row(-mxm, nx);
        mir = true;
      }
      if (col >= 0 && row >= 0) {
        const int cc = row * (ny + 1) + col;
        const T wg = swy[ly] * swx[lx];
#pragma unroll
        for (int i = 0; i < G; ++i) {
          const cplx<T> gv = g[i][cc];
          acc[i] += gv.x * wg;
          // NU_SIGN on the imaginary part of direct taps, + on mirrored ones
          acc[G + i] += (mir ? gv.y : -gv.y) * wg;
        }
      }
      ly += 32 - kTaps;
      lx += 1;
      if (ly >= kTaps) {
        ly -= kTaps;
        lx += 1;
      }
    }
  }
  transpose_reduce<V>(acc, lane);
  const T im = __shfl_xor_sync(0xffffffffu, acc[0], 16);
  const int fin = lane >> (5 - V);
  if (lane < 16 && (lane & ((1 << (5 - V)) - 1)) == 0) {
    const int slot = pos + fin;
    const int b = list[slot];
    double fr = (double)acc[0] * inv_mm, fi = (double)im * inv_mm;
    const size_t e = (size_t)b * geo.y2_bstride + P.k;
    if (ax_base) {
      fr += ax_base[e].x;
      fi += ax_base[e].y;
    }
    if (ax_out) ax_out[e] = make_double2(fr, fi);
    const double rr = (P.vr - fr) * P.w;
    const double ri = (P.vi - fi) * P.w;
    s_chi_w[slot] += rr * rr + ri * ri;
    if (y2) y2[e] = mk<T>((T)(rr * P.w), (T)(ri * P.w));
  }
}

template <typename T>
__global__ void __launch_bounds__(256, 3) k_nufft_interp_group_fly(
    NufftGeom<T> geo, const cplx<T>* __restrict__ gall, long gstride, int nx, int ny, double inv_mm,
    const ProbState* __restrict__ st, int gate, Partials part, int qchi, cplx<T>* __restrict__ y2, int B,
    const double2* __restrict__ ax_base, double2* __restrict__ ax_out, int ppw) {
  constexpr int PB = SharedChunk<T>::kInterp;
  constexpr int GM = GroupChunk<T>::kGmax;
  __shared__ double s_chi[8][PB];
  __shared__ int s_list[PB];
  __shared__ int s_cnt[8];
  __shared__ T s_wt[8][2][kTaps];  // per warp: the point's wx, wy
  const int nact = active_chunk<PB>(st, gate, B, blockIdx.y, s_list, s_cnt, geo.act_lists);
  if (nact == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mtot = geo.pt_hi[0];
  if (lane < PB) s_chi[warp][lane] = 0.0;
  __syncwarp();
  for (int q = 0; q < ppw; ++q) {
    TapPoint<T> P;
    P.k = (blockIdx.x * 8 + warp) * ppw + q;
    if (P.k >= mtot) break;
    const int k = P.k;
    const int mxk = geo.mx[k], myk = geo.my[k];
    if (lane < kTaps) {
      s_wt[warp][0][lane] = geo.wx[(size_t)k * kTaps + lane];
      s_wt[warp][1][lane] = geo.wy[(size_t)k * kTaps + lane];
    }
    P.mx0 = mxk - (kMSP - 1);
    P.my0 = myk - (kMSP - 1);
    // direct (0 <= ky < Ny) and inside (-Nx <= kx < Nx) for every tap
    P.plain = P.my0 >= 0 && myk + kMSP < ny && P.mx0 >= -nx && mxk + kMSP < nx;
    P.w = geo.weight[k];
    P.vr = geo.vis_r[k];
    P.vi = geo.vis_i[k];
    __syncwarp();
    const T* swx = s_wt[warp][0];
    const T* swy = s_wt[warp][1];
    int pos = 0;
    while (pos < nact) {
      const int rem = nact - pos;
      if (GM >= 8 && rem >= 8) {
        interp_group_fly<T, (GM >= 8 ? 8 : 1)>(P, swx, swy, gall, gstride, s_list, pos, lane, nx, ny, inv_mm, geo,
                                               ax_base, ax_out, y2, s_chi[warp]);
        pos += 8;
      } else if (GM >= 4 && rem >= 4) {
        interp_group_fly<T, (GM >= 4 ? 4 : 1)>(P, swx, swy, gall, gstride, s_list, pos, lane, nx, ny, inv_mm, geo,
                                               ax_base, ax_out, y2, s_chi[warp]);
        pos += 4;
      } else if (rem >= 2) {
        interp_group_fly<T, 2>(P, swx, swy, gall, gstride, s_list, pos, lane, nx, ny, inv_mm, geo, ax_base, ax_out,
                               y2, s_chi[warp]);
        pos += 2;
      } else {
        interp_group_fly<T, 1>(P, swx, swy, gall, gstride, s_list, pos, lane, nx, ny, inv_mm, geo, ax_base, ax_out,
                               y2, s_chi[warp]);
        pos += 1;
      }
    }
    __syncwarp();  // the next point's factors overwrite s_wt[warp]
  }
  __syncthreads();
  if (threadIdx.x < nact && qchi >= 0) {
    double c = 0.0;
#pragma unroll
    for (int wp = 0; wp < 8; ++wp) c += s_chi[wp][threadIdx.x];
    part.at(qchi, s_list[threadIdx.x])[blockIdx.x] = c;
  }
}

// asynchronous global -> shared copies (4, 8 or 16 bytes)
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src, int bytes) {
  const unsigned int d = (unsigned int)__cvta_generic_to_shared(smem_dst);
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem_src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Interpolation on the tensor cores (FP32 form, shared geometry)
//
// Every problem's grid is one matrix G (cells x problems), and interpolation
// is y = S G with S the points' tap weights.  The points are binned by their
// first tap (mx - 11, my - 11) into 8 x 8 tiles of the *virtual* grid (rows
// and columns before the wrap and the Hermitian fold), so a tile's points
// read a 32 x 32 window of virtual cells (31 used).  A CTA takes up to 128
// points of one tile and a chunk of 8 problems: it stages the window once in
// shared memory, every cell already resolved to its stored cell (direct, or
// mirrored with the conjugate) and to the sign the reference gives the
// imaginary part there (NU_SIGN on direct taps), so all points then run the
// same tap arithmetic with no per-tap tests.  The weights are separable,
// S[p, (r, c)] = wx_p[r] wy_p[c], so for each window row r a warp forms
// T_r = Wy G_r (16 points x 32 columns times 32 columns x 16 problem
// columns) with mma.sync m16n8k8 TF32 and adds wx_p[r] T_r to its result.
// Both operands are split into two TF32 parts (x = hi + lo) and the product
// taken as lo*hi + hi*lo + hi*hi with FP32 accumulation (about 2^-21
// relative per product, the accuracy of FP32 sums over the 576 taps).  The
// epilogue is the one of k_nufft_interp_group: FP64 residual, chi^2, the
// models of the corrected form.
// ---------------------------------------------------------------------------
constexpr int kItcTile = 8;    // home tile (first-tap positions per axis)
constexpr int kItcWin = 32;    // window cells per axis
constexpr int kItcProb = 8;    // problems per CTA (16 real columns)
constexpr int kItcPts = 128;   // points per CTA: 8 warps x 16
struct ItcTile {
  int row0, col0;    // window origin in virtual cells
  int start, count;  // this CTA's points: perm[start, start + count)
};
// perm entries: point index (24 bits) | first-tap row - row0 (3 bits) << 24
// | first-tap column - col0 (3 bits) << 27
constexpr int kItcMaxPoints = 1 << 24;
constexpr size_t kItcSmem = sizeof(float) * (size_t)kItcWin * kItcWin * 2 * kItcProb;  // the window

// x = hi + lo: hi is x rounded to the TF32 grid (half-ulp up in magnitude,
// by integer add and mask), lo = x - hi exactly; lo goes to the tensor core
// as it is, which reads its top 10 mantissa bits (2^-21 of x lost)
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
  lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32_1688(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// window cell (r, c) holds its 16 columns (problem s: 2s real, 2s + 1
// imaginary) at (r * 32 + c) * 16 + (n ^ itc_swz(c)): the xor spreads the
// B-fragment loads of a warp (four consecutive c, eight n) over all banks
__device__ __forceinline__ int itc_swz(int c) { return ((c >> 1) & 1) << 3; }

static __global__ void __launch_bounds__(256, 3) k_nufft_interp_tc(
    NufftGeom<float> geo, const ItcTile* __restrict__ tiles, int ntc, const int* __restrict__ perm,
    const cplx<float>* __restrict__ gall, long gstride, int nx, int ny, double inv_mm,
    const ProbState* __restrict__ st, int gate, Partials part, int qchi, int nslots, cplx<float>* __restrict__ y2,
    int B, const double2* __restrict__ ax_base, double2* __restrict__ ax_out) {
  extern __shared__ __align__(16) float itc_smem[];
  float* s_g = itc_smem;  // [32 * 32 cells][16]
  __shared__ int s_list[kItcProb];
  __shared__ int s_cnt[8];
  __shared__ double s_chi[8][kItcProb];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  // the CTA's points first (independent of the problem chunk): warps over
  // (block of 16 points, row group); a CTA of nb blocks splits each block's
  // window rows into ng = 8 / nb contiguous groups, so sparse tiles still
  // keep all eight warps busy; the groups' sums are added in group order
  const ItcTile tl = tiles[blockIdx.x];
  const int nb = (tl.count + 15) >> 4;
  const int ng = 8 / nb;
  const int blk = warp % nb, grp = warp / nb;
  const bool on = grp < ng;
  const int p0 = tl.start + blk * 16;
  const int np = on ? min(16, tl.start + tl.count - p0) : 0;
  int kq = 0, drq = 0, dcq = 0;
  if (lane < np) {
    const int pk = perm[p0 + lane];  // point | row offset << 24 | column offset << 27
    kq = pk & 0xffffff;
    drq = (pk >> 24) & 7;
    dcq = (pk >> 27) & 7;
  }
  const int nact = active_chunk<kItcProb>(st, gate, B, blockIdx.y, s_list, s_cnt, geo.act_lists);
  if (nact == 0) return;
  // chi^2 slots beyond the CTAs (the slot count other kernels of the
  // operator fill): zero partials
  if ((int)threadIdx.x < nact && qchi >= 0)
    for (int sl = blockIdx.x + ntc; sl < nslots; sl += ntc) part.at(qchi, s_list[threadIdx.x])[sl] = 0.0;
  // lane (g, t) works on points g and g + 8 of the block: its A fragments
  // are wy of those points at columns 8 kk + t (+ 4), loaded before the
  // window's cells so that both sets of loads are in flight together
  const int ka = __shfl_sync(0xffffffffu, kq, g), kb = __shfl_sync(0xffffffffu, kq, g + 8);
  const int dra = __shfl_sync(0xffffffffu, drq, g), drb = __shfl_sync(0xffffffffu, drq, g + 8);
  const int dca = __shfl_sync(0xffffffffu, dcq, g), dcb = __shfl_sync(0xffffffffu, dcq, g + 8);
  const bool va = g < np, vb = g + 8 < np;
  float fa[4][4];
#pragma unroll
  for (int kk = 0; kk < 4; ++kk)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool second = q & 1;
      const int jy = 8 * kk + t + 4 * (q >> 1) - (second ? dcb : dca);
      fa[kk][q] = ((second ? vb : va) && jy >= 0 && jy < kTaps)
                      ? geo.wy[(size_t)(second ? kb : ka) * kTaps + jy] : 0.f;
    }
  // the window: virtual cell -> stored cell, sign of the imaginary part
  for (int v = threadIdx.x; v < kItcWin * kItcWin; v += blockDim.x) {
    const int vr = tl.row0 + (v >> 5), vc = tl.col0 + (v & 31);
    int cell = -1;
    float sgn = -1.f;  // NU_SIGN on direct taps
    int col = half_col(vc, ny);
    if (col >= 0) {
      const int row = wrap_row(vr, nx);
      if (row >= 0) cell = row * (ny + 1) + col;
    } else {
      col = half_col(-vc, ny);
      const int row = wrap_row(-vr, nx);
      if (col >= 0 && row >= 0) {
        cell = row * (ny + 1) + col;
        sgn = 1.f;
      }
    }
    float* dst = s_g + (size_t)v * (2 * kItcProb);
    const int sw = itc_swz(v & 31);
    // the four 16-byte stores of a cell in an order rotated by the cell, so
    // that the 32 lanes of a store instruction cover all banks
#pragma unroll
    for (int q4 = 0; q4 < 4; ++q4) {
      const int s = 2 * ((q4 + (v >> 1)) & 3);
      float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
      if (cell >= 0) {
        if (s < nact) {
          const cplx<float> a = gall[(size_t)s_list[s] * gstride + cell];
          q.x = a.x;
          q.y = sgn * a.y;
        }
        if (s + 1 < nact) {
          const cplx<float> a = gall[(size_t)s_list[s + 1] * gstride + cell];
          q.z = a.x;
          q.w = sgn * a.y;
        }
      }
      *reinterpret_cast<float4*>(dst + ((2 * s) ^ sw)) = q;
    }
  }
  if (lane < kItcProb) s_chi[warp][lane] = 0.0;
  __syncthreads();
  const int nj = nact > 4 ? 2 : 1;  // n-tiles of 8 columns (4 problems) in use
  float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  if (on) {
    const int rlo = __reduce_min_sync(0xffffffffu, lane < np ? drq : kItcWin);
    const int rhi = __reduce_max_sync(0xffffffffu, lane < np ? drq + kTaps - 1 : -1);
    uint32_t ah[4][4], al[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
#pragma unroll
      for (int q = 0; q < 4; ++q) split_tf32(fa[kk][q], ah[kk][q], al[kk][q]);
    const int nr = rhi - rlo + 1, per = (nr + ng - 1) / ng;
    const int r0 = rlo + grp * per, r1 = min(rhi + 1, r0 + per);
    // row weights of points g and g + 8 (the next row's loaded a row ahead)
    auto wxa = [&](int r) {
      const int jx = r - dra;
      return (va && jx >= 0 && jx < kTaps) ? geo.wx[(size_t)ka * kTaps + jx] : 0.f;
    };
    auto wxb = [&](int r) {
      const int jx = r - drb;
      return (vb && jx >= 0 && jx < kTaps) ? geo.wx[(size_t)kb * kTaps + jx] : 0.f;
    };
    float wa = r0 < r1 ? wxa(r0) : 0.f, wb = r0 < r1 ? wxb(r0) : 0.f;
    for (int r = r0; r < r1; ++r) {
      const float wan = wxa(r + 1), wbn = wxb(r + 1);
      const float* grow = s_g + (size_t)r * kItcWin * (2 * kItcProb);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (j < nj) {
          // two accumulation chains (even and odd column groups)
          float ta[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
          const int n = 8 * j + g;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const int c0 = 8 * kk + t, c1 = c0 + 4;
            uint32_t bh0, bl0, bh1, bl1;
            split_tf32(grow[c0 * (2 * kItcProb) + (n ^ itc_swz(c0))], bh0, bl0);
            split_tf32(grow[c1 * (2 * kItcProb) + (n ^ itc_swz(c1))], bh1, bl1);
            mma_tf32_1688(ta[kk & 1], al[kk], bh0, bh1);
            mma_tf32_1688(ta[kk & 1], ah[kk], bl0, bl1);
            mma_tf32_1688(ta[kk & 1], ah[kk], bh0, bh1);
          }
          d[j][0] = fmaf(wa, ta[0][0] + ta[1][0], d[j][0]);
          d[j][1] = fmaf(wa, ta[0][1] + ta[1][1], d[j][1]);
          d[j][2] = fmaf(wb, ta[0][2] + ta[1][2], d[j][2]);
          d[j][3] = fmaf(wb, ta[0][3] + ta[1][3], d[j][3]);
        }
      }
      wa = wan;
      wb = wbn;
    }
  }
  // row groups 1.. hand their partial sums to group 0 (through the window's
  // space: nobody reads it any more)
  __syncthreads();
  float* s_part = s_g;  // [8 warps][8 values][32 lanes]
  if (on && grp > 0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) s_part[(warp * 8 + q) * 32 + lane] = d[q >> 2][q & 3];
  }
  __syncthreads();
  if (on && grp == 0) {
    for (int gg = 1; gg < ng; ++gg) {
      const int w2 = blk + gg * nb;
#pragma unroll
      for (int q = 0; q < 8; ++q) d[q >> 2][q & 3] += s_part[(w2 * 8 + q) * 32 + lane];
    }
    // epilogue: lane (g, t) holds points g and g + 8, problems 4 j + t
    double chi[2] = {0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h ? vb : va) {
        const int k = h ? kb : ka;
        const double w = geo.weight[k], vr = geo.vis_r[k], vi = geo.vis_i[k];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int slot = 4 * j + t;
          if (slot < nact) {
            const size_t e = (size_t)s_list[slot] * geo.y2_bstride + k;
            double fr = (double)d[j][2 * h] * inv_mm, fi = (double)d[j][2 * h + 1] * inv_mm;
            if (ax_base) {
              const double2 ab = ax_base[e];
              fr += ab.x;
              fi += ab.y;
            }
            if (ax_out) ax_out[e] = make_double2(fr, fi);
            const double rr = (vr - fr) * w, ri = (vi - fi) * w;
            chi[j] += rr * rr + ri * ri;
            if (y2) y2[e] = mk<float>((float)(rr * w), (float)(ri * w));
          }
        }
      }
    }
    // chi^2: over g (fixed butterfly), then over the blocks in order
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double c = chi[j];
      c += __shfl_xor_sync(0xffffffffu, c, 4);
      c += __shfl_xor_sync(0xffffffffu, c, 8);
      c += __shfl_xor_sync(0xffffffffu, c, 16);
      if (g == 0) s_chi[warp][4 * j + t] = c;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nact && qchi >= 0) {
    double c = 0.0;
    for (int wp = 0; wp < nb; ++wp) c += s_chi[wp][threadIdx.x];
    part.at(qchi, s_list[threadIdx.x])[blockIdx.x] = c;
  }
}

// ---------------------------------------------------------------------------
// Spreading on the tensor cores (FP32 form, shared geometry)
//
// Output-stationary like k_nufft_spread_shared, in matrix form: the grid is
// cut into tiles of 8 rows x 16 columns of the stored half plane; a cell's
// value is a sum over "virtual points": every uv point once as itself
// (direct taps, first tap (mx - 11, my - 11), imaginary part negated: the
// reference's NU_SIGN) and once mirrored (first tap (-mx - 12, -my - 12),
// both weight vectors reversed, imaginary part kept), each with half the
// residual.  A tile's list holds every virtual point with a tap on it
// (built on the host, padded to a multiple of 8 with empty entries), so a
// cell (row r, column c) with virtual coordinates (mr, mc) (the reference's
// wrap: mr = r or r - 2Nx, mc = c or -Ny) is
//   sum_p wy_p[mc - my0_p] * (wx_p[mr - mx0_p] * y_p)      (taps outside: 0)
// For one row that is a 16 (columns) x K (points) by K x 16 (problem
// columns) product: warp w of the CTA takes tile row w and runs it as
// mma.sync m16n8k8 TF32 with the operands split in two TF32 parts
// (lo*hi + hi*lo + hi*hi, FP32 accumulation).  Everything but the residual
// depends on the geometry alone and is formed once, at plan creation
// (k_stc_prep): the A operand (the column weights, split hi / lo) in
// mma fragment order, 1 KB per 8 list entries, and the row weights wx at
// each of the tile's 8 rows (read from L2 inside the product loop: staging
// them in shared memory cost more in occupancy than it saved).  A launch
// gathers the residuals of its segment's points into shared memory and runs
// the products.  Long lists
// are cut into segments of kStcSeg points run by separate CTAs, which leave
// their partial tiles in a scratch buffer; the last of a tile's CTAs to
// finish (a ticket per tile and problem chunk) adds the segments in segment
// order and writes the tile, so the result does not depend on the order the
// CTAs ran in.
// ---------------------------------------------------------------------------
constexpr int kStcRows = 8, kStcCols = 16;
constexpr int kStcProb = 8;   // problems per CTA (16 real columns)
constexpr int kStcSeg = 256;  // list entries per CTA at most (longer lists are cut)
struct StcItem {
  int tile;           // tile index (row-major over tile rows x tile columns)
  int start, count;   // the segment's list entries: [start, start + count), count a multiple of 8
  int seg, nseg;      // segment index and count of this tile
  int scratch;        // scratch slot of segment 0 of the tile (nseg > 1)
};

// geometry-only operands of the tensor-core spreading, one thread per
// (group of 8 list entries, lane): the lane's A fragments (hi, lo) of the
// group, and the row weights of entry (group, lane & 7) at the tile's rows
// (lanes 0..7 only).  vlist: point | mirrored << 24, or -1 (padding);
// etile: each entry's tile.
static __global__ void k_stc_prep(const int* __restrict__ vlist, const int* __restrict__ etile, int nent,
                                  const int* __restrict__ mxa, const int* __restrict__ mya,
                                  const float* __restrict__ wxa, const float* __restrict__ wya, int nx, int ny,
                                  int ntcol, float* __restrict__ afrag, float* __restrict__ bxg) {
  const int gi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);  // group of 8 entries
  const int lane = threadIdx.x & 31;
  if (gi * 8 >= nent) return;
  const int g = lane >> 2, t = lane & 3;
  auto entry = [&](int e, int& k, int& x0, int& y0, int& fl) {
    const int v = vlist[e];
    if (v < 0) return false;
    k = v & 0xffffff;
    fl = (v >> 24) & 1;
    x0 = fl ? -mxa[k] - kMSP : mxa[k] - (kMSP - 1);
    y0 = fl ? -mya[k] - kMSP : mya[k] - (kMSP - 1);
    return true;
  };
  float* out = afrag + ((size_t)gi * 32 + lane) * 8;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    // fragment element q: column g (+8 for q odd), point t (+4 for q >= 2)
    const int cc = g + 8 * (q & 1), pe = gi * 8 + t + 4 * (q >> 1);
    int k, x0, y0, fl;
    float w = 0.f;
    if (entry(pe, k, x0, y0, fl)) {
      const int tcl = etile[pe] % ntcol;
      const int col = tcl * kStcCols + cc;
      const int mcol = col < ny ? col : -ny;
      const int jy = mcol - y0;
      if (col <= ny && jy >= 0 && jy < kTaps) w = wya[(size_t)k * kTaps + (fl ? kTaps - 1 - jy : jy)];
    }
    uint32_t hi, lo;
    split_tf32(w, hi, lo);
    out[q] = __uint_as_float(hi);
    out[4 + q] = __uint_as_float(lo);
  }
  if (lane < 8) {
    const int pe = gi * 8 + lane;
    int k, x0, y0, fl;
    const bool ok = entry(pe, k, x0, y0, fl);
    const int tr = ok ? etile[pe] / ntcol : 0;
    for (int r = 0; r < kStcRows; ++r) {
      const int row = tr * kStcRows + r;
      const int mrow = row < nx ? row : row - 2 * nx;
      const int jx = mrow - x0;
      float w = 0.f;
      if (ok && row < 2 * nx && jx >= 0 && jx < kTaps) w = wxa[(size_t)k * kTaps + (fl ? kTaps - 1 - jx : jx)];
      bxg[((size_t)gi * kStcRows + r) * 8 + lane] = w;
    }
  }
}

static __global__ void __launch_bounds__(256) k_nufft_spread_tc(
    NufftGeom<float> geo, const StcItem* __restrict__ items, const int* __restrict__ vlist,
    const float4* __restrict__ afrag, const float* __restrict__ bxg, const cplx<float>* __restrict__ y2,
    cplx<float>* __restrict__ gall, long gstride, int nx, int ny, int ntcol, const ProbState* __restrict__ st,
    int gate, int B, float* __restrict__ scratch, unsigned int* __restrict__ tickets) {
  __shared__ float s_y[kStcSeg * 24];  // [entry][16 problem columns] (row stride 24: conflict-free B loads)
  __shared__ int s_list[kStcProb];
  __shared__ int s_cnt[8];
  __shared__ unsigned int s_ticket;
  const int nact = active_chunk<kStcProb>(st, gate, B, blockIdx.y, s_list, s_cnt, geo.act_lists);
  if (nact == 0) return;
  const StcItem it = items[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int tr = it.tile / ntcol, tcl = it.tile - tr * ntcol;
  const int row = tr * kStcRows + warp;
  const int nj = nact > 4 ? 2 : 1;
  // the chunk's half residuals of the segment's entries, imaginary sign of
  // direct / mirrored taps (the only data that changes between launches)
  for (int e = threadIdx.x; e < it.count * 2 * kStcProb; e += blockDim.x) {
    const int q = e >> 4, n = e & 15, sl = n >> 1;
    float v = 0.f;
    const int code = vlist[it.start + q];
    if (code >= 0 && sl < nact) {
      const cplx<float> r = y2[(size_t)s_list[sl] * geo.y2_bstride + (code & 0xffffff)];
      v = (n & 1) ? (((code >> 24) & 1) ? 0.5f * r.y : -0.5f * r.y) : 0.5f * r.x;
    }
    s_y[q * 24 + n] = v;
  }
  __syncthreads();
  float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  const int g0 = it.start >> 3;  // first group of 8 entries
  for (int kb = 0; kb < it.count; kb += 8) {
    const int gi = g0 + (kb >> 3);
    const float4 h4 = __ldg(afrag + ((size_t)gi * 32 + lane) * 2);
    const float4 l4 = __ldg(afrag + ((size_t)gi * 32 + lane) * 2 + 1);
    const uint32_t ah[4] = {__float_as_uint(h4.x), __float_as_uint(h4.y), __float_as_uint(h4.z), __float_as_uint(h4.w)};
    const uint32_t al[4] = {__float_as_uint(l4.x), __float_as_uint(l4.y), __float_as_uint(l4.z), __float_as_uint(l4.w)};
    const float bx0 = __ldg(bxg + ((size_t)gi * kStcRows + warp) * 8 + t);
    const float bx1 = __ldg(bxg + ((size_t)gi * kStcRows + warp) * 8 + t + 4);
    const int p0 = (kb + t) * 24, p1 = (kb + t + 4) * 24;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (j < nj) {
        uint32_t bh0, bl0, bh1, bl1;
        split_tf32(bx0 * s_y[p0 + 8 * j + g], bh0, bl0);
        split_tf32(bx1 * s_y[p1 + 8 * j + g], bh1, bl1);
        mma_tf32_1688(d[j], al, bh0, bh1);
        mma_tf32_1688(d[j], ah, bl0, bl1);
        mma_tf32_1688(d[j], ah, bh0, bh1);
      }
    }
  }
  // lane (g, t) holds columns g and g + 8 of its row, problems 4 j + t
  const size_t cstride = (size_t)gridDim.y * 2048;
  if (it.nseg > 1) {
    float* mine = scratch + (size_t)(it.scratch + it.seg) * cstride + (size_t)blockIdx.y * 2048;
#pragma unroll
    for (int q = 0; q < 8; ++q) mine[(warp * 32 + lane) * 8 + q] = d[q >> 2][q & 3];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_ticket = atomicAdd(&tickets[(size_t)it.tile * gridDim.y + blockIdx.y], 1u);
    __syncthreads();
    if (s_ticket != (unsigned int)(it.nseg - 1)) return;
    __threadfence();
#pragma unroll
    for (int q = 0; q < 8; ++q) d[q >> 2][q & 3] = 0.f;
    for (int sg = 0; sg < it.nseg; ++sg) {
      const float* part = scratch + (size_t)(it.scratch + sg) * cstride + (size_t)blockIdx.y * 2048;
#pragma unroll
      for (int q = 0; q < 8; ++q) d[q >> 2][q & 3] += __ldcg(part + (warp * 32 + lane) * 8 + q);
    }
    if (threadIdx.x == 0) tickets[(size_t)it.tile * gridDim.y + blockIdx.y] = 0u;  // for the next launch
  }
  if (row >= 2 * nx) return;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int col = tcl * kStcCols + g + 8 * h;
    if (col <= ny) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int sl = 4 * j + t;
        if (sl < nact)
          gall[(size_t)s_list[sl] * gstride + (size_t)row * (ny + 1) + col] = mk<float>(d[j][2 * h], d[j][2 * h + 1]);
      }
    }
  }
}

// spreading: one thread-block cluster per (16 x 16 tile, problem chunk); one
// thread per cell holding the chunk's accumulators.  The tile's point list is
// split into contiguous segments, one per CTA of the cluster, which bounds
// the serial loop of the densest tiles; rank 0 then adds the segments'
// accumulators from the other CTAs' shared memory (DSMEM) in rank order, so
// the result is deterministic and no atomics are used.  Points (taps, the
// chunk's residuals and 16-bit masks of the tile rows / columns their direct
// or mirrored footprint covers) are staged through shared memory and read as
// broadcasts, so a point that misses a cell costs one mask test.
constexpr int kSpreadTile = 16;

// asynchronous global -> shared copies (cp.async): 4, 8 or 16 bytes

// shared-memory staging of one CTA of the spreading kernel: two buffers, so
// the points of the next round are copied in while this round is summed
template <typename T, int PB> struct SpreadSmem {
  static constexpr int P = 32;  // points staged per round
  struct Buf {
    __align__(16) T wx[P][kTaps];
    __align__(16) T wy[P][kTaps];
    __align__(16) cplx<T> r[P][PB];
    int mx[P], my[P];
  } buf[2];
  int list[PB];                 // the chunk's active problems, compacted
  int cnt;
};

// issues the copies of points [c0, c0 + np) of the tile's list into b:
// their grid indices, 24 + 24 tap weights (16-byte pieces) and the first
// NB slots' residuals (zero for slots >= cnt)
template <typename T, int PB, int NB>
__device__ __forceinline__ void spread_stage(const NufftGeom<T>& geo, const cplx<T>* __restrict__ y2, int c0, int np,
                                             int b0, int cnt, SpreadSmem<T, PB>& sm,
                                             typename SpreadSmem<T, PB>::Buf& b) {
  constexpr int kPieces = kTaps * sizeof(T) / 16;  // 16-byte pieces per point and axis
  for (int t = threadIdx.x; t < np; t += blockDim.x) {
    const int k = geo.tile_pts[c0 + t];
    cp_async(&b.mx[t], geo.mx + k, 4);
    cp_async(&b.my[t], geo.my + k, 4);
  }
  for (int t = threadIdx.x; t < np * 2 * kPieces; t += blockDim.x) {
    const int pp = t / (2 * kPieces), r = t - pp * 2 * kPieces;
    const int axis = r / kPieces, piece = r - axis * kPieces;
    const int k = geo.tile_pts[c0 + pp];
    const T* src = (axis ? geo.wy : geo.wx) + (size_t)k * kTaps + piece * (16 / sizeof(T));
    T* dst = (axis ? &b.wy[pp][0] : &b.wx[pp][0]) + piece * (16 / sizeof(T));
    cp_async(dst, src, 16);
  }
  for (int t = threadIdx.x; t < np * NB; t += blockDim.x) {
    const int pp = t / NB, i = t - pp * NB;
    if (i < cnt) {
      const int k = geo.tile_pts[c0 + pp];
      cp_async(&b.r[pp][i], y2 + (size_t)(b0 + sm.list[i]) * geo.y2_bstride + k, (int)sizeof(cplx<T>));
    } else {
      b.r[pp][i] = mk<T>(0, 0);
    }
  }
}

// Accumulates the tile's segment of points for the first NB active problems
// of the chunk (NB >= cnt) and writes the cluster's sum.  NB is a compile-time
// bound so that a chunk with few active problems (the tail of a lambda grid)
// runs a short FMA loop while a full chunk keeps a fully unrolled one.
// Points come in rounds of P through the two shared buffers: the copies of
// round r + 1 (cp.async) are in flight while round r is summed.
template <typename T, int PB, int NB>
__device__ __forceinline__ void spread_tile(const NufftGeom<T>& geo, const cplx<T>* __restrict__ y2,
                                            cplx<T>* __restrict__ gall, long gstride, int nx, int ny, int tile,
                                            int b0, int cnt, SpreadSmem<T, PB>& sm, cplx<T>* s_acc,
                                            cg::cluster_group& cluster, int rank, int csize) {
  constexpr int P = SpreadSmem<T, PB>::P;
  constexpr int TILE = kSpreadTile;
  const int ntc = (ny + 1 + TILE - 1) / TILE;
  const int tr = tile / ntc, tc = tile - tr * ntc;
  const int ty = threadIdx.x / TILE, tx = threadIdx.x - ty * TILE;
  const int row = tr * TILE + ty, col = tc * TILE + tx;
  const bool valid = row < 2 * nx && col <= ny;
  const int mrow = row < nx ? row : row - 2 * nx;
  const int mcol = col < ny ? col : -ny;
  T ar[NB], ai[NB];
#pragma unroll
  for (int i = 0; i < NB; ++i) ar[i] = ai[i] = 0;
  const int lbeg = geo.tile_ptr[tile], lend = geo.tile_ptr[tile + 1];
  const int seg = (lend - lbeg + csize - 1) / csize;
  const int beg = min(lend, lbeg + rank * seg), end = min(lend, beg + seg);
  const int rounds = (end - beg + P - 1) / P;
  if (rounds > 0) spread_stage<T, PB, NB>(geo, y2, beg, min(P, end - beg), b0, cnt, sm, sm.buf[0]);
  cp_async_commit();
  for (int rd = 0; rd < rounds; ++rd) {
    const int c0 = beg + rd * P;
    const int np = min(P, end - c0);
    if (rd + 1 < rounds)
      spread_stage<T, PB, NB>(geo, y2, c0 + P, min(P, end - c0 - P), b0, cnt, sm, sm.buf[(rd + 1) & 1]);
    cp_async_commit();
    cp_async_wait<1>();  // this thread's copies of round rd have landed
    __syncthreads();     // and everyone's
    const typename SpreadSmem<T, PB>::Buf& b = sm.buf[rd & 1];
    if (valid) {
      for (int pp = 0; pp < np; ++pp) {
        const int ox = (kMSP - 1) - b.mx[pp], oy = (kMSP - 1) - b.my[pp];
        const int lxd = mrow + ox, lyd = mcol + oy;
        const int lxm = ox - mrow, lym = oy - mcol;
        const bool d = (unsigned)lxd < (unsigned)kTaps && (unsigned)lyd < (unsigned)kTaps;
        const bool mi = (unsigned)lxm < (unsigned)kTaps && (unsigned)lym < (unsigned)kTaps;
        if (!(d || mi)) continue;
        // the reference adds the two contributions of one point in ly order
        const bool mfirst = mi && d && lym < lyd;
        for (int pass = 0; pass < 2; ++pass) {
          const bool use_m = (pass == 0) ? mfirst : (mi && !mfirst);
          const bool use_d = (pass == 0) ? (d && !mfirst) : (d && mfirst);
          if (!(use_m || use_d)) continue;
          const T w = use_m ? b.wy[pp][lym] * b.wx[pp][lxm] : b.wy[pp][lyd] * b.wx[pp][lxd];
          const T hw = w * T(0.5);
          // the staged residual keeps its sign; NU_SIGN on Fin_i is folded
          // into the imaginary weight (exact: (-a) b == a (-b))
          const T hwi = use_m ? hw : -hw;
#pragma unroll
          for (int i = 0; i < NB; ++i) {
            cplx<T> r = b.r[pp][i];
            ar[i] += r.x * hw;
            ai[i] += r.y * hwi;
          }
        }
      }
    }
    __syncthreads();  // buffer rd & 1 is refilled by the copies issued in the next round
  }
  // segment accumulators -> shared memory; rank 0 adds ranks 1.. in order
#pragma unroll
  for (int i = 0; i < NB; ++i) s_acc[i * 256 + threadIdx.x] = mk<T>(ar[i], ai[i]);
  cluster.sync();
  if (rank == 0) {
    for (int r = 1; r < csize; ++r) {
      const cplx<T>* peer = cluster.map_shared_rank(s_acc, r);
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        cplx<T> v = peer[i * 256 + threadIdx.x];
        ar[i] += v.x;
        ai[i] += v.y;
      }
    }
    if (valid) {
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (i < cnt) gall[(size_t)(b0 + sm.list[i]) * gstride + (size_t)row * (ny + 1) + col] = mk<T>(ar[i], ai[i]);
    }
  }
  cluster.sync();  // peers' shared memory must stay alive until rank 0 is done
}

template <typename T>
__global__ void __launch_bounds__(256, SharedChunk<T>::kSpreadMinBlocks) k_nufft_spread_shared(NufftGeom<T> geo, const cplx<T>* __restrict__ y2,
                                                                cplx<T>* __restrict__ gall, long gstride, int nx,
                                                                int ny, int ntiles, const ProbState* __restrict__ st,
                                                                int gate, int B) {
  constexpr int PB = SharedChunk<T>::kSpread;
  static_assert(kSpreadTile == 16, "the footprint masks use 16 row and 16 column bits");
  static_assert(PB % 4 == 0, "problem chunks are multiples of 4");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* s_acc = reinterpret_cast<cplx<T>*>(smem_raw);  // [PB][256] segment accumulators
  __shared__ SpreadSmem<T, PB> sm;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int csize = (int)cluster.num_blocks();
  // chunks over the batch's active problems (list: problem indices)
  __shared__ int s_cnt[8];
  const int cnt = active_chunk<PB>(st, gate, B, blockIdx.y, sm.list, s_cnt, geo.act_lists);
  if (cnt == 0) return;  // uniform over the cluster: same problem chunk
  const int b0 = 0;
  // densest tiles first, so that the longest clusters start in the first wave
  const int tile = geo.tile_order ? geo.tile_order[blockIdx.x / csize] : blockIdx.x / csize;
  // accumulator slot i holds problem b0 + list[i]: the smallest unrolled
  // width that holds the chunk's active problems
  if (cnt == 1)
    spread_tile<T, PB, 1>(geo, y2, gall, gstride, nx, ny, tile, b0, cnt, sm, s_acc, cluster, rank, csize);
  else if (cnt == 2)
    spread_tile<T, PB, 2>(geo, y2, gall, gstride, nx, ny, tile, b0, cnt, sm, s_acc, cluster, rank, csize);
  else if (cnt <= 4)
    spread_tile<T, PB, 4>(geo, y2, gall, gstride, nx, ny, tile, b0, cnt, sm, s_acc, cluster, rank, csize);
  else if (PB > 8 && cnt <= 8)
    spread_tile<T, PB, (PB > 8 ? 8 : PB)>(geo, y2, gall, gstride, nx, ny, tile, b0, cnt, sm, s_acc, cluster, rank,
                                          csize);
  else
    spread_tile<T, PB, PB>(geo, y2, gall, gstride, nx, ny, tile, b0, cnt, sm, s_acc, cluster, rank, csize);
}

}  // namespace mf

// ===========================================================================
// Forward model at the momentum point by linearity (corrected FP32 form).
// MFISTA's momentum point is z = a x + b xnew with a, b set by the control
// step (and x <- xnew when the trial improves the objective), so with the
// models kept as visibility vectors ax = A x and axn = A xnew (written by
// the trial point's forward pass), A z = a ax + b axn needs no NUFFT.
// Vectors use the residual layout (problem b, point k at b y2_bstride + k).
// ===========================================================================
namespace mf {

// weighted residual (vis - az) w^2 for the adjoint and its chi^2 partials.
// The partials are summed in exactly the order of the interpolation kernel
// that produces the same quantity for a trial point (k_nufft_interp_shared
// with ppw points per warp, or k_nufft_interp with one point per warp), so
// when the trial point equals z (a problem resting at x = 0, say) F(xnew)
// and the f(z) inside Q agree to the bit and the backtracking test is not
// decided by rounding.  Grid (cdiv(chi slots, 8), B) for shared geometry
// (one warp per slot), (chi slots, B) otherwise; 256 threads.
template <typename T> __device__ __forceinline__ int slots_of(const NufftGeom<T>& geo, int ppw) {
  const int m = geo.pt_hi[0];
  return max(1, (m + 8 * ppw - 1) / (8 * ppw));
}

template <typename T>
__global__ void k_nufft_resid_model(NufftGeom<T> geo, const double2* __restrict__ az, cplx<T>* __restrict__ y2,
                                    int shared, int ppw, int nslots, const ProbState* __restrict__ st, int gate,
                                    Partials part, int qchi) {
  __shared__ double sh[32];
  const int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  auto term = [&](int k) {
    const size_t e = (size_t)b * geo.y2_bstride + k;
    const double2 m = az[e];
    const double w = geo.weight[k];
    const double rr = (geo.vis_r[k] - m.x) * w, ri = (geo.vis_i[k] - m.y) * w;
    y2[e] = mk<T>((T)(rr * w), (T)(ri * w));
    return rr * rr + ri * ri;
  };
  if (shared) {
    // one warp per slot (a CTA of the interpolation: 8 warps x ppw points);
    // the terms go through shared memory and lane 0 adds them in the
    // interpolation's order (per warp w in q order, then over w)
    __shared__ double s_t[8][8 * 32];
    const int slot = blockIdx.x * 8 + warp;
    if (slot >= slots_of(geo, ppw)) {  // a slot beyond the points (padding for another kernel's CTAs)
      if (lane == 0 && qchi >= 0 && slot < nslots) part.at(qchi, b)[slot] = 0.0;
      return;
    }
    const int mtot = geo.pt_hi[0];
    const int n = 8 * ppw, k0 = slot * n;
    for (int l = lane; l < n; l += 32) s_t[warp][l] = (k0 + l < mtot) ? term(k0 + l) : 0.0;
    __syncwarp();
    if (lane == 0 && qchi >= 0) {
      double tot = 0.0;
      for (int w = 0; w < 8; ++w) {
        double c = 0.0;
        for (int q = 0; q < ppw; ++q)
          if (k0 + w * ppw + q < mtot) c += s_t[warp][w * ppw + q];
        tot += c;
      }
      part.at(qchi, b)[slot] = tot;
    }
  } else {
    // one point per warp, reduced over the CTA as k_nufft_interp does
    const int k = geo.pt_lo[b] + blockIdx.x * 8 + warp;
    double chi[1] = {0.0};
    if (lane == 0 && k < geo.pt_hi[b]) chi[0] = term(k);
    block_sum<1>(chi, sh);
    if (threadIdx.x == 0 && qchi >= 0) part.at(qchi, b)[blockIdx.x] = chi[0];
  }
}

// ax = src (and az = src when az is given) for the problems passing `gate`
static __global__ void k_nufft_model_set(const int* __restrict__ pt_lo, const int* __restrict__ pt_hi, long bstride,
                                  const double2* __restrict__ src, double2* __restrict__ ax,
                                  double2* __restrict__ az, const ProbState* __restrict__ st, int gate) {
  const int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const int k = pt_lo[b] + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= pt_hi[b]) return;
  const size_t e = (size_t)b * bstride + k;
  ax[e] = src[e];
  if (az) az[e] = src[e];
}

}  // namespace mf
