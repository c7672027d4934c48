// Host side of the solver: FFT plans, the three operators (NUFFT, gridded
// FFT, dense DFT), and the batched MFISTA driver that records one MFISTA
// step as a CUDA graph body and repeats it on the device with a conditional
// WHILE node until every problem of the batch has stopped.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "dft_ops.cuh"
#include "dft_tc.cuh"
#include "fft_smem.cuh"
#include "fftvar_ops.cuh"
#include "fgp.cuh"
#include "mfista_ops.cuh"
#include "nufft_ops.cuh"

#include "../../include/mfista_b200.h"

namespace mf {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define MF_CK(x)                                                                                          \
  do {                                                                                                    \
    cudaError_t e_ = (x);                                                                                 \
    if (e_ != cudaSuccess)                                                                                \
      throw ::mf::Error(e_ == cudaErrorMemoryAllocation ? MFISTA_ERR_NOMEM : MFISTA_ERR_CUDA,             \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                                 \
  } while (0)

#define MF_LAUNCH_CK() MF_CK(cudaGetLastError())

struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
  DevMem() {}
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() { release(); }
  void alloc(size_t n) {
    release();
    if (n) MF_CK(cudaMalloc(&p, n));
    bytes = n;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename U> U* as() const { return reinterpret_cast<U*>(p); }
  template <typename U> void upload(const U* h, size_t count) {
    alloc(count * sizeof(U));
    if (count) MF_CK(cudaMemcpy(p, h, count * sizeof(U), cudaMemcpyHostToDevice));
  }
};

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// FFT plans
// ---------------------------------------------------------------------------
template <typename T> void make_twiddles(int n, DevMem& mem) {
  std::vector<cplx<T>> h(std::max(n, 1));
  for (int k = 0; k < n; ++k) {
    long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
    h[k] = mk<T>((T)cosl(a), (T)(-sinl(a)));
  }
  mem.upload(h.data(), h.size());
}

template <typename T> struct FftHost {
  FftDev<T> dev;
  DevMem tw;
  void init(int n) {
    memset(&dev, 0, sizeof(dev));
    dev.n = n;
    int m = n;
    auto push = [&](int r) {
      if (dev.nst >= kMaxStages) throw Error(MFISTA_ERR_ARG, "FFT length has too many factors");
      dev.radix[dev.nst++] = r;
    };
    while (m % 4 == 0) { push(4); m /= 4; }
    while (m % 2 == 0) { push(2); m /= 2; }
    while (m % 3 == 0) { push(3); m /= 3; }
    while (m % 5 == 0) { push(5); m /= 5; }
    for (int f = 7; m > 1 && f <= kMaxGenericRadix; f += 2)
      while (m % f == 0) { push(f); m /= f; }
    if (m > 1) throw Error(MFISTA_ERR_ARG, "FFT length " + std::to_string(n) + " has a prime factor above 16");
    make_twiddles<T>(n, tw);
    dev.tw = tw.as<cplx<T>>();
  }
};

// Raises a kernel's dynamic shared-memory limit to at least `bytes`.  The
// limit is per kernel and process-wide, so it is never lowered: another plan
// may have captured launches that need more.
template <typename K> void set_smem(K kernel, size_t bytes) {
  if (bytes > 227 * 1024) throw Error(MFISTA_ERR_ARG, "grid too large for the shared-memory FFT");
  cudaFuncAttributes fa;
  MF_CK(cudaFuncGetAttributes(&fa, kernel));
  if ((size_t)fa.maxDynamicSharedSizeBytes < bytes)
    MF_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// ---------------------------------------------------------------------------
// common solver context shared by the operators
// ---------------------------------------------------------------------------
struct Ctx {
  int B = 0;
  int N = 0;
  long xstride = 0;
  int tsvNX = 0, tsvNY = 0;  // TSV/TV view (reference's NX, NY)
  double* x = nullptr;
  double* z = nullptr;
  double* xnew = nullptr;
  double* dfdx = nullptr;
  double* xa = nullptr;  // FP32 form: anchor images of the defect correction
  ProbParams* prm = nullptr;
  ProbState* st = nullptr;
  Partials part{};
  // per-step gate lists (k_select_blocks), given to the kernels captured in
  // the device loop's body; null everywhere else
  const int* act_lists = nullptr;
};

// Launch shapes of the operator kernels that the autotuner may change.
//   interp_ppw:     points per warp of the shared-geometry interpolation
//   spread_cluster: CTAs per tile cluster of the shared-geometry spreading
//   rows_per_cta:   image rows per CTA of the row FFT passes
//   cols_per_cta:   grid columns per CTA of the column FFT passes
// 0 means "not used by this operator".  Row/column shapes leave every
// result bit-identical; the interpolation and spreading shapes regroup sums
// (chi^2 partials; spreading segments), which moves results by rounding only.
struct LaunchShapes {
  int interp_ppw = 0, spread_cluster = 0, rows_per_cta = 0, cols_per_cta = 0;
};

struct Op {
  virtual ~Op() {}
  // chi^2 partials of `src` into part[qchi]; `store` keeps the weighted
  // residual for the next adjoint()
  virtual void forward(cudaStream_t s, const double* src, int gate, int qchi, bool store) = 0;
  // gradient at z into ctx.dfdx (gate: need_grad); TSV fused when z_tsv != 0
  virtual void adjoint(cudaStream_t s, const double* z_tsv, int qtsv) = 0;
  virtual int chi_slots() const = 0;
  // largest chi_slots() over every launch shape set_shapes() accepts
  virtual int max_chi_slots() const { return chi_slots(); }
  virtual int tsv_slots() const = 0;
  virtual LaunchShapes shapes() const { return LaunchShapes(); }
  // throws Error(MFISTA_ERR_ARG) for a shape the operator cannot run
  virtual void set_shapes(const LaunchShapes& sh) { (void)sh; }
  virtual double fscale() const = 0;
  virtual int launches_forward() const = 0;
  virtual int launches_adjoint() const = 0;
  // one kernel alone (profiling): 0 interp, 1 spread, 2 rows fwd, 3 cols fwd,
  // 4 cols inv, 5 rows inv; returns its algorithmic bytes (compulsory reads
  // and writes of one launch over the whole batch), or < 0 if not defined
  virtual double launch_single(cudaStream_t s, int kernel) { (void)s; (void)kernel; return -1; }
  // defect correction (FP32 operators): recompute the exact FP64 model of the
  // anchors ctx.xa for the problems passing `gate`; forward_exact evaluates
  // chi^2 with the FP64 operator (initial and final objective)
  virtual bool corrected() const { return false; }
  virtual void refresh_anchor(cudaStream_t s, int gate) { (void)s; (void)gate; }
  virtual void forward_exact(cudaStream_t s, const double* src, int gate, int qchi, bool store) {
    forward(s, src, gate, qchi, store);
  }
  virtual int launches_refresh() const { return 0; }
  // non-zero when a device-side wait of the operator's kernels gave up
  virtual int device_error() { return 0; }
  // outer iterations between anchor refreshes of the corrected forms
  virtual int refresh_period() const { return 32; }
  // forward model at the momentum point z by linearity from kept models of
  // x and of the trial point (operators that keep them return true):
  // forward_z replaces forward(z, ...) (residual kept, chi^2 into qchi);
  // model_momentum gives k_momentum the models to update with the images
  virtual bool models_z() const { return false; }
  virtual void forward_z(cudaStream_t s, int gate, int qchi) { (void)s; (void)gate; (void)qchi; }
  virtual ModelMom model_momentum(int img_blocks) {
    ModelMom m;
    memset(&m, 0, sizeof(m));
    m.img_blocks = img_blocks;
    return m;
  }
  virtual int model_blocks() const { return 0; }
};

// ---------------------------------------------------------------------------
// NUFFT operator
// ---------------------------------------------------------------------------
struct NufftInput {
  const double *u, *v, *vis_r, *vis_i, *vis_std;
  const int* pt_off;  // B+1 (independent geometry) or null
  int shared;
  int M;              // points per problem (shared) or total
  int Nx, Ny;
};

// host binning of points to spread tiles (direct and mirrored footprints)
inline void bin_points(const std::vector<int>& mx, const std::vector<int>& my, int lo, int hi, int nx, int ny,
                       int tile_r, int tile_c, std::vector<std::vector<int>>& lists) {
  int ntc = cdiv(ny + 1, tile_c);
  std::vector<int> tr, tc, ids;
  for (int k = lo; k < hi; ++k) {
    ids.clear();
    for (int mir = 0; mir < 2; ++mir) {
      tr.clear();
      tc.clear();
      int sg = mir ? -1 : 1;
      for (int l = 0; l < kTaps; ++l) {
        int r = wrap_row(sg * (mx[k] + l - (kMSP - 1)), nx);
        if (r >= 0) tr.push_back(r / tile_r);
        int c = half_col(sg * (my[k] + l - (kMSP - 1)), ny);
        if (c >= 0) tc.push_back(c / tile_c);
      }
      std::sort(tr.begin(), tr.end());
      tr.erase(std::unique(tr.begin(), tr.end()), tr.end());
      std::sort(tc.begin(), tc.end());
      tc.erase(std::unique(tc.begin(), tc.end()), tc.end());
      for (int a : tr)
        for (int c : tc) ids.push_back(a * ntc + c);
    }
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    for (int t : ids) lists[t].push_back(k);
  }
}

template <typename T> struct NufftOp : Op {
  Ctx& c;
  int nx, ny, B, mtot, mmax;
  bool shared;
  std::unique_ptr<NufftOp<double>> exact;  // FP64 operator for the anchors
  DevMem d_axa;                            // exact model of the anchors [y2 layout]
  DevMem d_ax, d_axn, d_az;                // models of x, the trial point and z [y2 layout]
  bool model = false;                      // forward at z by linearity (corrected form)
  DevMem d_u, d_v, d_mx, d_my, d_wx, d_wy, d_vr, d_vi, d_w, d_lo, d_hi, d_tptr, d_tpts, d_e4, d_grid, d_y2, tw2h;
  DevMem d_tord;  // shared geometry: spreading tiles by falling point count
  FftHost<T> fh, fcol;
  NufftGeom<T> geo{};
  // default launch shapes: the autotuner's choice on the 128 x 128 lambda
  // grid with the tensor-core interpolation and spreading (8 rows and 8
  // columns per CTA)
  int rpc = 8, cpc = 8, tile_r = 8, tile_c = 32, ntiles = 0;
  int ippw = SharedChunk<T>::kInterpPts;  // interpolation points per warp (shared geometry)
  int spread_cs = 8;                      // spreading cluster size (shared geometry)
  // FP32 grouped interpolation with taps formed on the fly (fewer registers;
  // measured 8 % / 17 % faster with 64 / 1 problems active on the lambda
  // grid, 7 % slower with 16) instead of held in registers; both give the
  // same bits (MFISTA_INTERP_FLY=0 selects the register form)
  bool interp_fly = true;
  // FP32, shared geometry: interpolation on the tensor cores (k_nufft_interp_tc;
  // MFISTA_INTERP_TC=0 selects the CUDA-core kernels above)
  bool interp_tc = false;
  DevMem d_itc, d_iperm;  // its CTA tiles and the points in tile order
  int ntc = 0;
  // FP32, shared geometry: spreading on the tensor cores (k_nufft_spread_tc;
  // MFISTA_SPREAD_TC=0 selects the cluster kernel)
  bool spread_tc = false;
  DevMem d_sitems, d_svlist, d_sscratch, d_stickets, d_safrag, d_sbx;
  int nsitems = 0, stc_cols = 0;
  // chi^2 partial slots every interpolation kernel of this operator writes
  // (at least its own CTA count; the extra CTAs write zeros), so that the
  // CUDA-core, tensor-core and FP64 kernels fill the same slots
  int chi_pad = 0;
  size_t smem_rows = 0, smem_cols = 0;
  long gstride = 0;
  double inv_mm = 0;

  NufftOp(Ctx& ctx, const NufftInput& in, bool correct = false) : c(ctx) {
    if (const char* f = getenv("MFISTA_INTERP_FLY")) interp_fly = f[0] == '1';
    if (const char* f = getenv("MFISTA_FFT_DYN")) fft_dyn = f[0] != '0';
    if (sizeof(T) == 4 && in.shared != 0 && in.M < kItcMaxPoints) {
      const char* f = getenv("MFISTA_INTERP_TC");
      interp_tc = !(f && f[0] == '0');
      const char* f2 = getenv("MFISTA_SPREAD_TC");
      spread_tc = !(f2 && f2[0] == '0');
    }
    // with the tensor-core interpolation the points-per-warp knob only sets
    // the FP64 anchor interpolation's and the model residual's partition:
    // 8 points per warp (the autotuner's choice on the lambda grid) keeps
    // the chi^2 slot count at the tile count
    if (interp_tc) ippw = 8;
    nx = in.Nx;
    ny = in.Ny;
    B = ctx.B;
    shared = in.shared != 0;
    if (nx < 12 || ny < 12) throw Error(MFISTA_ERR_ARG, "NUFFT needs Nx, Ny >= 12");
    mtot = in.M;
    std::vector<int> lo(B), hi(B);
    if (shared) {
      for (int b = 0; b < B; ++b) { lo[b] = 0; hi[b] = mtot; }
    } else {
      mtot = in.pt_off[B];
      for (int b = 0; b < B; ++b) { lo[b] = in.pt_off[b]; hi[b] = in.pt_off[b + 1]; }
    }
    mmax = 0;
    for (int b = 0; b < B; ++b) mmax = std::max(mmax, hi[b] - lo[b]);
    // grid indices of the points (preNUFFT :92-96), on the host so that the
    // binning below and the device agree exactly
    std::vector<int> mx(mtot), my(mtot);
    const double pi = 3.14159265358979323846;
    double mrx = 2.0 * nx, mry = 2.0 * ny;
    for (int k = 0; k < mtot; ++k) {
      mx[k] = (int)round(in.u[k] * mrx / (2 * pi));
      my[k] = (int)round(in.v[k] * mry / (2 * pi));
    }
    std::vector<double> w(mtot);
    for (int k = 0; k < mtot; ++k) w[k] = 1 / in.vis_std[k];
    d_u.upload(in.u, mtot);
    d_v.upload(in.v, mtot);
    d_mx.upload(mx.data(), mtot);
    d_my.upload(my.data(), mtot);
    d_vr.upload(in.vis_r, mtot);
    d_vi.upload(in.vis_i, mtot);
    d_w.upload(w.data(), mtot);
    d_lo.upload(lo.data(), B);
    d_hi.upload(hi.data(), B);
    d_wx.alloc(sizeof(T) * (size_t)std::max(mtot, 1) * kTaps);
    d_wy.alloc(sizeof(T) * (size_t)std::max(mtot, 1) * kTaps);
    if (mtot > 0) {
      k_nufft_prep_points<T><<<cdiv(mtot, 256), 256>>>(d_u.as<double>(), d_v.as<double>(), d_mx.as<int>(),
                                                        d_my.as<int>(), mtot, nx, ny, d_wx.as<T>(), d_wy.as<T>());
      MF_LAUNCH_CK();
    }
    d_e4.alloc(sizeof(double) * nx * ny);
    k_nufft_prep_e4<<<cdiv(nx * ny, 256), 256>>>(d_e4.as<double>(), nx, ny);
    MF_LAUNCH_CK();
    // spread tiles (16 x 16 for the shared-geometry kernels)
    if (shared) tile_r = tile_c = 16;
    ntiles = cdiv(2 * nx, tile_r) * cdiv(ny + 1, tile_c);
    int ngeo = shared ? 1 : B;
    std::vector<int> tptr;
    std::vector<int> tpts;
    tptr.reserve((size_t)ngeo * ntiles + 1);
    tptr.push_back(0);
    for (int g = 0; g < ngeo; ++g) {
      std::vector<std::vector<int>> lists(ntiles);
      bin_points(mx, my, lo[g], hi[g], nx, ny, tile_r, tile_c, lists);
      for (int t = 0; t < ntiles; ++t) {
        tpts.insert(tpts.end(), lists[t].begin(), lists[t].end());
        tptr.push_back((int)tpts.size());
      }
    }
    d_tptr.upload(tptr.data(), tptr.size());
    d_tpts.upload(tpts.data(), std::max<size_t>(tpts.size(), 1));
    if (shared) {  // spreading launch order: tiles by falling point count (ties by index)
      std::vector<int> ord(ntiles);
      for (int t = 0; t < ntiles; ++t) ord[t] = t;
      std::stable_sort(ord.begin(), ord.end(),
                       [&](int a, int b) { return tptr[a + 1] - tptr[a] > tptr[b + 1] - tptr[b]; });
      d_tord.upload(ord.data(), ord.size());
    }
    if (interp_tc) build_itc_tiles(mx, my);
    if (spread_tc) build_stc_items(mx, my);
    // FFTs: rows as complex length Ny, columns length 2Nx
    fh.init(ny);
    fcol.init(2 * nx);
    make_twiddles<T>(2 * ny, tw2h);
    gstride = (long)2 * nx * (ny + 1);
    d_grid.alloc(sizeof(cplx<T>) * (size_t)B * gstride);
    long y2n = shared ? (long)B * std::max(mtot, 1) : std::max(mtot, 1);
    d_y2.alloc(sizeof(cplx<T>) * (size_t)y2n);
    inv_mm = 1.0 / ((double)(2 * nx) * (double)(2 * ny));
    // launch shapes: keep the ping-pong buffers within shared memory
    auto rows_smem = [&](int r) { return (size_t)2 * r * (ny + 1) * sizeof(cplx<T>); };
    auto cols_smem = [&](int cc) { return (size_t)2 * cc * (2 * nx + 1) * sizeof(cplx<T>); };
    while (rpc > 1 && rows_smem(rpc) > 96 * 1024) rpc /= 2;
    while (cpc > 1 && cols_smem(cpc) > 96 * 1024) cpc /= 2;
    smem_rows = rows_smem(rpc);
    smem_cols = cols_smem(cpc);
    set_smem(k_nufft_rows_fwd<T>, smem_rows);
    set_smem(k_nufft_rows_inv<T>, smem_rows);
    set_smem(k_nufft_cols<T>, smem_cols);
    set_smem(k_nufft_spread_shared<T>, spread_smem());
    MF_CK(cudaFuncSetAttribute(k_nufft_spread_shared<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    if (correct && sizeof(T) == 4) {
      exact.reset(new NufftOp<double>(ctx, in, false));
      exact->ippw = ippw;  // its chi^2 partials land in the same slots as ours
      exact->chi_pad = chi_pad;
      d_axa.alloc(sizeof(double2) * (size_t)y2n);
      const char* nm = getenv("MFISTA_NO_MODEL_Z");  // direct forward at z instead (comparison runs)
      model = !(nm && nm[0] == '1');
      if (model) {
        for (DevMem* d : {&d_ax, &d_axn, &d_az}) {
          d->alloc(sizeof(double2) * (size_t)y2n);
          MF_CK(cudaMemset(d->p, 0, d->bytes));
        }
      }
      MF_CK(cudaMemset(d_axa.p, 0, d_axa.bytes));
    }
    geo.mx = d_mx.as<int>();
    geo.my = d_my.as<int>();
    geo.wx = d_wx.as<T>();
    geo.wy = d_wy.as<T>();
    geo.vis_r = d_vr.as<double>();
    geo.vis_i = d_vi.as<double>();
    geo.weight = d_w.as<double>();
    geo.pt_lo = d_lo.as<int>();
    geo.pt_hi = d_hi.as<int>();
    geo.tile_ptr = d_tptr.as<int>();
    geo.tile_pts = d_tpts.as<int>();
    geo.tile_order = shared ? d_tord.as<int>() : nullptr;
    geo.tile_bstride = shared ? 0 : ntiles;
    geo.y2_bstride = shared ? mtot : 0;
    geo.e4 = d_e4.as<double>();
    MF_CK(cudaDeviceSynchronize());
  }

  int interp_blocks() const { return std::max({1, cdiv(mmax, shared ? 8 * ippw : 8), chi_pad}); }

  // Tensor-core spreading: each 8 x 16 tile of the stored half grid lists
  // the virtual points (point | mirrored << 24) with a tap on it, in (point,
  // mirrored) order; a tile's list is cut into CTA segments of kStcSeg.
  void build_stc_items(const std::vector<int>& mx, const std::vector<int>& my) {
    const int ntr = cdiv(2 * nx, kStcRows);
    stc_cols = cdiv(ny + 1, kStcCols);
    const int nt = ntr * stc_cols;
    std::vector<std::vector<int>> lists(nt);
    std::vector<int> trs, tcs;
    for (int k = 0; k < mtot; ++k)
      for (int fl = 0; fl < 2; ++fl) {
        const int x0 = fl ? -mx[k] - kMSP : mx[k] - (kMSP - 1);
        const int y0 = fl ? -my[k] - kMSP : my[k] - (kMSP - 1);
        trs.clear();
        tcs.clear();
        for (int v = x0; v < x0 + kTaps; ++v) {  // stored rows of the taps (the reference's wrap)
          const int r = (v >= 0 && v < nx) ? v : (v >= -nx && v < 0) ? v + 2 * nx : -1;
          if (r >= 0 && (trs.empty() || trs.back() != r / kStcRows)) trs.push_back(r / kStcRows);
        }
        for (int v = y0; v < y0 + kTaps; ++v) {  // stored columns (0..Ny-1 direct, -Ny -> Ny)
          const int c = (v >= 0 && v < ny) ? v : (v == -ny) ? ny : -1;
          if (c >= 0 && std::find(tcs.begin(), tcs.end(), c / kStcCols) == tcs.end()) tcs.push_back(c / kStcCols);
        }
        std::sort(trs.begin(), trs.end());
        trs.erase(std::unique(trs.begin(), trs.end()), trs.end());
        for (int a : trs)
          for (int b : tcs) lists[(size_t)a * stc_cols + b].push_back(k | (fl << 24));
      }
    // every tile's list padded to a multiple of 8 (empty entries: -1), so that
    // the groups of 8 entries of the prepared operands never straddle tiles
    std::vector<int> flat, etile;
    std::vector<StcItem> items;
    int nscr = 0;
    // list entries per CTA: kStcSeg, or fewer (a multiple of 8) from MFISTA_SPREAD_SEG
    int seg = kStcSeg;
    if (const char* e = getenv("MFISTA_SPREAD_SEG")) seg = std::max(8, std::min(kStcSeg, atoi(e) & ~7));
    for (int t = 0; t < nt; ++t) {
      const int start = (int)flat.size();
      const int cnt = ((int)lists[t].size() + 7) & ~7;
      flat.insert(flat.end(), lists[t].begin(), lists[t].end());
      flat.resize((size_t)start + cnt, -1);
      etile.resize(flat.size(), t);
      const int nseg = std::max(1, cdiv(cnt, seg));
      for (int sg = 0; sg < nseg; ++sg)
        items.push_back(StcItem{t, start + sg * seg, std::min(seg, cnt - sg * seg), sg, nseg, nscr});
      if (nseg > 1) nscr += nseg;
    }
    // launch order: longest segments first
    std::stable_sort(items.begin(), items.end(), [](const StcItem& a, const StcItem& b) { return a.count > b.count; });
    nsitems = (int)items.size();
    const int nent = (int)flat.size(), ngrp = std::max(1, nent / 8);
    d_sitems.upload(items.data(), items.size());
    d_svlist.upload(flat.data(), std::max<size_t>(flat.size(), 1));
    DevMem d_etile;
    d_etile.upload(etile.data(), std::max<size_t>(etile.size(), 1));
    d_safrag.alloc(sizeof(float) * (size_t)ngrp * 256);
    d_sbx.alloc(sizeof(float) * (size_t)ngrp * kStcRows * 8);
    if (nent > 0) {
      k_stc_prep<<<cdiv(ngrp, 8), 256>>>(d_svlist.as<int>(), d_etile.as<int>(), nent, d_mx.as<int>(), d_my.as<int>(),
                                          d_wx.as<float>(), d_wy.as<float>(), nx, ny, stc_cols, d_safrag.as<float>(),
                                          d_sbx.as<float>());
      MF_LAUNCH_CK();
    }
    MF_CK(cudaDeviceSynchronize());  // d_etile goes out of scope
    const int chunks = cdiv(B, kStcProb);
    d_sscratch.alloc(sizeof(float) * (size_t)std::max(nscr, 1) * chunks * 2048);
    d_stickets.alloc(sizeof(unsigned int) * (size_t)nt * chunks);
    MF_CK(cudaMemset(d_stickets.p, 0, d_stickets.bytes));
  }

  // Tensor-core interpolation tiles: every point binned by its first tap
  // (mx - 11, my - 11) into an 8 x 8 tile of the virtual grid; a tile's
  // points in (mx, my, index) order, cut into CTAs of at most kItcPts.
  void build_itc_tiles(const std::vector<int>& mx, const std::vector<int>& my) {
    auto fdiv = [](int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };
    std::vector<int> ord(mtot);
    for (int k = 0; k < mtot; ++k) ord[k] = k;
    auto key = [&](int k) {
      return std::make_tuple(fdiv(mx[k] - (kMSP - 1), kItcTile), fdiv(my[k] - (kMSP - 1), kItcTile), mx[k], my[k]);
    };
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return key(a) < key(b); });
    std::vector<ItcTile> tiles;
    for (int i = 0; i < mtot;) {
      const int tr = fdiv(mx[ord[i]] - (kMSP - 1), kItcTile), tcol = fdiv(my[ord[i]] - (kMSP - 1), kItcTile);
      int j = i;
      while (j < mtot && fdiv(mx[ord[j]] - (kMSP - 1), kItcTile) == tr &&
             fdiv(my[ord[j]] - (kMSP - 1), kItcTile) == tcol)
        ++j;
      for (int a = i; a < j; a += kItcPts) tiles.push_back(ItcTile{tr * kItcTile, tcol * kItcTile, a, std::min(kItcPts, j - a)});
      i = j;
    }
    // launch order: fullest CTAs first, so that the last wave holds short ones
    std::stable_sort(tiles.begin(), tiles.end(), [](const ItcTile& a, const ItcTile& b) { return a.count > b.count; });
    ntc = (int)tiles.size();
    chi_pad = std::max(chi_pad, ntc);
    std::vector<int> packed(std::max(mtot, 1), 0);
    for (const ItcTile& tl : tiles)
      for (int a = tl.start; a < tl.start + tl.count; ++a) {
        const int k = ord[a];
        packed[a] = k | ((mx[k] - (kMSP - 1) - tl.row0) << 24) | ((my[k] - (kMSP - 1) - tl.col0) << 27);
      }
    d_itc.upload(tiles.data(), std::max<size_t>(tiles.size(), 1));
    d_iperm.upload(packed.data(), packed.size());
    set_smem(k_nufft_interp_tc, kItcSmem);
  }
  int interp_chunks() const { return cdiv(B, SharedChunk<T>::kInterp); }
  static constexpr int kMaxInterpPpw = 32;
  static size_t spread_smem() { return sizeof(cplx<T>) * SharedChunk<T>::kSpread * 256; }
  int spread_chunks() const { return cdiv(B, SharedChunk<T>::kSpread); }

  // FFT passes inside the device loop: with few problems active the CTAs
  // spread over them with fewer rows / columns each (fft_work, from the
  // step's gate list); the fixed mapping elsewhere, or with MFISTA_FFT_DYN=0.
  // A batch of at most kDynFew problems gets the grid of the small shape.
  bool fft_dyn = true;
  DynUnits dyn(int gate, int units) const {
    const int sl = gate_list_slot(gate);
    if (!fft_dyn || !c.act_lists || sl < 0 || units <= 2) return DynUnits{nullptr, 0};
    return DynUnits{c.act_lists + (size_t)sl * (B + 1), 2};
  }
  int fft_grid(const DynUnits& d, int n, int units) const {
    return cdiv(n, (d.list && B <= kDynFew) ? d.small : units);
  }

  // the geometry with this launch's gate lists (set inside the device loop)
  NufftGeom<T> geo_now() const {
    NufftGeom<T> g = geo;
    g.act_lists = c.act_lists;
    return g;
  }

  void launch_interp(cudaStream_t s, cplx<T>* g, int gate, int qchi, cplx<T>* y2, const double2* base = nullptr,
                     double2* out = nullptr) {
    const NufftGeom<T> geo = geo_now();
    // FP32: grouped kernel; FP64 (register-bound with 2G double sums): one
    // problem at a time.  Both chunk the batch's active problems.
    if (shared) {
      if constexpr (sizeof(T) == 4) {
        if (interp_tc)
          k_nufft_interp_tc<<<dim3(ntc, cdiv(B, kItcProb)), 256, kItcSmem, s>>>(
              geo, d_itc.as<ItcTile>(), ntc, d_iperm.as<int>(), g, gstride, nx, ny, inv_mm, c.st, gate, c.part, qchi,
              chi_slots(), y2, B, base, out);
        else if (interp_fly)
          k_nufft_interp_group_fly<T><<<dim3(interp_blocks(), interp_chunks()), 256, 0, s>>>(
              geo, g, gstride, nx, ny, inv_mm, c.st, gate, c.part, qchi, y2, B, base, out, ippw);
        else
          k_nufft_interp_group<T><<<dim3(interp_blocks(), interp_chunks()), 256, 0, s>>>(
              geo, g, gstride, nx, ny, inv_mm, c.st, gate, c.part, qchi, y2, B, base, out, ippw);
      }
      else
        k_nufft_interp_shared<T, true><<<dim3(interp_blocks(), interp_chunks()), 256, 0, s>>>(
            geo, g, gstride, nx, ny, inv_mm, c.st, gate, c.part, qchi, y2, B, base, out, ippw);
    } else
      k_nufft_interp<T><<<dim3(interp_blocks(), B), 256, 0, s>>>(geo, g, gstride, nx, ny, inv_mm, c.st, gate,
                                                                 c.part, qchi, y2, base, out);
    MF_LAUNCH_CK();
  }

  void launch_rows_fwd(cudaStream_t s, const double* src, int gate, const double* sub) {
    const DynUnits d = dyn(gate, rpc);
    k_nufft_rows_fwd<T><<<dim3(fft_grid(d, nx, rpc), B), 256, smem_rows, s>>>(
        src, c.xstride, geo.e4, d_grid.as<cplx<T>>(), gstride, nx, ny, fh.dev, tw2h.as<cplx<T>>(), c.st, gate, rpc,
        sub, d);
    MF_LAUNCH_CK();
  }

  bool corrected() const override { return exact != nullptr; }
  int launches_refresh() const override { return exact ? (model ? 4 : 3) : 0; }

  // exact FP64 model of the anchors: A x_a -> d_axa (owner's layout); the
  // anchor is the current x, so its exact model also becomes the kept model
  // of x (and of z at the start of a solve, where z = x)
  void refresh_anchor(cudaStream_t s, int gate) override {
    if (!exact) return;
    exact->launch_rows_fwd(s, c.xa, gate, nullptr);
    exact->launch_cols_fwd(s, gate);
    exact->launch_interp(s, exact->d_grid.template as<cplx<double>>(), gate, -1, nullptr, nullptr,
                         d_axa.as<double2>());
    if (model) {
      k_nufft_model_set<<<dim3(std::max(1, cdiv(mmax, 256)), B), 256, 0, s>>>(
          geo.pt_lo, geo.pt_hi, geo.y2_bstride, d_axa.as<double2>(), d_ax.as<double2>(),
          gate == kGateInit ? d_az.as<double2>() : nullptr, c.st, gate);
      MF_LAUNCH_CK();
    }
  }

  bool models_z() const override { return model; }

  void forward_z(cudaStream_t s, int gate, int qchi) override {
    const int gx = shared ? cdiv(chi_slots(), 8) : chi_slots();
    k_nufft_resid_model<T><<<dim3(gx, B), 256, 0, s>>>(geo, d_az.as<double2>(), d_y2.as<cplx<T>>(), shared ? 1 : 0,
                                                        ippw, chi_slots(), c.st, gate, c.part, qchi);
    MF_LAUNCH_CK();
  }

  ModelMom model_momentum(int img_blocks) override {
    ModelMom m = Op::model_momentum(img_blocks);
    if (!model) return m;
    m.pt_lo = geo.pt_lo;
    m.pt_hi = geo.pt_hi;
    m.bstride = geo.y2_bstride;
    m.ax = d_ax.as<double2>();
    m.axn = d_axn.as<double2>();
    m.az = d_az.as<double2>();
    return m;
  }
  int model_blocks() const override { return model ? std::max(1, cdiv(mmax, 256)) : 0; }

  void forward_exact(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    if (exact) exact->forward(s, src, gate, qchi, store);
    else forward(s, src, gate, qchi, store);
  }

  void launch_cols_fwd(cudaStream_t s, int gate) {
    const DynUnits d = dyn(gate, cpc);
    k_nufft_cols<T><<<dim3(fft_grid(d, ny + 1, cpc), B), 256, smem_cols, s>>>(
        d_grid.as<cplx<T>>(), gstride, nx, ny, fcol.dev, -1, cpc, 1, 0, c.st, gate, d);
    MF_LAUNCH_CK();
  }

  void launch_spread(cudaStream_t s, cplx<T>* g, int gate) {
    const NufftGeom<T> geo = geo_now();
    if constexpr (sizeof(T) == 4) {
      if (spread_tc) {
        k_nufft_spread_tc<<<dim3(nsitems, cdiv(B, kStcProb)), 256, 0, s>>>(
            geo, d_sitems.as<StcItem>(), d_svlist.as<int>(), d_safrag.as<float4>(), d_sbx.as<float>(),
            d_y2.as<cplx<float>>(), g, gstride, nx, ny, stc_cols, c.st, gate, B, d_sscratch.as<float>(),
            d_stickets.as<unsigned int>());
        MF_LAUNCH_CK();
        return;
      }
    }
    if (shared) {
      // cluster of spread_cs CTAs per tile, each a segment of its points
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(ntiles * spread_cs, spread_chunks(), 1);
      cfg.blockDim = dim3(256, 1, 1);
      cfg.dynamicSmemBytes = spread_smem();
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = spread_cs;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      MF_CK(cudaLaunchKernelEx(&cfg, k_nufft_spread_shared<T>, geo, (const cplx<T>*)d_y2.as<cplx<T>>(), g, gstride,
                               nx, ny, ntiles, (const ProbState*)c.st, gate, B));
      return;
    }
    else
      k_nufft_spread<T><<<dim3(ntiles, B), tile_r * tile_c, 0, s>>>(geo, d_y2.as<cplx<T>>(), g, gstride, nx, ny,
                                                                    tile_r, tile_c, ntiles, c.st, gate);
    MF_LAUNCH_CK();
  }

  void forward(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    cplx<T>* g = d_grid.as<cplx<T>>();
    // with defect correction: A v = A x_a (FP64) + A32 (v - x_a)
    launch_rows_fwd(s, src, gate, exact ? c.xa : nullptr);
    launch_cols_fwd(s, gate);
    // the trial point's model is kept for the next momentum point
    launch_interp(s, g, gate, qchi, store ? d_y2.as<cplx<T>>() : nullptr, exact ? d_axa.as<double2>() : nullptr,
                  model && !store ? d_axn.as<double2>() : nullptr);
  }

  void adjoint(cudaStream_t s, const double* z_tsv, int qtsv) override {
    cplx<T>* g = d_grid.as<cplx<T>>();
    launch_spread(s, g, kGateGrad);
    const DynUnits dc = dyn(kGateGrad, cpc);
    k_nufft_cols<T><<<dim3(fft_grid(dc, ny + 1, cpc), B), 256, smem_cols, s>>>(g, gstride, nx, ny, fcol.dev, +1, cpc,
                                                                               0, 1, c.st, kGateGrad, dc);
    MF_LAUNCH_CK();
    TsvFuse tf{z_tsv, c.prm, c.tsvNX, c.tsvNY};
    const DynUnits dr = qtsv < 0 ? dyn(kGateGrad, rpc) : DynUnits{nullptr, 0};
    k_nufft_rows_inv<T><<<dim3(fft_grid(dr, nx, rpc), B), 256, smem_rows, s>>>(
        g, gstride, c.dfdx, c.xstride, geo.e4, nx, ny, inv_mm, fh.dev, tw2h.as<cplx<T>>(), tf, c.part, qtsv, c.st,
        kGateGrad, rpc, dr);
    MF_LAUNCH_CK();
  }

  int chi_slots() const override { return interp_blocks(); }
  int max_chi_slots() const override { return std::max({1, cdiv(mmax, 8), chi_pad}); }
  int tsv_slots() const override { return nx; }  // row-pass CTAs at rows_per_cta = 1

  LaunchShapes shapes() const override {
    LaunchShapes sh;
    sh.interp_ppw = shared ? ippw : 0;
    sh.spread_cluster = shared ? spread_cs : 0;
    sh.rows_per_cta = rpc;
    sh.cols_per_cta = cpc;
    return sh;
  }

  void set_shapes(const LaunchShapes& sh) override {
    auto rows_smem = [&](int r) { return (size_t)2 * r * (ny + 1) * sizeof(cplx<T>); };
    auto cols_smem = [&](int cc) { return (size_t)2 * cc * (2 * nx + 1) * sizeof(cplx<T>); };
    if (shared && sh.interp_ppw && (sh.interp_ppw < 1 || sh.interp_ppw > kMaxInterpPpw))
      throw Error(MFISTA_ERR_ARG, "interp_ppw must be 1..32");
    if (shared && sh.spread_cluster && (sh.spread_cluster < 1 || sh.spread_cluster > 16))
      throw Error(MFISTA_ERR_ARG, "spread_cluster must be 1..16");
    if (sh.rows_per_cta && (sh.rows_per_cta < 1 || sh.rows_per_cta > nx || rows_smem(sh.rows_per_cta) > 227 * 1024))
      throw Error(MFISTA_ERR_ARG, "rows_per_cta out of range");
    if (sh.cols_per_cta &&
        (sh.cols_per_cta < 1 || sh.cols_per_cta > ny + 1 || cols_smem(sh.cols_per_cta) > 227 * 1024))
      throw Error(MFISTA_ERR_ARG, "cols_per_cta out of range");
    if (shared && sh.interp_ppw) {
      ippw = sh.interp_ppw;
      if (exact) exact->ippw = ippw;  // same chi^2 partial slots for forward_exact
    }
    if (shared && sh.spread_cluster) spread_cs = sh.spread_cluster;
    if (sh.rows_per_cta) {
      rpc = sh.rows_per_cta;
      smem_rows = rows_smem(rpc);
      set_smem(k_nufft_rows_fwd<T>, smem_rows);
      set_smem(k_nufft_rows_inv<T>, smem_rows);
    }
    if (sh.cols_per_cta) {
      cpc = sh.cols_per_cta;
      smem_cols = cols_smem(cpc);
      set_smem(k_nufft_cols<T>, smem_cols);
    }
  }
  double fscale() const override { return 0.5; }
  int launches_forward() const override { return 3; }
  int launches_adjoint() const override { return 3; }

  double launch_single(cudaStream_t s, int kernel) override {
    cplx<T>* g = d_grid.as<cplx<T>>();
    const double cs = sizeof(cplx<T>), ts = sizeof(T);
    const double G = (double)gstride, N = (double)nx * ny, half_rows = (double)nx * (ny + 1);
    const double pts_geo = (double)mtot;                          // point arrays read once
    const double pts_res = shared ? (double)B * mtot : (double)mtot;  // per-problem residuals
    switch (kernel) {
      case 0:
        launch_interp(s, g, kGateTrial, kQChiX, d_y2.as<cplx<T>>());
        return B * G * cs + pts_geo * (8 + 2 * kTaps * ts + 24) + pts_res * cs;
      case 1:
        launch_spread(s, g, kGateGrad);
        return pts_geo * (8 + 2 * kTaps * ts) + pts_res * cs + B * G * cs;
      case 2:
        launch_rows_fwd(s, c.z, kGateTrial, nullptr);
        return B * N * 8 + N * 8 + B * half_rows * cs;
      case 3:
        k_nufft_cols<T><<<dim3(cdiv(ny + 1, cpc), B), 256, smem_cols, s>>>(g, gstride, nx, ny, fcol.dev, -1, cpc, 1, 0,
                                                                           c.st, kGateTrial, DynUnits{nullptr, 0});
        MF_LAUNCH_CK();
        return B * (half_rows + G) * cs;
      case 4:
        k_nufft_cols<T><<<dim3(cdiv(ny + 1, cpc), B), 256, smem_cols, s>>>(g, gstride, nx, ny, fcol.dev, +1, cpc, 0, 1,
                                                                           c.st, kGateGrad, DynUnits{nullptr, 0});
        MF_LAUNCH_CK();
        return B * (G + half_rows) * cs;
      case 5: {
        TsvFuse tf{c.z, c.prm, c.tsvNX, c.tsvNY};
        k_nufft_rows_inv<T><<<dim3(cdiv(nx, rpc), B), 256, smem_rows, s>>>(
            g, gstride, c.dfdx, c.xstride, geo.e4, nx, ny, inv_mm, fh.dev, tw2h.as<cplx<T>>(), tf, c.part, kQTsvZ,
            c.st, kGateGrad, rpc, DynUnits{nullptr, 0});
        MF_LAUNCH_CK();
        return B * (half_rows * cs + 2 * N * 8) + N * 8;
      }
      default:
        return -1;
    }
  }
};

// ---------------------------------------------------------------------------
// gridded FFT operator
// ---------------------------------------------------------------------------
struct FftVarInput {
  const int *u_idx, *v_idx;
  const double *y_r, *y_i, *noise;
  int M, NX, NY;
};

template <typename T> struct FftVarOp : Op {
  Ctx& c;
  int NX, NY, NYh, B;
  DevMem d_mask, d_yf, d_H, tw2h;
  FftHost<T> fh, fnx;
  FftVarGeom geo{};
  int rpc = 8, cpc = 8;
  size_t smem_rows = 0, smem_cols = 0;
  long hstride = 0;
  double sqrtn = 0;
  // corrected FP32 form: the FP64 operator computes the exact spectrum of
  // the anchors x_a (d_axa, [B][NX*NYh]); the FP32 transforms then see only
  // the departure v - x_a
  std::unique_ptr<FftVarOp<double>> exact;
  DevMem d_axa;

  FftVarOp(Ctx& ctx, const FftVarInput& in, bool correct = false) : c(ctx) {
    NX = in.NX;
    NY = in.NY;
    B = ctx.B;
    if (NY % 2 != 0 || NX < 2 || NY < 2) throw Error(MFISTA_ERR_ARG, "FFT variant needs an even NY >= 2");
    NYh = NY / 2 + 1;
    // idx2mat (:70-88) then full2half / fft_full2half (:50-68)
    std::vector<double> mk_full((size_t)NX * NY, 0.0);
    std::vector<double2> yf_full((size_t)NX * NY, make_double2(0.0, 0.0));
    for (int i = 0; i < in.M; ++i) {
      int u = in.u_idx[i], v = in.v_idx[i];
      if (u < 0 || u >= NX || v < 0 || v >= NY) throw Error(MFISTA_ERR_ARG, "u_idx/v_idx outside the grid");
      size_t e = (size_t)NY * u + v;
      mk_full[e] = 1 / in.noise[i];
      yf_full[e] = make_double2(in.y_r[i] / in.noise[i], in.y_i[i] / in.noise[i]);
    }
    std::vector<double> mh((size_t)NX * NYh);
    std::vector<double2> yh((size_t)NX * NYh);
    for (int i = 0; i < NX; ++i)
      for (int j = 0; j < NYh; ++j) {
        mh[(size_t)NYh * i + j] = mk_full[(size_t)NY * i + j];
        yh[(size_t)NYh * i + j] = yf_full[(size_t)NY * i + j];
      }
    d_mask.upload(mh.data(), mh.size());
    d_yf.upload(yh.data(), yh.size());
    geo.mask_h = d_mask.as<double>();
    geo.yf_h = d_yf.as<double2>();
    geo.geo_stride = 0;
    fh.init(NY / 2);
    fnx.init(NX);
    make_twiddles<T>(NY, tw2h);
    hstride = (long)NX * NYh;
    d_H.alloc(sizeof(cplx<T>) * (size_t)B * hstride);
    sqrtn = sqrt((double)(NX * NY));
    // launch shapes: the FP64 operator's (the larger buffers) bound both, so
    // that the exact and the FP32 passes write the same partial-sum slots
    auto fits = [&](int r, int len) { return (size_t)2 * r * (len + 1) * sizeof(cplx<double>) <= 96 * 1024; };
    while (rpc > 1 && !fits(rpc, NY / 2)) rpc /= 2;
    while (cpc > 1 && !fits(cpc, NX)) cpc /= 2;
    set_rpc_cpc(rpc, cpc);
    if (correct && sizeof(T) == 4) {
      exact.reset(new FftVarOp<double>(ctx, in, false));
      exact->set_rpc_cpc(rpc, cpc);
      d_axa.alloc(sizeof(double2) * (size_t)B * hstride);
      MF_CK(cudaMemset(d_axa.p, 0, d_axa.bytes));
    }
  }

  void set_rpc_cpc(int r, int cc) {
    rpc = r;
    cpc = cc;
    smem_rows = (size_t)2 * rpc * (NY / 2 + 1) * sizeof(cplx<T>);
    smem_cols = (size_t)2 * cpc * (NX + 1) * sizeof(cplx<T>);
    set_smem(k_fftv_rows_fwd<T>, smem_rows);
    set_smem(k_fftv_rows_inv<T>, smem_rows);
    set_smem(k_fftv_cols<T>, smem_cols);
  }

  void launch_rows_fwd(cudaStream_t s, const double* src, int gate, const double* sub) {
    k_fftv_rows_fwd<T><<<dim3(cdiv(NX, rpc), B), 256, smem_rows, s>>>(src, c.xstride, d_H.as<cplx<T>>(), hstride, NX,
                                                                      NY, fh.dev, tw2h.as<cplx<T>>(), c.st, gate, rpc,
                                                                      sub);
    MF_LAUNCH_CK();
  }

  void launch_cols_fwd(cudaStream_t s, int gate, int qchi, bool store, const double2* base, double2* raw_out) {
    k_fftv_cols<T><<<dim3(cdiv(NYh, cpc), B), 256, smem_cols, s>>>(d_H.as<cplx<T>>(), hstride, NX, NYh, fnx.dev, -1,
                                                                   cpc, geo, sqrtn, c.st, gate, c.part, qchi,
                                                                   store ? 1 : 0, base, raw_out);
    MF_LAUNCH_CK();
  }

  void forward(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    // with defect correction: F(v) = F(x_a) (FP64) + F32(v - x_a)
    launch_rows_fwd(s, src, gate, exact ? c.xa : nullptr);
    launch_cols_fwd(s, gate, qchi, store, exact ? d_axa.as<double2>() : nullptr, nullptr);
  }

  bool corrected() const override { return exact != nullptr; }
  int launches_refresh() const override { return exact ? 2 : 0; }

  void refresh_anchor(cudaStream_t s, int gate) override {
    if (!exact) return;
    exact->launch_rows_fwd(s, c.xa, gate, nullptr);
    exact->launch_cols_fwd(s, gate, -1, false, nullptr, d_axa.as<double2>());
  }

  void forward_exact(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    if (exact) exact->forward(s, src, gate, qchi, store);
    else forward(s, src, gate, qchi, store);
  }

  void adjoint(cudaStream_t s, const double* z_tsv, int qtsv) override {
    cplx<T>* H = d_H.as<cplx<T>>();
    k_fftv_cols<T><<<dim3(cdiv(NYh, cpc), B), 256, smem_cols, s>>>(H, hstride, NX, NYh, fnx.dev, +1, cpc, geo, sqrtn,
                                                                   c.st, kGateGrad, c.part, -1, 0, nullptr, nullptr);
    MF_LAUNCH_CK();
    k_fftv_rows_inv<T><<<dim3(cdiv(NX, rpc), B), 256, smem_rows, s>>>(
        H, hstride, c.dfdx, c.xstride, NX, NY, fh.dev, tw2h.as<cplx<T>>(), z_tsv, c.prm, c.tsvNX, c.tsvNY, c.part,
        qtsv, c.st, kGateGrad, rpc);
    MF_LAUNCH_CK();
  }

  int chi_slots() const override { return cdiv(NYh, cpc); }
  int tsv_slots() const override { return cdiv(NX, rpc); }
  double fscale() const override { return 0.25; }
  int launches_forward() const override { return 2; }
  int launches_adjoint() const override { return 2; }
};

// ---------------------------------------------------------------------------
// dense DFT operator (FP64)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// tensor-core split-BF16 GEMM launcher (tc::k_gemm_bf16x3)
// ---------------------------------------------------------------------------
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  if (!fn) throw Error(MFISTA_ERR_CUDA, "the driver does not provide cuTensorMapEncodeTiled");
  return fn;
}

// TMA map of a K-major BF16 plane [rows][kpad]: boxes of kTK x box_rows
// elements with the 128-byte swizzle the MMA descriptors expect
inline CUtensorMap bf16_tile_map(const void* base, int rows, int kpad, int box_rows) {
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (kpad % tc::kTK) || (rows % box_rows))
    throw Error(MFISTA_ERR_ARG, "tensor-core operand not tiled");
  CUtensorMap m;
  cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kpad * 2};
  cuuint32_t box[2] = {(cuuint32_t)tc::kTK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(MFISTA_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

// P[s][b][r] = sum_{k in split s} Amat[r][k] X[b][k] over K-major BF16 planes
// (np = 2 or 3 planes per operand)
struct TcGemm {
  int np = 2, rows = 0, kpad = 0, bpad = 0, nsplit = 1, kblocks = 0, kblocks_all = 0;
  tc::TcMaps maps{};
  DevMem part;  // [nsplit][bpad][rows] FP32
  int* err = nullptr;

  int smem_bytes() const { return np == 3 ? tc::Ring<3>::kSmemBytes : tc::Ring<2>::kSmemBytes; }

  // split K so that the tiles cover the GPU's SMs about once (one CTA per SM)
  void init(int np_, void* const* a_planes, int rows_, int kpad_, void* const* x_planes, int bpad_, int* err_) {
    np = np_;
    rows = rows_;
    kpad = kpad_;
    bpad = bpad_;
    err = err_;
    kblocks_all = kpad / tc::kTK;
    int dev = 0, sms = 148;
    MF_CK(cudaGetDevice(&dev));
    MF_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int tiles = (rows / tc::kTM) * (bpad / tc::kTN);
    nsplit = std::max(1, std::min(kblocks_all, sms / std::max(tiles, 1)));
    kblocks = cdiv(kblocks_all, nsplit);
    nsplit = cdiv(kblocks_all, kblocks);  // no empty split
    for (int p = 0; p < np; ++p) {
      maps.a[p] = bf16_tile_map(a_planes[p], rows, kpad, tc::kTM);
      maps.x[p] = bf16_tile_map(x_planes[p], bpad, kpad, tc::kTN);
    }
    part.alloc(sizeof(float) * (size_t)nsplit * bpad * rows);
    MF_CK(cudaMemset(part.p, 0, part.bytes));
    if (np == 3) set_smem(tc::k_gemm_split_bf16<3>, tc::Ring<3>::kSmemBytes);
    else set_smem(tc::k_gemm_split_bf16<2>, tc::Ring<2>::kSmemBytes);
  }

  void launch(cudaStream_t s, const ProbState* st, int gate, int B) {
    tc::TcArgs a{part.as<float>(), rows, bpad, kblocks, kblocks_all, err};
    dim3 grid(rows / tc::kTM, nsplit, bpad / tc::kTN);
    if (np == 3) tc::k_gemm_split_bf16<3><<<grid, 128, tc::Ring<3>::kSmemBytes, s>>>(maps, a, st, gate, B);
    else tc::k_gemm_split_bf16<2><<<grid, 128, tc::Ring<2>::kSmemBytes, s>>>(maps, a, st, gate, B);
    MF_LAUNCH_CK();
  }

  // algorithmic bytes of one launch: the A planes, the X planes, the partials
  double bytes() const {
    return 2.0 * np * rows * kpad + 2.0 * np * bpad * kpad + 4.0 * nsplit * bpad * rows;
  }
};

// ---------------------------------------------------------------------------
// DFT operator: FP64 (GEMV for one problem, register-blocked GEMM for a
// batch), or the split-BF16 tensor-core GEMMs with FP64 defect correction
// ---------------------------------------------------------------------------
struct DftOp : Op {
  Ctx& c;
  DftGeom g{};
  DevMem d_A, d_y, d_part, d_resid, d_atr;
  int B;
  bool gemm = false;     // batched problems: GEMMs instead of per-problem GEMVs
  int mchunk = 0, nmchunk = 0;
  // split-BF16 form (np planes per operand)
  bool tcm = false;
  int np = 2;
  int mrow = 0, nk = 0, nrow = 0, mk = 0, bpad = 0;
  DevMem rm[3], cm[3], xv[3], xr[3], d_axa, d_ra, d_ga, d_err;
  TcGemm fwd, adj;

  DftOp(Ctx& ctx, const double* A, const double* y, int M, int N, int precision = MFISTA_FP64) : c(ctx) {
    B = ctx.B;
    tcm = precision == MFISTA_BF16X3 || precision == MFISTA_BF16X6;
    np = precision == MFISTA_BF16X6 ? 3 : 2;
    if (!tcm && precision != MFISTA_FP64)
      throw Error(MFISTA_ERR_ARG, "the DFT operator runs in FP64, BF16X3 or BF16X6");
    d_A.upload(A, (size_t)M * N);
    d_y.upload(y, M);
    g.A = d_A.as<double>();
    g.y = d_y.as<double>();
    g.M = M;
    g.N = N;
    g.chunk = 64;
    g.nchunk = cdiv(N, g.chunk);
    gemm = B > 1 || tcm;  // the anchors of the split-BF16 form use the FP64 GEMMs
    if (gemm) {  // split-K so that the tiles fill the GPU
      g.chunk = std::max(kGK, cdiv(cdiv(N, 4), kGK) * kGK);
      g.nchunk = cdiv(N, g.chunk);
      mchunk = std::max(kGK, cdiv(cdiv(M, 8), kGK) * kGK);
      nmchunk = cdiv(M, mchunk);
      d_atr.alloc(sizeof(double) * (size_t)B * nmchunk * std::max(N, 1));
    }
    d_part.alloc(sizeof(double) * (size_t)B * g.nchunk * std::max(M, 1));
    d_resid.alloc(sizeof(double) * (size_t)B * std::max(M, 1));
    g.az_part = d_part.as<double>();
    g.resid = d_resid.as<double>();
    if (tcm) setup_tc(M, N);
    // the uploads above ran on the legacy stream; the solver's streams do
    // not wait for it
    MF_CK(cudaDeviceSynchronize());
  }

  static tc::Planes planes(DevMem* d, int np) {
    tc::Planes q{};
    for (int p = 0; p < np; ++p) q.p[p] = d[p].as<__nv_bfloat16>();
    return q;
  }

  void setup_tc(int M, int N) {
    mrow = cdiv(M, tc::kTM) * tc::kTM;
    nk = cdiv(N, tc::kTK) * tc::kTK;
    nrow = cdiv(N, tc::kTM) * tc::kTM;
    mk = cdiv(M, tc::kTK) * tc::kTK;
    bpad = cdiv(B, tc::kTN) * tc::kTN;
    const size_t h = 2;  // bytes per BF16
    for (int p = 0; p < np; ++p) {
      rm[p].alloc(h * mrow * nk);
      cm[p].alloc(h * nrow * mk);
      xv[p].alloc(h * bpad * nk);
      xr[p].alloc(h * bpad * mk);
      MF_CK(cudaMemset(xv[p].p, 0, xv[p].bytes));
      MF_CK(cudaMemset(xr[p].p, 0, xr[p].bytes));
    }
    dim3 grid(cdiv(std::max(mrow, mk), 32), cdiv(std::max(nrow, nk), 32));
    if (np == 3)
      tc::k_split_matrix<3><<<grid, 256>>>(g.A, M, N, mrow, nk, nrow, mk, planes(rm, 3), planes(cm, 3));
    else
      tc::k_split_matrix<2><<<grid, 256>>>(g.A, M, N, mrow, nk, nrow, mk, planes(rm, 2), planes(cm, 2));
    MF_LAUNCH_CK();
    d_axa.alloc(sizeof(double) * (size_t)B * M);
    d_ra.alloc(sizeof(double) * (size_t)B * M);
    d_ga.alloc(sizeof(double) * (size_t)B * N);
    for (DevMem* d : {&d_axa, &d_ra, &d_ga}) MF_CK(cudaMemset(d->p, 0, d->bytes));
    d_err.alloc(sizeof(int));
    MF_CK(cudaMemset(d_err.p, 0, sizeof(int)));
    void *a_rm[3], *a_cm[3], *x_v[3], *x_r[3];
    for (int p = 0; p < np; ++p) {
      a_rm[p] = rm[p].p;
      a_cm[p] = cm[p].p;
      x_v[p] = xv[p].p;
      x_r[p] = xr[p].p;
    }
    fwd.init(np, a_rm, mrow, nk, x_v, bpad, d_err.as<int>());
    adj.init(np, a_cm, nrow, mk, x_r, bpad, d_err.as<int>());
    MF_CK(cudaDeviceSynchronize());
  }

  void split_vectors(cudaStream_t s, const double* src, long sstride, const double* sub, int K, int kpad,
                     DevMem* out, int gate) {
    dim3 grid(cdiv(kpad, 256), bpad);
    if (np == 3)
      tc::k_split_vectors<3><<<grid, 256, 0, s>>>(src, sstride, sub, sstride, K, kpad, B, c.st, gate, planes(out, 3));
    else
      tc::k_split_vectors<2><<<grid, 256, 0, s>>>(src, sstride, sub, sstride, K, kpad, B, c.st, gate, planes(out, 2));
    MF_LAUNCH_CK();
  }

  // FP64 A z -> residual (and chi^2 partials)
  void forward_fp64(cudaStream_t s, const double* src, int gate, int qchi, bool store) {
    if (gemm)
      k_dft_az_gemm<<<dim3(cdiv(g.M, kGT), g.nchunk, cdiv(B, kGT)), 256, 0, s>>>(g, src, c.xstride, c.st, gate, B);
    else
      k_dft_az<<<dim3(std::max(1, cdiv(g.M, 256)), g.nchunk, B), 256, g.chunk * sizeof(double), s>>>(
          g, src, c.xstride, c.st, gate);
    MF_LAUNCH_CK();
    k_dft_resid<<<dim3(std::max(1, cdiv(g.M, 256)), B), 256, 0, s>>>(g, c.st, gate, c.part, qchi, store ? 1 : 0);
    MF_LAUNCH_CK();
  }

  void forward(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    if (!tcm) {
      forward_fp64(s, src, gate, qchi, store);
      return;
    }
    split_vectors(s, src, c.xstride, c.xa, g.N, nk, xv, gate);
    fwd.launch(s, c.st, gate, B);
    k_dft_tc_resid<<<dim3(std::max(1, cdiv(g.M, 256)), B), 256, 0, s>>>(fwd.part.as<float>(), fwd.nsplit, bpad, mrow,
                                                                        d_axa.as<double>(), g, c.st, gate, c.part,
                                                                        qchi, store ? 1 : 0);
    MF_LAUNCH_CK();
  }

  void adjoint(cudaStream_t s, const double* z_tsv, int qtsv) override {
    if (tcm) {
      split_vectors(s, g.resid, g.M, d_ra.as<double>(), g.M, mk, xr, kGateGrad);
      adj.launch(s, c.st, kGateGrad, B);
      k_dft_tc_atr_finish<<<dim3(cdiv(g.N, 256), B), 256, 0, s>>>(adj.part.as<float>(), adj.nsplit, bpad, nrow,
                                                                   d_ga.as<double>(), g.N, c.dfdx, c.xstride, z_tsv,
                                                                   c.prm, c.tsvNX, c.tsvNY, c.st, kGateGrad);
      MF_LAUNCH_CK();
      return;
    }
    if (gemm) {
      k_dft_atr_gemm<<<dim3(cdiv(g.N, kGT), nmchunk, cdiv(B, kGT)), 256, 0, s>>>(g, d_atr.as<double>(), mchunk,
                                                                                 nmchunk, c.st, kGateGrad, B);
      MF_LAUNCH_CK();
      k_dft_atr_finish<<<dim3(cdiv(g.N, 256), B), 256, 0, s>>>(g, d_atr.as<double>(), nmchunk, c.dfdx, c.xstride,
                                                               z_tsv, c.prm, c.tsvNX, c.tsvNY, c.st, kGateGrad);
      MF_LAUNCH_CK();
      return;
    }
    k_dft_atr<<<dim3(cdiv(g.N, 8), B), 256, 0, s>>>(g, c.dfdx, c.xstride, z_tsv, c.prm, c.tsvNX, c.tsvNY, c.st,
                                                     kGateGrad, c.part, qtsv);
    MF_LAUNCH_CK();
  }

  // FP64 A^T r over a residual buffer (FP64 GEMM; no TSV term)
  void atr_fp64(cudaStream_t s, const double* resid, double* out, long ostride, int gate) {
    DftGeom gg = g;
    gg.resid = const_cast<double*>(resid);
    k_dft_atr_gemm<<<dim3(cdiv(g.N, kGT), nmchunk, cdiv(B, kGT)), 256, 0, s>>>(gg, d_atr.as<double>(), mchunk,
                                                                               nmchunk, c.st, gate, B);
    MF_LAUNCH_CK();
    k_dft_atr_finish<<<dim3(cdiv(g.N, 256), B), 256, 0, s>>>(gg, d_atr.as<double>(), nmchunk, out, ostride, nullptr,
                                                             c.prm, c.tsvNX, c.tsvNY, c.st, gate);
    MF_LAUNCH_CK();
  }

  bool corrected() const override { return tcm; }
  int launches_refresh() const override { return tcm ? 4 : 0; }
  // the two-plane products (~2^-16) need a closer anchor than the
  // three-plane ones to reach 1e-6 of the FP64 objective
  int refresh_period() const override { return np == 2 ? 8 : 32; }

  // FP64 anchor terms: ax_a = A x_a, r_a = y - ax_a, g_a = A^T r_a
  void refresh_anchor(cudaStream_t s, int gate) override {
    if (!tcm) return;
    k_dft_az_gemm<<<dim3(cdiv(g.M, kGT), g.nchunk, cdiv(B, kGT)), 256, 0, s>>>(g, c.xa, c.xstride, c.st, gate, B);
    MF_LAUNCH_CK();
    k_dft_anchor<<<dim3(std::max(1, cdiv(g.M, 256)), B), 256, 0, s>>>(g, c.st, gate, d_axa.as<double>(),
                                                                      d_ra.as<double>());
    MF_LAUNCH_CK();
    atr_fp64(s, d_ra.as<double>(), d_ga.as<double>(), g.N, gate);
  }

  void forward_exact(cudaStream_t s, const double* src, int gate, int qchi, bool store) override {
    forward_fp64(s, src, gate, qchi, store);
  }

  int device_error() override {
    if (!tcm) return 0;
    int e = 0;
    MF_CK(cudaMemcpy(&e, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    return e;
  }

  // 0: A z GEMM, 1: A^T r GEMM (the split-BF16 ones when in that form)
  double launch_single(cudaStream_t s, int kernel) override {
    if (kernel == 0) {
      if (tcm) {
        fwd.launch(s, c.st, kGateAll, B);
        return fwd.bytes();
      }
      if (!gemm) return -1;
      k_dft_az_gemm<<<dim3(cdiv(g.M, kGT), g.nchunk, cdiv(B, kGT)), 256, 0, s>>>(g, c.z, c.xstride, c.st, kGateAll,
                                                                                 B);
      MF_LAUNCH_CK();
      return 8.0 * g.M * g.N + 8.0 * B * g.N + 8.0 * B * g.nchunk * g.M;
    }
    if (kernel == 1) {
      if (tcm) {
        adj.launch(s, c.st, kGateAll, B);
        return adj.bytes();
      }
      if (!gemm) return -1;
      k_dft_atr_gemm<<<dim3(cdiv(g.N, kGT), nmchunk, cdiv(B, kGT)), 256, 0, s>>>(g, d_atr.as<double>(), mchunk,
                                                                                 nmchunk, c.st, kGateAll, B);
      MF_LAUNCH_CK();
      return 8.0 * g.M * g.N + 8.0 * B * g.M + 8.0 * B * nmchunk * g.N;
    }
    return -1;
  }

  int chi_slots() const override { return std::max(1, cdiv(g.M, 256)); }
  int tsv_slots() const override { return cdiv(g.N, 8); }
  double fscale() const override { return 0.5; }
  int launches_forward() const override { return tcm ? 3 : 2; }
  int launches_adjoint() const override { return tcm ? 3 : (gemm ? 2 : 1); }
};

// ---------------------------------------------------------------------------
// batched MFISTA driver
// ---------------------------------------------------------------------------
struct Solver {
  Ctx ctx;
  std::unique_ptr<Op> op;
  int form = kFormTSV;
  int precision = MFISTA_FP64;
  int fgp_iter = 100;
  int refresh_every = 0;  // defect correction: anchor refresh period (outer iterations)
  int step_cap = 0;
  DevMem d_x, d_z, d_xnew, d_dfdx, d_xa, d_prm, d_st, d_part, d_out, d_box, d_fgp, d_steps, d_ticket, d_lists;
  unsigned long long step_budget = 0;
  ImgDims dm{};
  cudaStream_t stream = nullptr, cap_stream = nullptr, cap_block = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t body_graph = nullptr;  // host-loop fallback
  cudaGraphExec_t body_exec = nullptr;
  bool host_loop = false;
  int* h_any = nullptr;
  int* d_any = nullptr;
  // FGP launch shape
  int fgp_cs = 8, fgp_rpc = 0;
  bool fgp_smem = true;
  size_t fgp_smem_bytes = 0;
  long fgp_scratch_stride = 0;
  int per_step_launches = 0;
  int loop_unroll = 4;  // steps per pass of the device loop (MFISTA_LOOP_UNROLL)
  // the gradient block under an IF node (MFISTA_GRAD_IF=1), or launched
  // every step with its kernels exiting at their per-problem gates (the
  // default: a taken IF node cost about 15 us per step on B200, more than
  // the empty launches of the steps that skip it; measured 1-3 % faster)
  bool grad_if = false;
  int fixed_launches = 0;
  int ref_block_launches = 0, grad_block_launches = 0, rest_launches = 0;
  // movie mode (set_movie before finish_setup): the B problems are the
  // frames of one problem coupled by lam_t sum_b |x_b - x_{b+1}|^2 wt_b
  bool joint = false;
  double lam_t = 0.0;
  DevMem d_wt, d_jq;
  // first-iteration backtracking factor (0: ETA, the C library's loop)
  double eta_first = 0.0;

  void set_movie(const std::vector<double>& wt, double lam) {
    joint = true;
    lam_t = lam;
    std::vector<double> w(wt);
    if (w.empty()) w.push_back(0.0);
    d_wt.upload(w.data(), w.size());
    d_jq.alloc(sizeof(double) * (size_t)ctx.B * kNumQ);
  }
  // every thresholded pixel f is scaled by mask[f] (mask: [N], shared by
  // all problems)
  void set_mask(const double* mask) {
    d_mask.upload(mask, (size_t)ctx.N);
    mask_ptr = d_mask.as<double>();
  }
  // device loop with conditional IF blocks: the refresh and gradient blocks
  // run only in steps where some problem needs them (k_select_blocks)
  bool cond_blocks = false;
  const float* box_ptr = nullptr;
  DevMem d_mask;
  const double* mask_ptr = nullptr;  // pixel scale of the thresholded image (movie c_box), or null

  Solver() {}
  ~Solver() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (body_exec) cudaGraphExecDestroy(body_exec);
    if (body_graph) cudaGraphDestroy(body_graph);
    if (h_any) cudaFreeHost(h_any);
    if (stream) cudaStreamDestroy(stream);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (cap_block) cudaStreamDestroy(cap_block);
  }

  void init_common(int B, int N, int NX, int NY, int form_, int fgp_iter_, const float* box) {
    ctx.B = B;
    ctx.N = N;
    ctx.xstride = N;
    ctx.tsvNX = NX;
    ctx.tsvNY = NY;
    form = form_;
    fgp_iter = fgp_iter_;
    MF_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    MF_CK(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    MF_CK(cudaStreamCreateWithFlags(&cap_block, cudaStreamNonBlocking));
    d_x.alloc(sizeof(double) * (size_t)B * N);
    d_z.alloc(sizeof(double) * (size_t)B * N);
    d_xnew.alloc(sizeof(double) * (size_t)B * N);
    d_dfdx.alloc(sizeof(double) * (size_t)B * N);
    d_prm.alloc(sizeof(ProbParams) * B);
    d_st.alloc(sizeof(ProbState) * B);
    d_out.alloc(sizeof(FinalOut) * B);
    d_steps.alloc(3 * sizeof(unsigned long long));
    d_ticket.alloc(sizeof(unsigned int));
    MF_CK(cudaMemset(d_ticket.p, 0, sizeof(unsigned int)));
    d_lists.alloc(sizeof(int) * (size_t)kGateLists * (B + 1));
    MF_CK(cudaMemset(d_lists.p, 0, d_lists.bytes));
    ctx.x = d_x.as<double>();
    ctx.z = d_z.as<double>();
    ctx.xnew = d_xnew.as<double>();
    ctx.dfdx = d_dfdx.as<double>();
    ctx.prm = d_prm.as<ProbParams>();
    ctx.st = d_st.as<ProbState>();
    d_xa.alloc(sizeof(double) * (size_t)B * N);
    ctx.xa = d_xa.as<double>();
    dm.N = N;
    dm.NX = NX;
    dm.NY = NY;
    dm.xstride = N;
    if (box) {
      d_box.upload(box, N);
      box_ptr = d_box.as<float>();
    }
    MF_CK(cudaHostAlloc((void**)&h_any, sizeof(int), cudaHostAllocMapped));
    MF_CK(cudaHostGetDevicePointer((void**)&d_any, h_any, 0));
  }

  int img_blocks() const { return cdiv(ctx.N, 256); }

  void finish_setup() {
    // capacity for every launch shape, so that set_shapes/tune never regrow it
    int slots = std::max({op->max_chi_slots(), op->tsv_slots(), img_blocks(), 1});
    d_part.alloc(sizeof(double) * (size_t)kNumQ * ctx.B * slots);
    MF_CK(cudaMemset(d_part.p, 0, d_part.bytes));
    ctx.part.p = d_part.as<double>();
    ctx.part.slots = slots;
    ctx.part.B = ctx.B;
    if (form == kFormTV) setup_fgp();
    refresh_every = op->corrected() ? op->refresh_period() : 0;
    if (const char* re = getenv("MFISTA_REFRESH_EVERY"))  // anchor refresh period (tuning)
      if (op->corrected() && atoi(re) > 0) refresh_every = atoi(re);
    // kernels per loop step: the anchor refresh block, the gradient block
    // and the rest (trial point, its forward pass, control, momentum)
    ref_block_launches = op->corrected() ? 1 + op->launches_refresh() : 0;
    grad_block_launches = (op->models_z() ? 1 : op->launches_forward()) + op->launches_adjoint() + (joint ? 1 : 0);
    rest_launches = op->launches_forward() + 3 + (form == kFormTV ? 1 : 0) + (joint ? 1 : 0);
    per_step_launches = ref_block_launches + grad_block_launches + rest_launches;
    fixed_launches = 2 * (op->launches_forward() + 2) + 1 + (joint ? 2 : 0);
    const char* hl = getenv("MFISTA_HOST_LOOP");
    host_loop = hl && hl[0] == '1';
    if (const char* lu = getenv("MFISTA_LOOP_UNROLL")) loop_unroll = std::max(1, std::min(8, atoi(lu)));
    if (const char* gi = getenv("MFISTA_GRAD_IF")) grad_if = gi[0] != '0';
    build_graph();
    // set-up copies and memsets ran on the legacy stream, which the solver's
    // non-blocking streams do not wait for
    MF_CK(cudaDeviceSynchronize());
  }

  template <typename K> int max_clusters(K kern, int cs, size_t smem) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return n;
  }

  template <typename K> void prep_fgp_kernel(K kern, int cs, size_t smem) {
    if (cs > 8) MF_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    if (smem) set_smem(kern, smem);
  }

  // Picks the FGP cluster shape: slabs in shared memory with 8 or 16 CTAs
  // when they fit and such a cluster can be resident, else global slabs.
  template <typename T> void pick_fgp_shape() {
    int NX = ctx.tsvNX, NY = ctx.tsvNY;
    const size_t limit = 200 * 1024;
    // few problems: 16 CTAs per problem (more SMs busy, half the rows per CTA);
    // otherwise 8 (the GPU is full either way, fewer cluster-wide barriers)
    const bool few = ctx.B * 8 < 148;
    for (int cs : {few ? 16 : 8, few ? 8 : 16}) {
      int rpc = cdiv(NY, cs);
      size_t bytes = (size_t)6 * rpc * NX * sizeof(T);
      if (bytes > limit) continue;
      prep_fgp_kernel(k_fgp<T, true>, cs, bytes);
      if (max_clusters(k_fgp<T, true>, cs, bytes) > 0) {
        fgp_cs = cs;
        fgp_rpc = rpc;
        fgp_smem = true;
        fgp_smem_bytes = bytes;
        return;
      }
    }
    fgp_cs = 8;
    fgp_rpc = cdiv(NY, fgp_cs);
    fgp_smem = false;
    fgp_smem_bytes = 0;
    prep_fgp_kernel(k_fgp<T, false>, fgp_cs, 0);
    fgp_scratch_stride = (long)fgp_cs * 6 * fgp_rpc * NX * sizeof(T);
    d_fgp.alloc((size_t)ctx.B * fgp_scratch_stride);
  }

  void setup_fgp() {
    if (precision == MFISTA_FP32) pick_fgp_shape<float>();
    else pick_fgp_shape<double>();
  }

  void launch_fgp(cudaStream_t s) {
    FgpArgs a;
    a.z = ctx.z;
    a.dfdx = ctx.dfdx;
    a.xnew = ctx.xnew;
    a.xstride = ctx.xstride;
    a.prm = ctx.prm;
    a.st = ctx.st;
    a.box = box_ptr;
    a.NX = ctx.tsvNX;
    a.NY = ctx.tsvNY;
    a.iters = fgp_iter;
    a.rows_per_cta = fgp_rpc;
    a.scratch = d_fgp.p;
    a.scratch_stride = fgp_scratch_stride;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(fgp_cs, ctx.B, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = fgp_smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = fgp_cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (precision == MFISTA_FP32) {
      if (fgp_smem) MF_CK(cudaLaunchKernelEx(&cfg, k_fgp<float, true>, a));
      else MF_CK(cudaLaunchKernelEx(&cfg, k_fgp<float, false>, a));
    } else {
      if (fgp_smem) MF_CK(cudaLaunchKernelEx(&cfg, k_fgp<double, true>, a));
      else MF_CK(cudaLaunchKernelEx(&cfg, k_fgp<double, false>, a));
    }
  }

  CtrlCfg ctrl_cfg(int mode) const {
    CtrlCfg cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.slots[kQChiZ] = op->chi_slots();
    cfg.slots[kQChiX] = op->chi_slots();
    cfg.slots[kQTsvZ] = form == kFormTSV ? img_blocks() : 0;
    cfg.slots[kQDq1] = img_blocks();
    cfg.slots[kQDq2] = img_blocks();
    cfg.slots[kQL1] = img_blocks();
    cfg.slots[kQReg] = img_blocks();
    cfg.slots[kQNact] = img_blocks();
    cfg.fscale = op->fscale();
    cfg.form = form;
    cfg.mode = mode;
    cfg.B = ctx.B;
    cfg.steps = d_steps.as<unsigned long long>();
    cfg.refresh_every = refresh_every;
    // the corrected forms evaluate F(xnew) and f(z) through differently
    // rounded FP32 paths: near convergence that noise (~1e-9 of F on noisy
    // data) exceeds the true change of a step and would make every trial
    // fail until c overflows; 1e-9 of |Q| stays far below the 1e-6
    // objective the forms are held to, and MFISTA's monotone rule still
    // keeps x whenever F(xnew) rises
    cfg.bt_slack = refresh_every > 0 ? 1e-9 : 0.0;
    cfg.joint = joint ? 1 : 0;
    cfg.lam_t = lam_t;
    cfg.jq = d_jq.as<double>();
    cfg.slots[kQDtZ] = joint ? img_blocks() : 0;
    cfg.slots[kQDtX] = joint ? img_blocks() : 0;
    cfg.eta_first = eta_first;
    return cfg;
  }

  void launch_control(cudaStream_t s, int mode, cudaGraphConditionalHandle h, int set_handle) {
    k_control<<<ctx.B, kControlThreads, 0, s>>>(ctx.prm, ctx.st, ctx.part, ctrl_cfg(mode), d_out.as<FinalOut>(), h, set_handle,
                                     d_any, d_ticket.as<unsigned int>());
    MF_LAUNCH_CK();
  }

  // Adds an IF node (condition hc) at the capture position of s and starts
  // capturing its body on cap_block; returns the stream to enqueue it on.
  cudaStream_t begin_if(cudaStream_t s, cudaGraphConditionalHandle hc) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    MF_CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    MF_CK(cudaGraphAddNode(&node, g, deps, nd, &cp));
    MF_CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    MF_CK(cudaStreamBeginCaptureToGraph(cap_block, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
    return cap_block;
  }
  void end_if() {
    cudaGraph_t out;
    MF_CK(cudaStreamEndCapture(cap_block, &out));
  }

  // One loop step.  cond: inside the device loop's WHILE body, with the
  // refresh and gradient blocks under IF nodes set by k_select_blocks.
  void enqueue_body(cudaStream_t s, cudaGraphConditionalHandle h, int set_handle, bool cond = false) {
    dim3 ig(img_blocks(), ctx.B);
    cudaGraphConditionalHandle h_ref = 0, h_grad = 0;
    if (cond) {
      cudaStreamCaptureStatus cs;
      cudaGraph_t g = nullptr;
      MF_CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
      if (op->corrected()) MF_CK(cudaGraphConditionalHandleCreate(&h_ref, g, 0, 0));
      if (grad_if) MF_CK(cudaGraphConditionalHandleCreate(&h_grad, g, 0, 0));
      k_select_blocks<<<1, 256, 0, s>>>(ctx.st, ctx.B, op->corrected() ? 1 : 0, grad_if ? 1 : 0, h_ref, h_grad,
                                        ref_block_launches,
                                        grad_block_launches, d_steps.as<unsigned long long>() + 2,
                                        d_lists.as<int>());
      MF_LAUNCH_CK();
      ctx.act_lists = d_lists.as<int>();  // for the NUFFT kernels of this step
    }
    if (op->corrected()) {  // new FP64 anchor x_a = x every refresh_every outer iterations
      cudaStream_t bs = cond ? begin_if(s, h_ref) : s;
      k_copy_gated<<<ig, 256, 0, bs>>>(ctx.xa, ctx.x, dm, ctx.st, kGateRefresh);
      MF_LAUNCH_CK();
      op->refresh_anchor(bs, kGateRefresh);
      if (cond) end_if();
    }
    {
      cudaStream_t bs = (cond && grad_if) ? begin_if(s, h_grad) : s;
      // gradient at z (only problems that start a new outer iteration)
      if (op->models_z()) op->forward_z(bs, kGateGrad, kQChiZ);
      else op->forward(bs, ctx.z, kGateGrad, kQChiZ, true);
      // the adjoint folds in the TSV gradient of z; TSV(z) itself is reduced by
      // k_update_tsv with the same tree as TSV(xnew)
      op->adjoint(bs, form == kFormTSV ? ctx.z : nullptr, -1);
      if (joint) {  // temporal gradient and term at z
        k_movie_tgrad<<<ig, 256, 0, bs>>>(ctx.z, ctx.dfdx, dm, d_wt.as<double>(), lam_t, ctx.st, ctx.part);
        MF_LAUNCH_CK();
      }
      if (cond && grad_if) end_if();
    }
    // trial point
    if (form == kFormTSV) {
      k_update_tsv<<<ig, 256, 0, s>>>(ctx.z, ctx.dfdx, ctx.xnew, dm, ctx.prm, ctx.st, box_ptr, mask_ptr, ctx.part);
      MF_LAUNCH_CK();
      if (joint) {
        k_movie_dx<<<ig, 256, 0, s>>>(ctx.xnew, dm, d_wt.as<double>(), ctx.st, kGateTrial, ctx.part);
        MF_LAUNCH_CK();
      }
    } else {
      launch_fgp(s);
      k_stats<<<ig, 256, 0, s>>>(ctx.xnew, ctx.z, ctx.dfdx, dm, ctx.prm, ctx.st, kGateTrial, form, 0, 1, ctx.part);
      MF_LAUNCH_CK();
    }
    op->forward(s, ctx.xnew, kGateTrial, kQChiX, false);
    launch_control(s, kCtrlStep, h, set_handle);
    // image momentum and, for operators that keep visibility models, the
    // models' momentum in the same launch
    k_momentum<<<dim3(img_blocks() + op->model_blocks(), ctx.B), 256, 0, s>>>(ctx.x, ctx.z, ctx.xnew, dm, ctx.st,
                                                                            op->model_momentum(img_blocks()));
    MF_LAUNCH_CK();
    ctx.act_lists = nullptr;
  }

  void drop_graphs() {
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
    if (body_exec) { cudaGraphExecDestroy(body_exec); body_exec = nullptr; }
    if (body_graph) { cudaGraphDestroy(body_graph); body_graph = nullptr; }
  }

  // new operator launch shapes; the solve graph is captured again
  void apply_shapes(const LaunchShapes& sh) {
    MF_CK(cudaStreamSynchronize(stream));
    op->set_shapes(sh);
    drop_graphs();
    const char* hl = getenv("MFISTA_HOST_LOOP");
    host_loop = hl && hl[0] == '1';
    build_graph();
  }

  // Autotuner: times each operator kernel alone (profile_kernel) over its
  // candidate shapes, one knob at a time with the others at their current
  // choice, and captures the graph again.  A batched solve runs most of its
  // iterations with few problems left (the tail of a lambda grid), where
  // launch shapes that spread one problem over more CTAs win, so every
  // candidate is timed twice: with the whole batch active (t_all) and with
  // one problem active (t_one).  The choice minimises
  // t_all / min t_all + 2 t_one / min t_one: a lambda grid's iteration
  // counts spread over decades, so many loop steps run with a handful of
  // problems left (the 128x128 64-problem grid: 2234 of 4553 steps with 8
  // or fewer).  ms_out[k]: t_all (ms per launch) of knob k's choice.
  LaunchShapes tune(int reps, double ms_out[4]) {
    LaunchShapes cur = op->shapes();
    // knob -> kernels timed (profile_kernel ids) and candidates
    struct Knob { int LaunchShapes::*field; std::vector<int> kernels; std::vector<int> cand; };
    std::vector<Knob> knobs = {
        {&LaunchShapes::interp_ppw, {0}, {1, 2, 4, 8, 16}},
        {&LaunchShapes::spread_cluster, {1}, {1, 2, 4, 8, 16}},
        {&LaunchShapes::rows_per_cta, {2, 5}, {1, 2, 4, 8, 16}},
        {&LaunchShapes::cols_per_cta, {3, 4}, {1, 2, 4, 8, 16}},
    };
    for (size_t k = 0; k < knobs.size(); ++k) {
      ms_out[k] = 0;
      Knob& kb = knobs[k];
      if (cur.*(kb.field) == 0) continue;  // not used by this operator
      std::vector<int> vals;
      std::vector<double> t_all, t_one;
      for (int v : kb.cand) {
        LaunchShapes tr = cur;
        tr.*(kb.field) = v;
        try {
          op->set_shapes(tr);
        } catch (const Error&) {
          continue;  // shape not possible for this problem size
        }
        if (kb.field == &LaunchShapes::spread_cluster && !spread_cluster_fits(v)) continue;
        double ta = 0, t1 = 0;
        for (int kern : kb.kernels) {
          double ms = 0, by = 0;
          profile_kernel(kern, 1, ms, by);  // warm
          profile_kernel(kern, reps, ms, by);
          ta += ms;
          profile_kernel(kern, reps, ms, by, 1);
          t1 += ms;
        }
        vals.push_back(v);
        t_all.push_back(ta);
        t_one.push_back(t1);
      }
      if (!vals.empty()) {
        const double ma = *std::min_element(t_all.begin(), t_all.end());
        const double m1 = *std::min_element(t_one.begin(), t_one.end());
        size_t best = 0;
        double best_score = 1e300;
        for (size_t i = 0; i < vals.size(); ++i) {
          const double score = t_all[i] / ma + 2.0 * t_one[i] / m1;
          if (score < best_score) {
            best_score = score;
            best = i;
          }
        }
        cur.*(kb.field) = vals[best];
        ms_out[k] = t_all[best];
      }
      op->set_shapes(cur);
    }
    apply_shapes(cur);
    return cur;
  }

  // can a cluster of `cs` spreading CTAs be resident on this GPU?
  bool spread_cluster_fits(int cs) {
    if (precision == MFISTA_FP32)
      return max_clusters(k_nufft_spread_shared<float>, cs, sizeof(cplx<float>) * SharedChunk<float>::kSpread * 256) > 0;
    return max_clusters(k_nufft_spread_shared<double>, cs, sizeof(cplx<double>) * SharedChunk<double>::kSpread * 256) > 0;
  }

  void build_graph() {
    cond_blocks = false;
    if (!host_loop) {
      cudaError_t e = try_build_conditional();
      ctx.act_lists = nullptr;  // only the captured loop body uses them
      if (e == cudaSuccess) return;
      cudaGetLastError();
      if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
      if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
      host_loop = true;
    }
    MF_CK(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
    enqueue_body(cap_stream, 0, 0);
    MF_CK(cudaStreamEndCapture(cap_stream, &body_graph));
    MF_CK(cudaGraphInstantiate(&body_exec, body_graph, 0));
  }

  cudaError_t try_build_conditional() {
    cudaError_t e;
    if ((e = cudaGraphCreate(&graph, 0)) != cudaSuccess) return e;
    cudaGraphConditionalHandle h;
    if ((e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp)) != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(cap_stream, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return e;
    try {
      // the body holds loop_unroll steps: each pass of the WHILE node costs
      // a device-side body launch (about 17 us measured between the last
      // kernel of a step and the first of the next), paid once per
      // loop_unroll steps; steps after every problem has stopped find all
      // gates closed and change nothing
      for (int u = 0; u < loop_unroll; ++u) enqueue_body(cap_stream, h, 1, true);
    } catch (...) {
      cudaGraph_t tmp;
      cudaStreamEndCapture(cap_block, &tmp);
      cudaStreamEndCapture(cap_stream, &tmp);
      cudaGetLastError();
      return cudaErrorNotSupported;  // falls back to the host loop
    }
    cudaGraph_t out;
    if ((e = cudaStreamEndCapture(cap_stream, &out)) != cudaSuccess) return e;
    if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) return e;
    cond_blocks = true;
    return cudaSuccess;
  }

  // params: per problem; x0: [B*N] host (null = zeros); skip_loop: start
  // from x0 and only compute the summary (reference early-return cases)
  void upload_problems(const std::vector<ProbParams>& prm, const double* x0) {
    MF_CK(cudaMemcpyAsync(ctx.prm, prm.data(), sizeof(ProbParams) * ctx.B, cudaMemcpyHostToDevice, stream));
    size_t bytes = sizeof(double) * (size_t)ctx.B * ctx.N;
    if (x0) MF_CK(cudaMemcpyAsync(ctx.x, x0, bytes, cudaMemcpyHostToDevice, stream));
    else MF_CK(cudaMemsetAsync(ctx.x, 0, bytes, stream));
    // device step budget: generous against the reference's own bound
    // (maxiter outer iterations, each with at most maxiter trials)
    long long mx = 1;
    for (const ProbParams& p : prm) mx = std::max<long long>(mx, p.maxiter);
    steps_host[0] = 0;
    steps_host[1] = (unsigned long long)(mx * 64 + 4096);
    steps_host[2] = 0;
    MF_CK(cudaMemcpyAsync(d_steps.p, steps_host, sizeof(steps_host), cudaMemcpyHostToDevice, stream));
  }
  // [0] loop steps taken, [1] step budget, [2] kernels launched by the
  // conditional blocks
  unsigned long long steps_host[3] = {0, 0, 0};

  // times one kernel alone: every problem active at the start of an outer
  // iteration, `reps` launches between two events on the solver stream
  // Times one operator kernel alone with the first n_active problems active
  // (every problem when n_active < 0).
  void profile_kernel(int kernel, int reps, double& ms, double& bytes, int n_active = -1) {
    std::vector<ProbState> st(ctx.B);
    std::vector<ProbParams> prm(ctx.B);
    MF_CK(cudaMemcpy(prm.data(), ctx.prm, sizeof(ProbParams) * ctx.B, cudaMemcpyDeviceToHost));
    for (int b = 0; b < ctx.B; ++b) {
      memset(&st[b], 0, sizeof(ProbState));
      st[b].active = (n_active < 0 || b < n_active) ? 1 : 0;
      st[b].need_grad = 1;
      st[b].c = prm[b].cinit > 0 ? prm[b].cinit : 1.0;
    }
    MF_CK(cudaMemcpy(ctx.st, st.data(), sizeof(ProbState) * ctx.B, cudaMemcpyHostToDevice));
    auto one = [&]() -> double {
      if (kernel == 6) {
        dim3 ig(img_blocks(), ctx.B);
        if (form == kFormTSV) {
          k_update_tsv<<<ig, 256, 0, stream>>>(ctx.z, ctx.dfdx, ctx.xnew, dm, ctx.prm, ctx.st, box_ptr, mask_ptr,
                                                ctx.part);
          MF_LAUNCH_CK();
        } else {
          launch_fgp(stream);
        }
        return (double)ctx.B * ctx.N * 24.0;
      }
      return op->launch_single(stream, kernel);
    };
    bytes = one();
    if (bytes < 0) throw Error(MFISTA_ERR_ARG, "no such kernel for this operator");
    cudaEvent_t e0, e1;
    MF_CK(cudaEventCreate(&e0));
    MF_CK(cudaEventCreate(&e1));
    MF_CK(cudaEventRecord(e0, stream));
    for (int r = 0; r < reps; ++r) one();
    MF_CK(cudaEventRecord(e1, stream));
    MF_CK(cudaEventSynchronize(e1));
    float t = 0;
    MF_CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ms = t / reps;
  }

  long long steps_taken() {
    unsigned long long h[3];
    MF_CK(cudaMemcpy(h, d_steps.p, sizeof(h), cudaMemcpyDeviceToHost));
    return (long long)h[0];
  }
  // kernels launched by the last solve's loop
  long long loop_launches() {
    unsigned long long h[3];
    MF_CK(cudaMemcpy(h, d_steps.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (!cond_blocks) return (long long)h[0] * per_step_launches;
    return (long long)h[0] * (rest_launches + 1 + (grad_if ? 0 : grad_block_launches)) + (long long)h[2];
  }

  void enqueue_solve(bool skip_loop) {
    dim3 ig(img_blocks(), ctx.B);
    size_t bytes = sizeof(double) * (size_t)ctx.B * ctx.N;
    MF_CK(cudaMemcpyAsync(ctx.z, ctx.x, bytes, cudaMemcpyDeviceToDevice, stream));
    k_init_state<<<cdiv(ctx.B, 128), 128, 0, stream>>>(ctx.st, ctx.B, 0);
    MF_LAUNCH_CK();
    if (op->corrected()) {  // anchor = starting point
      k_copy_gated<<<ig, 256, 0, stream>>>(ctx.xa, ctx.x, dm, ctx.st, kGateInit);
      MF_LAUNCH_CK();
      op->refresh_anchor(stream, kGateInit);
    }
    if (!skip_loop) {
      op->forward_exact(stream, ctx.x, kGateInit, kQChiX, false);
      k_stats<<<ig, 256, 0, stream>>>(ctx.x, nullptr, nullptr, dm, ctx.prm, ctx.st, kGateInit, form, 0, 0, ctx.part);
      MF_LAUNCH_CK();
      if (joint) {
        k_movie_dx<<<ig, 256, 0, stream>>>(ctx.x, dm, d_wt.as<double>(), ctx.st, kGateInit, ctx.part);
        MF_LAUNCH_CK();
      }
      launch_control(stream, kCtrlInit, 0, 0);
      if (!host_loop) {
        MF_CK(cudaGraphLaunch(exec, stream));
      } else {
        for (;;) {
          for (int k = 0; k < 8; ++k) MF_CK(cudaGraphLaunch(body_exec, stream));
          MF_CK(cudaStreamSynchronize(stream));
          if (*(volatile int*)h_any == 0) break;
        }
      }
    }
    // summary at x (calc_result_*), with the FP64 operator
    op->forward_exact(stream, ctx.x, kGateAll, kQChiX, true);
    k_stats<<<ig, 256, 0, stream>>>(ctx.x, nullptr, nullptr, dm, ctx.prm, ctx.st, kGateAll, form, 1, 0, ctx.part);
    MF_LAUNCH_CK();
    if (joint) {
      k_movie_dx<<<ig, 256, 0, stream>>>(ctx.x, dm, d_wt.as<double>(), ctx.st, kGateAll, ctx.part);
      MF_LAUNCH_CK();
    }
    launch_control(stream, kCtrlFinal, 0, 0);
  }

  void fetch(double* xout, std::vector<FinalOut>& out) {
    out.resize(ctx.B);
    MF_CK(cudaMemcpyAsync(out.data(), d_out.p, sizeof(FinalOut) * ctx.B, cudaMemcpyDeviceToHost, stream));
    if (xout)
      MF_CK(cudaMemcpyAsync(xout, ctx.x, sizeof(double) * (size_t)ctx.B * ctx.N, cudaMemcpyDeviceToHost, stream));
    MF_CK(cudaStreamSynchronize(stream));
  }
};

}  // namespace mf
