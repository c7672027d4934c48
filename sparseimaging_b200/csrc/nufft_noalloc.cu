// mfista_nufft_forward_noalloc: the FP64 NUFFT forward operator A x
// (NUFFT2d2, c/mfista_nufft_lib.c:187-243) for callers that may not
// allocate GPU memory.
//
// Who cannot allocate: a host framework that owns the device's memory
// through its own pool and forbids cudaMalloc/cudaFree behind its back
// (a free also synchronises the device), a real-time pipeline that fixes
// all of its memory at start-up, and a caller that is building a CUDA graph
// or streaming work and cannot afford a device-wide synchronisation.  Those
// callers already hold u, v, x and the output on the device.
// mfista_nufft_forward allocates its working buffers on every call; this
// variant keeps all of its intermediates (grid indices and tap weights of the
// points, the grid-correction factors, FFT twiddles, the half-plane grid,
// A x) in one file-scope device array of fixed size instead.
//
// What a caller must know:
//   * the array is MFISTA_NOALLOC_SCRATCH_BYTES (16 MiB).  A device holds it
//     from the time this file's device code is loaded there (at the latest,
//     the first call on that device) until the process exits;
//   * inputs whose working set does not fit it are rejected with
//     MFISTA_ERR_ARG before any work is enqueued;
//   * the first call on a device looks up the array's device address there
//     (cudaGetSymbolAddress, with that device current) and keeps it: make
//     that first call before any stream capture.  A cudaDeviceReset unloads
//     the array with the rest of the device's state, and the kept address
//     then points at freed memory: after resetting a device, do not call this
//     entry point on it again in the same process;
//   * a CUDA error already pending in the calling thread when the call starts
//     (an earlier launch of the caller's that failed) is reported as
//     MFISTA_ERR_CUDA before anything is enqueued, and left pending for the
//     caller to read;
//   * every call uses the same array and leaves its contents behind; calls
//     that run at the same time on one GPU (two streams, two host threads)
//     race on it and must be ordered by the caller;
//   * the work is enqueued on `stream`; the call does not wait for it.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include <string.h>

#include "common.cuh"
#include "fft_smem.cuh"
#include "nufft_ops.cuh"

#include "../../include/mfista_b200.h"

namespace mf {
namespace {

constexpr size_t kNoAllocBytes = MFISTA_NOALLOC_SCRATCH_BYTES;
// the scratch array; host code must not pass this name to a kernel (on the
// host it is a stand-in object, not a device address)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_dev[kMaxDevices] = {};  // device address, per device

// default dynamic shared-memory limit: larger FFTs would need a per-kernel
// attribute, which is global state shared with the allocating entry points
constexpr size_t kSmemDefault = 48 * 1024;

// 256-byte aligned pieces of the scratch array
struct Carve {
  size_t off = 0;
  template <typename U> size_t take(size_t count) {
    size_t at = off;
    off += (count * sizeof(U) + 255) & ~size_t(255);
    return at;
  }
};

// grid index of each point, preNUFFT (c/mfista_nufft_lib.c:92-96)
__global__ void k_noalloc_grid_index(const double* __restrict__ u, const double* __restrict__ v, int m, int nx,
                                     int ny, int* __restrict__ mx, int* __restrict__ my) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double pi = 3.14159265358979323846;
  double mrx = 2.0 * nx, mry = 2.0 * ny;
  mx[k] = (int)round(u[k] * mrx / (2 * pi));
  my[k] = (int)round(v[k] * mry / (2 * pi));
}

// tw[k] = exp(-2 pi i k / n)
__global__ void k_noalloc_twiddles(cplx<double>* __restrict__ tw, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s, c;
  sincospi(2.0 * (double)k / (double)n, &s, &c);
  tw[k] = mk<double>(c, -s);
}

// one active problem over points [0, m)
__global__ void k_noalloc_state(ProbState* st, int* lo, int* hi, int m) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  memset(st, 0, sizeof(ProbState));
  st->active = 1;
  st->need_grad = 1;
  lo[0] = 0;
  hi[0] = m;
}

__global__ void k_noalloc_split(const double2* __restrict__ ax, int m, double* __restrict__ out_r,
                                double* __restrict__ out_i) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  out_r[k] = ax[k].x;
  out_i[k] = ax[k].y;
}

// same radix order as the allocating operator's FFT plans
bool factor(int n, FftDev<double>& f) {
  memset(&f, 0, sizeof(f));
  f.n = n;
  int m = n;
  auto push = [&](int r) {
    if (f.nst >= kMaxStages) return false;
    f.radix[f.nst++] = r;
    return true;
  };
  while (m % 4 == 0) { if (!push(4)) return false; m /= 4; }
  while (m % 2 == 0) { if (!push(2)) return false; m /= 2; }
  while (m % 3 == 0) { if (!push(3)) return false; m /= 3; }
  while (m % 5 == 0) { if (!push(5)) return false; m /= 5; }
  for (int p = 7; m > 1 && p <= kMaxGenericRadix; p += 2)
    while (m % p == 0) { if (!push(p)) return false; m /= p; }
  return m == 1;
}

inline int cdiv_i(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace
}  // namespace mf

using namespace mf;

extern "C" int mfista_nufft_forward_noalloc(const double* u_dx, const double* v_dy, int M, int Nx, int Ny,
                                            const double* x, double* out_r, double* out_i, void* stream) {
  if (M < 1 || Nx < 12 || Ny < 12 || !u_dx || !v_dy || !x || !out_r || !out_i) return MFISTA_ERR_ARG;
  if ((long)Nx * Ny > (long)kNoAllocBytes || M > (int)(kNoAllocBytes / 256)) return MFISTA_ERR_ARG;
  // working set laid out in the scratch array
  Carve cv;
  const size_t o_grid = cv.take<cplx<double>>((size_t)2 * Nx * (Ny + 1));
  const size_t o_wx = cv.take<double>((size_t)M * kTaps);
  const size_t o_wy = cv.take<double>((size_t)M * kTaps);
  const size_t o_mx = cv.take<int>(M);
  const size_t o_my = cv.take<int>(M);
  const size_t o_ax = cv.take<double2>(M);
  const size_t o_e4 = cv.take<double>((size_t)Nx * Ny);
  const size_t o_tw_h = cv.take<cplx<double>>(Ny);
  const size_t o_tw_c = cv.take<cplx<double>>((size_t)2 * Nx);
  const size_t o_tw_2h = cv.take<cplx<double>>((size_t)2 * Ny);
  const size_t o_st = cv.take<ProbState>(1);
  const size_t o_lo = cv.take<int>(1);
  const size_t o_hi = cv.take<int>(1);
  if (cv.off > kNoAllocBytes) return MFISTA_ERR_ARG;
  // an error pending from the caller's own work: report it, do not consume it
  if (cudaPeekAtLastError() != cudaSuccess) return MFISTA_ERR_CUDA;
  FftDev<double> fh, fcol;
  if (!factor(Ny, fh) || !factor(2 * Nx, fcol)) return MFISTA_ERR_ARG;
  // one row / one column per CTA, ping-pong buffers in shared memory
  const size_t smem_rows = (size_t)2 * (Ny + 1) * sizeof(cplx<double>);
  const size_t smem_cols = (size_t)2 * (2 * Nx + 1) * sizeof(cplx<double>);
  if (smem_rows > kSmemDefault || smem_cols > kSmemDefault) return MFISTA_ERR_ARG;

  // device address of the scratch array on the current device (once per device)
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MFISTA_ERR_CUDA;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();  // this call's own error (none was pending on entry)
        return MFISTA_ERR_CUDA;
      }
      g_scratch_dev[dev] = static_cast<unsigned char*>(p);
    }
    base = g_scratch_dev[dev];
  }

  cplx<double>* grid = reinterpret_cast<cplx<double>*>(base + o_grid);
  double* wx = reinterpret_cast<double*>(base + o_wx);
  double* wy = reinterpret_cast<double*>(base + o_wy);
  int* mx = reinterpret_cast<int*>(base + o_mx);
  int* my = reinterpret_cast<int*>(base + o_my);
  double2* ax = reinterpret_cast<double2*>(base + o_ax);
  double* e4 = reinterpret_cast<double*>(base + o_e4);
  cplx<double>* tw_2h = reinterpret_cast<cplx<double>*>(base + o_tw_2h);
  ProbState* st = reinterpret_cast<ProbState*>(base + o_st);
  int* lo = reinterpret_cast<int*>(base + o_lo);
  int* hi = reinterpret_cast<int*>(base + o_hi);
  fh.tw = reinterpret_cast<cplx<double>*>(base + o_tw_h);
  fcol.tw = reinterpret_cast<cplx<double>*>(base + o_tw_c);

  // Every piece is written in full before it is read, so nothing left by an
  // earlier call is used and nothing needs clearing: the row pass writes all
  // Ny + 1 columns of the Nx grid rows that hold image data, the column pass
  // reads only those rows and writes all 2 Nx.
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int T = 256;
  k_noalloc_state<<<1, 32, 0, s>>>(st, lo, hi, M);
  k_noalloc_twiddles<<<cdiv_i(Ny, T), T, 0, s>>>(const_cast<cplx<double>*>(fh.tw), Ny);
  k_noalloc_twiddles<<<cdiv_i(2 * Nx, T), T, 0, s>>>(const_cast<cplx<double>*>(fcol.tw), 2 * Nx);
  k_noalloc_twiddles<<<cdiv_i(2 * Ny, T), T, 0, s>>>(tw_2h, 2 * Ny);
  k_noalloc_grid_index<<<cdiv_i(M, T), T, 0, s>>>(u_dx, v_dy, M, Nx, Ny, mx, my);
  k_nufft_prep_points<double><<<cdiv_i(M, T), T, 0, s>>>(u_dx, v_dy, mx, my, M, Nx, Ny, wx, wy);
  k_nufft_prep_e4<<<cdiv_i((long)Nx * Ny, T), T, 0, s>>>(e4, Nx, Ny);
  k_nufft_rows_fwd<double><<<dim3(Nx, 1), T, smem_rows, s>>>(x, (long)Nx * Ny, e4, grid, 0, Nx, Ny, fh, tw_2h, st,
                                                              kGateAll, 1, nullptr, DynUnits{nullptr, 0});
  k_nufft_cols<double><<<dim3(Ny + 1, 1), T, smem_cols, s>>>(grid, 0, Nx, Ny, fcol, -1, 1, 1, 0, st, kGateAll,
                                                              DynUnits{nullptr, 0});
  NufftGeom<double> geo;
  memset(&geo, 0, sizeof(geo));
  geo.mx = mx;
  geo.my = my;
  geo.wx = wx;
  geo.wy = wy;
  // the interpolation also forms a weighted residual against visibilities;
  // with no residual or chi^2 output requested it only reads them, so any
  // M readable doubles serve
  geo.vis_r = u_dx;
  geo.vis_i = u_dx;
  geo.weight = u_dx;
  geo.pt_lo = lo;
  geo.pt_hi = hi;
  geo.y2_bstride = M;
  geo.e4 = e4;
  Partials none;
  memset(&none, 0, sizeof(none));
  none.B = 1;
  constexpr int ppw = SharedChunk<double>::kInterpPts;
  k_nufft_interp_shared<double><<<dim3(cdiv_i(M, 8 * ppw), 1), T, 0, s>>>(
      geo, grid, 0, Nx, Ny, 1.0 / ((double)(2 * Nx) * (double)(2 * Ny)), st, kGateAll, none, -1, nullptr, 1, nullptr,
      ax, ppw);
  k_noalloc_split<<<cdiv_i(M, T), T, 0, s>>>(ax, M, out_r, out_i);
  // nothing was pending on entry, so an error now is one of these launches
  return cudaGetLastError() == cudaSuccess ? MFISTA_OK : MFISTA_ERR_CUDA;
}
