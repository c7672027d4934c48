// Shared device/host definitions for the sparseimaging B200 solver library.
//
// Layout conventions are the reference's (c/mfista_nufft_lib.c):
//   image        x[i*Ny + j], i < Nx, j < Ny                      (FP64 always)
//   half grid    G[row*(Ny+1) + col], row < 2Nx, col <= Ny        (complex T)
//   TSV/TV view  the flat image as NY rows of NX (c/mfista_tools.c:145-186)
// T is the arithmetic type of the operators (double for the plain method,
// float for the precision form); objective, reductions and the MFISTA scalar
// logic are FP64 in both.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mf {

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };
template <typename T> using cplx = typename Vec2<T>::type;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T a, T b) {
  cplx<T> r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename T> __device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cplx<T> cconj(cplx<T> a) { return mk<T>(a.x, -a.y); }
// a * (sign * i)
template <typename T> __device__ __forceinline__ cplx<T> cmul_si(cplx<T> a, int sign) {
  return sign < 0 ? mk<T>(a.y, -a.x) : mk<T>(-a.y, a.x);
}

// ---------------------------------------------------------------------------
// reference constants (c/mfista.h:36-41, c/mfista_nufft_lib.c:27-28)
// ---------------------------------------------------------------------------
constexpr int kMinIter = 100;
constexpr int kTD = 50;
constexpr double kEta = 1.1;
constexpr int kMSP = 12;
constexpr int kTaps = 2 * kMSP;  // 24 taps per axis
constexpr int kCostRing = 64;    // holds cost[iter - TD .. iter]

// ---------------------------------------------------------------------------
// per-problem solver state (device resident)
// ---------------------------------------------------------------------------
enum Form { kFormTSV = 0, kFormTV = 1 };
enum Gate { kGateInit = 0, kGateGrad = 1, kGateTrial = 2, kGateFinal = 3, kGateAll = 4, kGateRefresh = 5 };

struct ProbParams {
  double lambda_l1, lambda_tv, lambda_tsv;
  double cinit;
  double eps;  // already scaled the way the reference scales it
  int maxiter;
  int nonneg;
  int box_flag;
  int pad_;
  double target;  // > 0: stop once the accepted objective is <= target
};

struct ProbState {
  // scalars of the MFISTA loop (c/mfista_nufft_lib.c:557-787)
  double c, mu, munew;
  double cost_now;  // costtmp
  double qcore;
  double l1x;       // |x|_1 of the current iterate x
  double mom_a, mom_b;  // z = a*x + b*xnew after an accepted step
  double cost[kCostRing];
  int iter;
  int trial;
  int active;     // problem still iterating
  int need_grad;  // next step starts a new outer iteration
  int grad_now;   // the step in flight computed a gradient
  int accepted;   // momentum kernel must run for this problem
  int take_x;     // accepted step is a monotone improvement: x = xnew
  int iters_out;  // RESULT.ITER once finished
  int status;     // 0 ok; nonzero = error (see mfista_status_*)
  int refresh;    // FP32 form: recompute the FP64 anchor model in this step
};

// reduction quantities written as per-CTA partials
enum Quantity {
  kQChiZ = 0,   // chi^2 at z (gradient step)
  kQTsvZ,       // TSV(z)
  kQChiX,       // chi^2 at the trial point / x / final x
  kQDq1,        // <dfdx, xnew - z>
  kQDq2,        // |xnew - z|^2
  kQL1,         // |v|_1
  kQReg,        // TSV(v) or TV(v)
  kQNact,       // number of nonzero pixels (final summary)
  kQDtZ,        // movie: temporal term sum_i (z_b - z_{b+1})^2 / dt_b at z
  kQDtX,        // movie: the same at the trial point / x
  kNumQ
};

struct Partials {
  double* p;     // [kNumQ][B][slots]
  int slots;     // capacity per (quantity, problem)
  int B;
  __host__ __device__ double* at(int q, int b) const { return p + ((size_t)q * B + b) * slots; }
};

__device__ __forceinline__ bool gate_ok(const ProbState& s, int gate) {
  switch (gate) {
    case kGateGrad: return s.active && s.need_grad;
    case kGateTrial: return s.active != 0;
    case kGateRefresh: return s.active && s.need_grad && s.refresh;
    default: return true;
  }
}

// Problem chunks over the batch's active problems: the problems passing
// `gate`, in index order, are cut into chunks of PB; chunk `chunk` gets
// ranks [chunk PB, chunk PB + PB).  Writes that chunk's problem indices to
// list[] and returns their count (0: nothing to do).  Every CTA of a launch
// sees the same ranking, so a problem lands in exactly one chunk however
// the active problems are spread over the batch.  Called by all threads of
// a 256-thread CTA; s_cnt is 8 ints of shared memory.
//
// Inside the device loop the ranking comes ready-made: k_select_blocks
// writes, at the head of every step, the problems passing the three loop
// gates in index order (`lists`: per gate slot, the count then the indices;
// gate_list_slot), and a CTA copies its chunk from there instead of reading
// every problem's state.  The chunks are the same either way.
__host__ __device__ __forceinline__ int gate_list_slot(int gate) {
  return gate == kGateGrad ? 0 : gate == kGateTrial ? 1 : gate == kGateRefresh ? 2 : -1;
}
constexpr int kGateLists = 3;

template <int PB>
__device__ __forceinline__ int active_chunk(const ProbState* __restrict__ st, int gate, int B, int chunk, int* list,
                                            int* s_cnt, const int* __restrict__ lists = nullptr) {
  const int gl = lists ? gate_list_slot(gate) : -1;
  if (gl >= 0) {
    const int* L = lists + (size_t)gl * (B + 1);
    const int lo = chunk * PB;
    const int cnt = min(max(L[0] - lo, 0), PB);
    if ((int)threadIdx.x < cnt) list[threadIdx.x] = L[1 + lo + threadIdx.x];
    __syncthreads();
    return cnt;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lo = chunk * PB;
  int base_rank = 0;
  for (int base = 0; base < B; base += 256) {
    const int b = base + (int)threadIdx.x;
    const bool on = b < B && gate_ok(st[b], gate);
    const unsigned int bal = __ballot_sync(0xffffffffu, on);
    if (lane == 0) s_cnt[warp] = __popc(bal);
    __syncthreads();
    int r = base_rank + __popc(bal & ((1u << lane) - 1u)), tot = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const int c = s_cnt[w];
      if (w < warp) r += c;
      tot += c;
    }
    if (on && r >= lo && r < lo + PB) list[r - lo] = b;
    base_rank += tot;
    __syncthreads();  // s_cnt is rewritten by the next round
  }
  return min(max(base_rank - lo, 0), PB);
}

// deterministic reductions --------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV values, fixed order (warp butterflies then warp 0).
// `sh` needs 32*NV doubles.  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * 32 + wid] = v[k];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < nw ? sh[k * 32 + lane] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// FFT plan passed by value to kernels
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 20;
template <typename T> struct FftDev {
  int n;
  int nst;
  int radix[kMaxStages];
  const cplx<T>* tw;  // tw[k] = exp(-2 pi i k / n), k < n
};

}  // namespace mf
