// Operator-independent MFISTA kernels: the fused gradient-step / proximal /
// objective-terms kernel of the TSV form, the statistics kernel (|x|_1, TSV or
// TV, Q-model terms, active pixels), the momentum update, and the FP64
// control kernel that runs the reference's backtracking, monotone-accept and
// stopping logic (c/mfista_nufft_lib.c:660-744 and its copies in
// c/mfista_fft_lib.c and c/mfista_dft_lib.c) for every problem of a batch.
#pragma once
#include "common.cuh"

namespace mf {

// soft thresholds (c/mfista_tools.c:81-141), P_positive(_box) in TV_lib
__device__ __forceinline__ double prox_l1(double v, double eta, int nonneg, const float* box, int f) {
  if (nonneg == 1) {
    if (box) return (box[f] == 0.0f || v < eta) ? 0.0 : v - eta;
    return v < eta ? 0.0 : v - eta;
  }
  if (box) {
    if (box[f] == 0.0f || (v < eta && v > -eta)) return 0.0;
    return v >= eta ? v - eta : v + eta;
  }
  if (v >= eta) return v - eta;
  if (v <= -eta) return v + eta;
  return 0.0;
}

__device__ __forceinline__ double tv_terms_at(const double* __restrict__ x, int f, int NX, int NY) {
  int i = f % NX, j = f / NX;
  double xf = x[f];
  if (i < NX - 1 && j < NY - 1) {
    double a = xf - x[f + 1], c = xf - x[f + NX];
    return sqrt(a * a + c * c);
  }
  if (j == NY - 1 && i < NX - 1) return fabs(xf - x[f + 1]);
  if (i == NX - 1 && j < NY - 1) return fabs(xf - x[f + NX]);
  return 0.0;
}

__device__ __forceinline__ double tsv_pairs_at(const double* __restrict__ x, int f, int NX, int NY) {
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

// regulariser measured for a problem: 0 none, 1 TSV, 2 TV
__device__ __forceinline__ int reg_kind(const ProbParams& p, int form, int final_summary) {
  if (final_summary) {  // calc_result_* (:873-883)
    if (p.lambda_tsv > 0) return 1;
    if (p.lambda_tv > 0) return 2;
    return 0;
  }
  if (form == kFormTV) return 2;
  return p.lambda_tsv > 0 ? 1 : 0;
}

struct ImgDims {
  int N;       // pixels
  int NX, NY;  // TSV/TV view
  long xstride;
};

// ---------------------------------------------------------------------------
// TSV form trial step (c/mfista_nufft_lib.c:684-700):
//   xtmp = dfdx/c + z ; xnew = soft_th(xtmp, lambda_l1/c)
// fused with the Q-model dot products (calc_Q_part), |xnew|_1, TSV(xnew) and
// TSV(z).  TSV(z) (for Qcore) and TSV(xnew) (for F) go through the same
// decomposition and summation tree, so that xnew == z gives F == Q exactly,
// as the reference's single TSV() does; two different reduction orders let
// rounding fail the backtracking test forever once the step is tiny.
// ---------------------------------------------------------------------------
__global__ void k_update_tsv(const double* __restrict__ zall, const double* __restrict__ dall,
                             double* __restrict__ xnall, ImgDims dm, const ProbParams* __restrict__ prm,
                             const ProbState* __restrict__ st, const float* __restrict__ box,
                             const double* __restrict__ mask, Partials part) {
  __shared__ double sh[5 * 32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], kGateTrial)) return;
  const ProbParams p = prm[b];
  const double c = st[b].c;
  const double cinv = 1.0 / c;
  const double eta = p.lambda_l1 / c;
  const double* z = zall + (size_t)b * dm.xstride;
  const double* d = dall + (size_t)b * dm.xstride;
  double* xn = xnall + (size_t)b * dm.xstride;
  const float* bx = p.box_flag == 1 ? box : nullptr;
  // the movie's c_box (matlab/MFISTA_movie_eht.m:143-146) scales the
  // thresholded image pixel by pixel
  auto prox_at = [&](int ff) {
    const double pv = prox_l1(d[ff] * cinv + z[ff], eta, p.nonneg, bx, ff);
    return mask ? pv * mask[ff] : pv;
  };
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < dm.N) {
    double xv = prox_at(f);
    xn[f] = xv;
    double df = xv - z[f];
    v[0] = d[f] * df;
    v[1] = df * df;
    v[2] = fabs(xv);
    if (p.lambda_tsv > 0) {
      int i = f % dm.NX, j = f / dm.NX;
      if (i < dm.NX - 1) {
        double o = prox_at(f + 1);
        v[3] += (xv - o) * (xv - o);
      }
      if (j < dm.NY - 1) {
        double o = prox_at(f + dm.NX);
        v[3] += (xv - o) * (xv - o);
      }
      v[4] = tsv_pairs_at(z, f, dm.NX, dm.NY);
    }
  }
  block_sum<5>(v, sh);
  if (threadIdx.x == 0) {
    part.at(kQDq1, b)[blockIdx.x] = v[0];
    part.at(kQDq2, b)[blockIdx.x] = v[1];
    part.at(kQL1, b)[blockIdx.x] = v[2];
    part.at(kQReg, b)[blockIdx.x] = v[3];
    part.at(kQTsvZ, b)[blockIdx.x] = v[4];
  }
}

// ---------------------------------------------------------------------------
// statistics of a vector v: |v|_1, regulariser, active pixels and (optionally)
// the Q-model dot products against z and dfdx.  Used for the initial cost,
// the TV form's trial point and the final summary (calc_result_*).
// ---------------------------------------------------------------------------
__global__ void k_stats(const double* __restrict__ vall, const double* __restrict__ zall,
                        const double* __restrict__ dall, ImgDims dm, const ProbParams* __restrict__ prm,
                        const ProbState* __restrict__ st, int gate, int form, int final_summary, int want_q,
                        Partials part) {
  __shared__ double sh[5 * 32];
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  const ProbParams p = prm[b];
  const double* v = vall + (size_t)b * dm.xstride;
  int rk = reg_kind(p, form, final_summary);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < dm.N) {
    double xv = v[f];
    acc[2] = fabs(xv);
    acc[4] = fabs(xv) > 0 ? 1.0 : 0.0;
    if (rk == 1) acc[3] = tsv_pairs_at(v, f, dm.NX, dm.NY);
    else if (rk == 2) acc[3] = tv_terms_at(v, f, dm.NX, dm.NY);
    if (want_q) {
      const double* z = zall + (size_t)b * dm.xstride;
      const double* d = dall + (size_t)b * dm.xstride;
      double df = xv - z[f];
      acc[0] = d[f] * df;
      acc[1] = df * df;
    }
  }
  block_sum<5>(acc, sh);
  if (threadIdx.x == 0) {
    if (want_q) {
      part.at(kQDq1, b)[blockIdx.x] = acc[0];
      part.at(kQDq2, b)[blockIdx.x] = acc[1];
    }
    part.at(kQL1, b)[blockIdx.x] = acc[2];
    part.at(kQReg, b)[blockIdx.x] = acc[3];
    part.at(kQNact, b)[blockIdx.x] = acc[4];
  }
}

// ---------------------------------------------------------------------------
// momentum (c/mfista_nufft_lib.c:714-739):
//   monotone improvement: z = x (1-mu)/mu' + xnew (1 + (mu-1)/mu'); x = xnew
//   otherwise:            z = x (1 - mu/mu') + xnew mu/mu'
// ---------------------------------------------------------------------------
// Kept visibility models of the corrected FP32 NUFFT form, updated with the
// same momentum (az = mom_a ax + mom_b axn, ax = axn when the trial point is
// taken) by the CTAs of k_momentum beyond the image's: one launch for both.
struct ModelMom {
  const int* pt_lo;
  const int* pt_hi;
  long bstride;
  double2* ax;
  const double2* axn;
  double2* az;
  int img_blocks;  // CTAs of the image part; the rest cover points
};

__global__ void k_momentum(double* __restrict__ xall, double* __restrict__ zall, const double* __restrict__ xnall,
                           ImgDims dm, const ProbState* __restrict__ st, ModelMom mm) {
  int b = blockIdx.y;
  const ProbState& s = st[b];
  if (!s.accepted) return;
  if (mm.ax && (int)blockIdx.x >= mm.img_blocks) {
    const int k = mm.pt_lo[b] + ((int)blockIdx.x - mm.img_blocks) * blockDim.x + threadIdx.x;
    if (k >= mm.pt_hi[b]) return;
    const size_t e = (size_t)b * mm.bstride + k;
    const double2 x = mm.ax[e], xn = mm.axn[e];
    mm.az[e] = make_double2(s.mom_a * x.x + s.mom_b * xn.x, s.mom_a * x.y + s.mom_b * xn.y);
    if (s.take_x) mm.ax[e] = xn;
    return;
  }
  if ((int)blockIdx.x >= mm.img_blocks) return;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= dm.N) return;
  double* x = xall + (size_t)b * dm.xstride;
  double* z = zall + (size_t)b * dm.xstride;
  const double* xn = xnall + (size_t)b * dm.xstride;
  double xv = x[f], xnv = xn[f];
  z[f] = xv * s.mom_a + xnv * s.mom_b;
  if (s.take_x) x[f] = xnv;
}

// per-problem vector copy dst = src for the problems passing `gate`
__global__ void k_copy_gated(double* __restrict__ dst, const double* __restrict__ src, ImgDims dm,
                             const ProbState* __restrict__ st, int gate) {
  int b = blockIdx.y;
  if (!gate_ok(st[b], gate)) return;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < dm.N) dst[(size_t)b * dm.xstride + f] = src[(size_t)b * dm.xstride + f];
}

// ---------------------------------------------------------------------------
// movie: frames coupled by lam_t sum_b sum_i (x_b,i - x_{b+1},i)^2 wt_b,
// wt_b = 1 / (t_{b+1} - t_b)  (matlab/lib/d_X.m, matlab/lib/dt_X.m)
// ---------------------------------------------------------------------------
// gradient step: dfdx_b -= lam_t dtX(z)_b with
//   dtX_b = 2 (z_b - z_{b+1}) wt_b - 2 (z_{b-1} - z_b) wt_{b-1}
// (missing neighbours drop out), and the partial sums of the pair term
// (z_b - z_{b+1})^2 wt_b into kQDtZ
__global__ void k_movie_tgrad(const double* __restrict__ zall, double* __restrict__ dall, ImgDims dm,
                              const double* __restrict__ wt, double lam_t, const ProbState* __restrict__ st,
                              Partials part) {
  __shared__ double sh[32];
  const int b = blockIdx.y, B = gridDim.y;
  if (!gate_ok(st[b], kGateGrad)) return;
  double acc[1] = {0.0};
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < dm.N) {
    const double zb = zall[(size_t)b * dm.xstride + f];
    double g = 0.0;
    if (b + 1 < B) {
      const double d = zb - zall[(size_t)(b + 1) * dm.xstride + f];
      g += 2 * d * wt[b];
      acc[0] = d * d * wt[b];
    }
    if (b > 0) g -= 2 * (zall[(size_t)(b - 1) * dm.xstride + f] - zb) * wt[b - 1];
    dall[(size_t)b * dm.xstride + f] -= lam_t * g;
  }
  block_sum<1>(acc, sh);
  if (threadIdx.x == 0) part.at(kQDtZ, b)[blockIdx.x] = acc[0];
}

// partial sums of the pair term (v_b - v_{b+1})^2 wt_b into kQDtX
__global__ void k_movie_dx(const double* __restrict__ vall, ImgDims dm, const double* __restrict__ wt,
                           const ProbState* __restrict__ st, int gate, Partials part) {
  __shared__ double sh[32];
  const int b = blockIdx.y, B = gridDim.y;
  if (!gate_ok(st[b], gate)) return;
  double acc[1] = {0.0};
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < dm.N && b + 1 < B) {
    const double d = vall[(size_t)b * dm.xstride + f] - vall[(size_t)(b + 1) * dm.xstride + f];
    acc[0] = d * d * wt[b];
  }
  block_sum<1>(acc, sh);
  if (threadIdx.x == 0) part.at(kQDtX, b)[blockIdx.x] = acc[0];
}

// ---------------------------------------------------------------------------
// control
// ---------------------------------------------------------------------------
enum CtrlMode { kCtrlInit = 0, kCtrlStep = 1, kCtrlFinal = 2 };

struct CtrlCfg {
  int slots[kNumQ];   // partial slots written per quantity
  double fscale;      // F = fscale * sum(chi partials)
  int form;
  int mode;
  int B;
  // steps[0]: loop steps taken so far, steps[1]: budget after which every
  // still-active problem stops (device memory, set per solve)
  unsigned long long* steps;
  int refresh_every;  // > 0: FP32 form, refresh the FP64 anchor this often
  // relative slack of the backtracking test F(xnew) <= Q (1 + slack): 0 for
  // the FP64 forms (the reference's test); a rounding-level allowance for
  // the corrected low-precision forms, whose F and Q come from differently
  // rounded operator paths
  double bt_slack;
  // movie mode: the B problems are the frames of ONE problem with the
  // temporal term lam_t sum_b |x_b - x_{b+1}|^2 / dt_b; one joint c, mu,
  // cost and backtracking decision for all frames.  jq: [B][kNumQ] scratch
  // for the frames' reduced quantities.
  int joint;
  double lam_t;
  double* jq;
  // > 0: backtracking factor of the first outer iteration (the reference's
  // C++ build starts with 10, c++/mfista_nufft_lib.cpp:818, :860-863);
  // 0: ETA throughout (the C library)
  double eta_first;
};

// status codes written to ProbState.status (values of enum mfista_status)
constexpr int kStatusNonFinite = 5;
constexpr int kStatusStepCap = 6;

struct FinalOut {       // one per problem, read back by the host
  double sq_error, l1cost, regcost, finalcost;
  double n_active;
  double lip;
  double dt_pair;       // movie: sum_i (x_b - x_{b+1})^2 / dt_b (0 for the last frame)
  int iters;
  int status;
};

__device__ __forceinline__ double warp_partial_sum(const double* p, int n, int lane) {
  // loads issued 8 ahead (the partials are independent), sums in slot order
  double s = 0.0;
#pragma unroll 8
  for (int i = lane; i < n; i += 32) s += p[i];
  return warp_sum(s);
}

// Movie mode, init and step (matlab/MFISTA_movie_eht.m:93-194): every CTA
// has reduced its frame's quantities into red[]; they go to cfg.jq, and the
// last CTA to arrive sums them over the frames in order and runs the scalar
// logic once for the whole movie:
//   F = sum_b (chi2_b / 2 + lambda_tsv TSV_b) + lam_t dX,  Q likewise at z,
// one backtracking test, one c and mu, one cost ring and stopping rule, and
// the same state written to every frame.  The matlab code has no "x
// becomes a 0 vector" stop; its backtracking also ends once c > 1e200.
__device__ void control_joint(const ProbParams* __restrict__ prm, ProbState* __restrict__ st, const CtrlCfg& cfg,
                              const double* red, cudaGraphConditionalHandle handle, int set_handle,
                              int* __restrict__ any_active, unsigned int* __restrict__ ticket) {
  const int b = blockIdx.x;
  if (threadIdx.x != 0) return;
  for (int q = 0; q < kNumQ; ++q) cfg.jq[(size_t)b * kNumQ + q] = red[q];
  __threadfence();
  const unsigned int t = atomicAdd(ticket, 1u);
  if (t != gridDim.x - 1) return;
  __threadfence();
  double tot[kNumQ];
  for (int q = 0; q < kNumQ; ++q) tot[q] = 0.0;
  for (int k = 0; k < (int)gridDim.x; ++k)
    for (int q = 0; q < kNumQ; ++q) tot[q] += ((volatile double*)cfg.jq)[(size_t)k * kNumQ + q];
  // the frames' states are identical and no CTA of this launch writes them
  ProbState s = st[0];
  const ProbParams p = prm[0];
  const bool tsv_on = p.lambda_tsv > 0;
  if (cfg.mode == kCtrlInit) {
    s.cost_now = cfg.fscale * tot[kQChiX] + p.lambda_l1 * tot[kQL1] + (tsv_on ? p.lambda_tsv * tot[kQReg] : 0.0);
    s.l1x = tot[kQL1];
    s.c = p.cinit;
    s.mu = 1.0;
    s.iter = 0;
    s.trial = 0;
    s.iters_out = 0;
    s.accepted = 0;
    s.take_x = 0;
    s.active = (p.maxiter > 0 && s.status == 0) ? 1 : 0;
    s.need_grad = s.active;
    s.refresh = 0;
  } else if (!s.active) {
    s.accepted = 0;
  } else {
    const bool capped = cfg.steps && (cfg.steps[0] + 1ull >= cfg.steps[1]);
    if (s.need_grad) {
      s.cost[s.iter % kCostRing] = s.cost_now;
      s.qcore = cfg.fscale * tot[kQChiZ] + (tsv_on ? p.lambda_tsv * tot[kQTsvZ] : 0.0) + cfg.lam_t * tot[kQDtZ];
      s.trial = 0;
      s.need_grad = 0;
      s.refresh = 0;
    }
    s.accepted = 0;
    double fval = cfg.fscale * tot[kQChiX] + (tsv_on ? p.lambda_tsv * tot[kQReg] : 0.0) + cfg.lam_t * tot[kQDtX];
    const double qval = (-tot[kQDq1] + s.c * tot[kQDq2] / 2) + s.qcore;
    if (isnan(fval) || isnan(qval) || capped) {
      s.status = capped ? kStatusStepCap : kStatusNonFinite;
      s.active = 0;
      s.iters_out = s.iter + 1;
    } else {
      bool finish = fval <= qval + cfg.bt_slack * fabs(qval);
      if (!finish) {
        s.c *= kEta;
        s.trial += 1;
        finish = s.trial >= p.maxiter || s.c > 1.0e200;
      }
      if (finish) {
        s.c /= kEta;
        const double mu = s.mu;
        const double munew = (1 + sqrt(1 + 4 * mu * mu)) / 2;
        fval += p.lambda_l1 * tot[kQL1];
        if (fval < s.cost[s.iter % kCostRing]) {
          s.cost_now = fval;
          s.mom_a = (1 - mu) / munew;
          s.mom_b = 1 + ((mu - 1) / munew);
          s.take_x = 1;
          s.l1x = tot[kQL1];
        } else {
          s.mom_a = 1 - (mu / munew);
          s.mom_b = mu / munew;
          s.take_x = 0;
        }
        s.accepted = 1;
        bool stop = s.iter >= kMinIter && (s.cost[(s.iter - kTD) % kCostRing] - s.cost[s.iter % kCostRing]) < p.eps;
        if (!stop && p.target > 0 && s.cost_now <= p.target) stop = true;
        if (stop) {
          s.active = 0;
          s.iters_out = s.iter + 1;
        } else {
          s.mu = munew;
          s.iter += 1;
          if (s.iter >= p.maxiter) {
            s.active = 0;
            s.iters_out = p.maxiter;
          } else {
            s.need_grad = 1;
            s.refresh = (cfg.refresh_every > 0 && s.iter % cfg.refresh_every == 0) ? 1 : 0;
          }
        }
      }
    }
  }
  for (int k = 0; k < (int)gridDim.x; ++k) st[k] = s;
  __threadfence();
  if (set_handle) cudaGraphSetConditional(handle, s.active ? 1u : 0u);
  if (any_active) *any_active = s.active;
  if (cfg.mode == kCtrlStep && cfg.steps) cfg.steps[0] += 1ull;
  *ticket = 0u;
}

// One CTA per problem.  One warp per quantity reduces its partial sums (fixed order),
// thread 0 runs the MFISTA scalar logic, and the last CTA to finish (atomic
// ticket) ORs the active flags into the graph's WHILE condition.
constexpr int kControlThreads = 32 * kNumQ;  // one warp per reduced quantity

__global__ void __launch_bounds__(kControlThreads) k_control(const ProbParams* __restrict__ prm, ProbState* __restrict__ st,
                                                 Partials part, CtrlCfg cfg, FinalOut* __restrict__ out,
                                                 cudaGraphConditionalHandle handle, int set_handle,
                                                 int* __restrict__ any_active, unsigned int* __restrict__ ticket) {
  __shared__ double red[kNumQ];
  __shared__ int s_skip;
  __shared__ int s_last;
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_skip = (cfg.mode == kCtrlStep && !st[b].active) ? 1 : 0;
  __syncthreads();
  if (!s_skip) {
    for (int q = warp; q < kNumQ; q += kControlThreads / 32) {
      bool need = q == kQChiX || q == kQL1 || q == kQReg;
      if (cfg.mode == kCtrlStep) need = need || q == kQChiZ || q == kQTsvZ || q == kQDq1 || q == kQDq2;
      if (cfg.mode == kCtrlFinal) need = need || q == kQNact;
      if (cfg.joint) need = need || (q == kQDtX) || (cfg.mode == kCtrlStep && q == kQDtZ);
      double v = need ? warp_partial_sum(part.at(q, b), cfg.slots[q], lane) : 0.0;
      if (lane == 0) red[q] = v;
    }
  }
  __syncthreads();
  if (cfg.joint && cfg.mode != kCtrlFinal) {
    control_joint(prm, st, cfg, red, handle, set_handle, any_active, ticket);
    return;
  }
  if (threadIdx.x == 0) {
    ProbState s = st[b];
    const ProbParams p = prm[b];
    const bool tsv_on = cfg.form == kFormTSV && p.lambda_tsv > 0;
    const double chiX = red[kQChiX], l1 = red[kQL1], reg = red[kQReg];
    if (s_skip) {
      s.accepted = 0;  // finished on an earlier step: its last momentum update already ran
    } else if (cfg.mode == kCtrlInit) {
      double cost = cfg.fscale * chiX + p.lambda_l1 * l1;
      if (cfg.form == kFormTV) cost += p.lambda_tv * reg;
      else if (tsv_on) cost += p.lambda_tsv * reg;
      s.cost_now = cost;
      s.l1x = l1;
      s.c = p.cinit;
      s.mu = 1.0;
      s.iter = 0;
      s.trial = 0;
      s.iters_out = 0;
      s.accepted = 0;
      s.take_x = 0;
      s.active = (p.maxiter > 0 && s.status == 0) ? 1 : 0;
      s.need_grad = s.active;
      s.refresh = 0;
    } else if (cfg.mode == kCtrlStep) {
      const bool capped = cfg.steps && (cfg.steps[0] + 1ull >= cfg.steps[1]);
      if (s.need_grad) {  // a new outer iteration began with this step
        s.cost[s.iter % kCostRing] = s.cost_now;
        s.qcore = cfg.fscale * red[kQChiZ] + (tsv_on ? p.lambda_tsv * red[kQTsvZ] : 0.0);
        s.trial = 0;
        s.need_grad = 0;
        s.refresh = 0;
      }
      s.accepted = 0;
      double fval = cfg.fscale * chiX + (tsv_on ? p.lambda_tsv * reg : 0.0);
      double qval = (-red[kQDq1] + s.c * red[kQDq2] / 2) + s.qcore;
      if (isnan(fval) || isnan(qval) || capped) {
        // NaN never passes the backtracking test; the reference would retry
        // maxiter times per iteration.  Stop this problem with a status.
        s.status = capped ? kStatusStepCap : kStatusNonFinite;
        s.active = 0;
        s.iters_out = s.iter + 1;
      } else {
        bool finish = fval <= qval + cfg.bt_slack * fabs(qval);
        if (!finish) {
          s.c *= (s.iter == 0 && cfg.eta_first > 0) ? cfg.eta_first : kEta;
          s.trial += 1;
          finish = s.trial >= p.maxiter;  // backtracking loop exhausted
        }
        if (finish) {
          s.c /= kEta;
          double mu = s.mu;
          double munew = (1 + sqrt(1 + 4 * mu * mu)) / 2;
          fval += p.lambda_l1 * l1;
          if (cfg.form == kFormTV) fval += p.lambda_tv * reg;
          bool stop = false;
          if (fval < s.cost[s.iter % kCostRing]) {
            s.cost_now = fval;
            s.mom_a = (1 - mu) / munew;
            s.mom_b = 1 + ((mu - 1) / munew);
            s.take_x = 1;
            s.l1x = l1;
          } else {
            s.mom_a = 1 - (mu / munew);
            s.mom_b = mu / munew;
            s.take_x = 0;
            if (s.iter > 1 && s.l1x == 0) stop = true;  // "x becomes a 0 vector"
          }
          s.accepted = 1;
          if (!stop && s.iter >= kMinIter &&
              (s.cost[(s.iter - kTD) % kCostRing] - s.cost[s.iter % kCostRing]) < p.eps)
            stop = true;
          if (!stop && p.target > 0 && s.cost_now <= p.target) stop = true;
          if (stop) {
            s.active = 0;
            s.iters_out = s.iter + 1;
          } else {
            s.mu = munew;
            s.iter += 1;
            if (s.iter >= p.maxiter) {
              s.active = 0;
              s.iters_out = p.maxiter;
            } else {
              s.need_grad = 1;
              s.refresh = (cfg.refresh_every > 0 && s.iter % cfg.refresh_every == 0) ? 1 : 0;
            }
          }
        }
      }
    } else {  // final summary (calc_result_*)
      FinalOut o;
      int rk = reg_kind(p, cfg.form, 1);
      o.sq_error = 2 * (cfg.fscale * chiX);
      o.l1cost = l1;
      o.regcost = reg;
      o.n_active = red[kQNact];
      double fc = o.sq_error / 2;
      if (p.lambda_l1 > 0) fc += p.lambda_l1 * l1;
      if (rk == 1) fc += p.lambda_tsv * reg;
      else if (rk == 2) fc += p.lambda_tv * reg;
      o.finalcost = fc;
      o.lip = s.c;
      o.dt_pair = cfg.joint ? red[kQDtX] : 0.0;
      o.iters = s.iters_out;
      o.status = s.status;
      out[b] = o;
    }
    st[b] = s;
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (s_last) {  // last problem done: publish the loop condition
    __threadfence();
    // the whole CTA reads the problems' flags
    int any = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) any |= ((volatile ProbState*)st)[k].active;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
      if (set_handle) cudaGraphSetConditional(handle, any ? 1u : 0u);
      if (any_active) *any_active = any;
      if (cfg.mode == kCtrlStep && cfg.steps) cfg.steps[0] += 1ull;
      *ticket = 0u;
    }
  }
}

// initialise a batch's states before the init evaluation
__global__ void k_init_state(ProbState* st, int B, int bad_nonneg_tsv) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  ProbState s;
  memset(&s, 0, sizeof(s));
  s.status = 0;
  s.active = 0;
  st[b] = s;
  (void)bad_nonneg_tsv;
}


// Conditional blocks of the device loop: sets the IF handles of the anchor
// refresh block (has_ref) and of the gradient block (has_grad) for this step -- 1 when
// some problem needs it -- and counts the kernels that those blocks launch
// (launched[0]).  With `lists` it also writes this step's problem lists of
// the three loop gates (count, then indices in increasing order; see
// active_chunk), which the NUFFT kernels of the step read instead of every
// problem's state.  One CTA of 256 threads; the blocks' kernels keep their
// per-problem gates.
__global__ void __launch_bounds__(256) k_select_blocks(const ProbState* __restrict__ st, int B, int has_ref,
                                                       int has_grad, cudaGraphConditionalHandle h_ref,
                                                       cudaGraphConditionalHandle h_grad, int n_ref, int n_grad,
                                                       unsigned long long* __restrict__ launched,
                                                       int* __restrict__ lists) {
  __shared__ int s_cnt[kGateLists][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gates[kGateLists] = {kGateGrad, kGateTrial, kGateRefresh};
  int base[kGateLists] = {0, 0, 0};
  int g = 0, r = 0;
  for (int b0 = 0; b0 < B; b0 += 256) {
    const int b = b0 + (int)threadIdx.x;
    bool on[kGateLists];
#pragma unroll
    for (int q = 0; q < kGateLists; ++q) on[q] = b < B && gate_ok(st[b], gates[q]);
    g |= on[0] ? 1 : 0;
    r |= on[2] ? 1 : 0;
    if (lists) {
      unsigned int bal[kGateLists];
#pragma unroll
      for (int q = 0; q < kGateLists; ++q) {
        bal[q] = __ballot_sync(0xffffffffu, on[q]);
        if (lane == 0) s_cnt[q][warp] = __popc(bal[q]);
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kGateLists; ++q) {
        int rank = base[q] + __popc(bal[q] & ((1u << lane) - 1u)), tot = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
          if (w < warp) rank += s_cnt[q][w];
          tot += s_cnt[q][w];
        }
        if (on[q]) lists[(size_t)q * (B + 1) + 1 + rank] = b;
        base[q] += tot;
      }
      __syncthreads();  // s_cnt is rewritten by the next round
    }
  }
  g = __syncthreads_or(g);
  r = __syncthreads_or(r);
  if (threadIdx.x == 0) {
    if (has_ref) cudaGraphSetConditional(h_ref, r ? 1u : 0u);
    if (has_grad) cudaGraphSetConditional(h_grad, g ? 1u : 0u);
    launched[0] += (unsigned long long)((has_ref && r ? n_ref : 0) + (has_grad && g ? n_grad : 0));
    if (lists)
      for (int q = 0; q < kGateLists; ++q) lists[(size_t)q * (B + 1)] = base[q];
  }
}

}  // namespace mf
