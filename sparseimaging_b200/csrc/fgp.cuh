// FGP total-variation proximal operator (c/mfista_TV_lib.c:124-384) as one
// persistent launch per problem: a thread-block cluster owns a problem, each
// CTA a slab of image rows (the NY x NX view of the flat image), and all FGP
// iterations run inside the kernel.  Dual variables live in shared memory
// when the slab fits (halo rows are read from the neighbouring CTA's shared
// memory through DSMEM), otherwise in a per-problem global scratch that the
// same code addresses directly; cluster barriers separate the two stencil
// phases of every iteration.  No TMA and no multicast are used.
//
// Per iteration (c/mfista_TV_lib.c:208-244):
//   A: xv = prox(b - lambda_tv * Lpq(r, s))
//   B: r' = r + Lx(xv)_p / (8 lambda_tv), s' likewise; (np, nq) = P_pqiso(r', s');
//      r = np (1 + (t-1)/t') - p (t-1)/t'; p = np  (same for s, q)
// and finally x = prox(b - lambda_tv * Lpq(p, q)).
#pragma once
#include <cooperative_groups.h>
#include "common.cuh"

namespace mf {

namespace cg = cooperative_groups;

struct FgpArgs {
  const double* z;      // per problem, stride xstride
  const double* dfdx;
  double* xnew;
  long xstride;
  const ProbParams* prm;
  const ProbState* st;
  const float* box;     // shared clean box or null
  int NX, NY;
  int iters;
  int rows_per_cta;
  void* scratch;        // global slabs when not in shared memory
  long scratch_stride;  // bytes per problem
};

// slab arrays: xv, p, q, r, s, b — each rows_per_cta x NX values of T
template <typename T, bool SMEM>
__global__ void k_fgp(FgpArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int csize = (int)cluster.num_blocks();
  const int b = blockIdx.y;
  const ProbState& S = a.st[b];
  // uniform over the cluster (same problem): safe to return before barriers
  if (!gate_ok(S, kGateTrial)) return;
  const ProbParams P = a.prm[b];
  const int NX = a.NX, NY = a.NY, rpc = a.rows_per_cta;
  const int j0 = rank * rpc;
  const int j1 = min(NY, j0 + rpc);
  const int nrow = max(0, j1 - j0);
  const size_t slab = (size_t)rpc * NX;
  T* base;
  if (SMEM) base = reinterpret_cast<T*>(smem_raw);
  else base = reinterpret_cast<T*>(reinterpret_cast<char*>(a.scratch) + (size_t)b * a.scratch_stride) + (size_t)rank * 6 * slab;
  T* XV = base;
  T* PP = base + slab;
  T* QQ = base + 2 * slab;
  T* RR = base + 3 * slab;
  T* SS = base + 4 * slab;
  T* BB = base + 5 * slab;
  // neighbour slabs (rank-1 for the row above, rank+1 for the row below)
  auto peer = [&](T* local, int r) -> T* {
    if (SMEM) return cluster.map_shared_rank(local, r);
    return local + (ptrdiff_t)(r - rank) * 6 * (ptrdiff_t)slab;
  };
  const double c = S.c;
  const double lam_tv = P.lambda_tv / c;
  const double lam_l1 = P.lambda_l1 / c;
  const bool nonneg = P.nonneg == 1;
  const float* box = P.box_flag == 1 ? a.box : nullptr;
  const double* z = a.z + (size_t)b * a.xstride;
  const double* d = a.dfdx + (size_t)b * a.xstride;
  // b = xtmp (c/mfista_nufft_lib.c:424-441) ; duals start at zero
  // thread -> (row, column) walk without integer division: rows_per_pass
  // rows of NX columns per pass when NX <= blockDim.x, else one row with
  // the columns strided by blockDim.x
  const int nt = (int)blockDim.x;
  const int rpp = NX <= nt ? nt / NX : 1;
  const int c_step = NX <= nt ? NX : nt;
  const int jl0 = NX <= nt ? (int)threadIdx.x / NX : 0;
  const int ic0 = NX <= nt ? (int)threadIdx.x - jl0 * NX : (int)threadIdx.x;
  const bool walker = jl0 < rpp;
#define FGP_FOR_LOCAL(JL, I) \
  if (walker)                \
    for (int JL = jl0; JL < nrow; JL += rpp) \
      for (int I = ic0; I < NX; I += c_step)
  FGP_FOR_LOCAL(jl_, i_) {
    const int t = jl_ * NX + i_;
    int f = j0 * NX + t;
    double bv;
    if (nonneg) bv = ((1.0 * (-P.lambda_l1 / c)) + d[f] * (1.0 / c)) + z[f];
    else bv = d[f] * (1.0 / c) + z[f];
    BB[t] = (T)bv;
    PP[t] = 0;
    QQ[t] = 0;
    RR[t] = 0;
    SS[t] = 0;
  }
  const T alpha1 = (T)(-lam_tv);
  const T alpha3 = (T)(1.0 / (8 * lam_tv));
  const T eta = (T)lam_l1;
  auto prox = [&](T v, int f) -> T {
    if (nonneg) {
      if (box && box[f] == 0.0f) return 0;
      return v < 0 ? T(0) : v;
    }
    if (box) {
      if (box[f] == 0.0f || (v < eta && v > -eta)) return 0;
      return v >= eta ? v - eta : v + eta;
    }
    if (v >= eta) return v - eta;
    if (v <= -eta) return v + eta;
    return 0;
  };
  // Lpq of (p, q) at local element t (global row j, column i)
  auto lpq = [&](const T* p, const T* q, const T* q_above, int t, int i, int j) -> T {
    T v = 0;
    if (i >= 1) v -= p[t - 1];
    if (i < NX - 1) v += p[t];
    if (j >= 1) v -= (t >= NX ? q[t - NX] : q_above[i]);
    if (j < NY - 1) v += q[t];
    return v;
  };
  cluster.sync();
  double tt = 1.0;
  for (int it = 0; it <= a.iters; ++it) {
    const bool last = it == a.iters;
    const T* pr = last ? PP : RR;
    const T* qs = last ? QQ : SS;
    // phase A
    {
      const T* qa = (j0 >= 1 && nrow > 0) ? peer(const_cast<T*>(qs), rank - 1) + (size_t)(rpc - 1) * NX : nullptr;
      FGP_FOR_LOCAL(jl, i) {
        const int t = jl * NX + i;
        int j = j0 + jl;
        T l = lpq(pr, qs, qa, t, i, j);
        T v = l * alpha1 + BB[t];
        v = prox(v, j * NX + i);
        if (last) a.xnew[(size_t)b * a.xstride + (size_t)j * NX + i] = (double)v;
        else XV[t] = v;
      }
    }
    if (last) {
      cluster.sync();  // peers may still be reading this CTA's q slab
      break;
    }
    cluster.sync();
    double tnew = (1 + sqrt(1 + 4 * tt * tt)) / 2;
    const T beta1 = (T)(1 + (tt - 1) / tnew);
    const T beta2 = (T)(-(tt - 1) / tnew);
    // phase B
    {
      const T* xb = (j1 < NY && nrow > 0 && rank + 1 < csize) ? peer(XV, rank + 1) : nullptr;
      FGP_FOR_LOCAL(jl, i) {
        const int t = jl * NX + i;
        int j = j0 + jl;
        T xv = XV[t];
        bool hp = i < NX - 1, hq = j < NY - 1;
        T rp = 0, sq = 0;
        if (hp) rp = RR[t] + alpha3 * (xv - XV[t + 1]);
        if (hq) {
          T below = (jl + 1 < nrow) ? XV[t + NX] : xb[i];
          sq = SS[t] + alpha3 * (xv - below);
        }
        T np = 0, nq = 0;
        if (hp && hq) {
          T tmp = sqrt(rp * rp + sq * sq);
          if (tmp < 1) tmp = 1;
          np = rp / tmp;
          nq = sq / tmp;
        } else if (hp) {
          T tmp = fabs(rp);
          if (tmp < 1) tmp = 1;
          np = rp / tmp;
        } else if (hq) {
          T tmp = fabs(sq);
          if (tmp < 1) tmp = 1;
          nq = sq / tmp;
        }
        if (hp) {
          RR[t] = np * beta1 + beta2 * PP[t];
          PP[t] = np;
        }
        if (hq) {
          SS[t] = nq * beta1 + beta2 * QQ[t];
          QQ[t] = nq;
        }
      }
    }
    tt = tnew;
    cluster.sync();
  }
}
#undef FGP_FOR_LOCAL

}  // namespace mf
