// C ABI of libmfista_b200.so (declared in include/mfista_b200.h).
//
// The three reference entry points keep the reference's argument handling
// and RESULT bookkeeping (c/mfista_nufft_lib.c:909-957,
// c/mfista_fft_lib.c:701-756, c/mfista_dft_lib.c:540-589); the iteration
// itself runs on the GPU through mf::Solver.
#include <time.h>

#include <mutex>

#include "solver.cuh"
#include "looe.cuh"
#include "cpp_nufft.cuh"

using namespace mf;

namespace {

thread_local int g_status = 0;
thread_local std::string g_msg;
thread_local int g_fgp_iter = 100;  // FGPITER, c/mfista.h:38

void set_ok() {
  g_status = MFISTA_OK;
  g_msg.clear();
  cudaGetLastError();  // do not inherit a launch error of an earlier call
}

int fail(int st, const std::string& m, bool print) {
  g_status = st;
  g_msg = m;
  if (print) printf("mfista_b200: %s\n", m.c_str());
  return st;
}

bool quiet() {
  const char* q = getenv("MFISTA_QUIET");
  return q && q[0] == '1';
}

double now_s() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

// result summary fields common to the three variants (calc_result_*)
void fill_result(RESULT* r, const FinalOut& o, int m_report, double m_div, int nx, int ny, int n, double l1,
                 double ltv, double ltsv, int maxiter, int nonneg, double comp_time, bool skipped, double cinit) {
  r->M = m_report;
  r->N = n;
  r->NX = nx;
  r->NY = ny;
  r->lambda_l1 = l1;
  r->lambda_tv = ltv;
  r->lambda_tsv = ltsv;
  r->sq_error = o.sq_error;
  r->mean_sq_error = o.sq_error / m_div;
  r->l1cost = o.l1cost;
  r->N_active = (int)llround(o.n_active);
  r->finalcost = o.finalcost;
  if (ltsv > 0) r->tsvcost = o.regcost;
  else if (ltv > 0) r->tvcost = o.regcost;
  r->comp_time = comp_time;
  r->ITER = skipped ? 0 : o.iters;
  r->nonneg = nonneg;
  r->Lip_const = skipped ? cinit : o.lip;
  r->maxiter = maxiter;
}

template <typename MakeOp>
void run_single(MakeOp make_op, int N, int NX, int NY, int form, const float* box, const ProbParams& p,
                const double* x0, bool skip, double* xout, FinalOut& out, double& comp_time) {
  Solver S;
  S.precision = MFISTA_FP64;
  S.init_common(1, N, NX, NY, form, g_fgp_iter, box);
  S.op.reset(make_op(S.ctx));
  S.finish_setup();
  double t0 = now_s();
  S.upload_problems({p}, x0);
  S.enqueue_solve(skip);
  std::vector<FinalOut> o;
  S.fetch(xout, o);
  comp_time = now_s() - t0;
  out = o[0];
}

// Solvers of the NUFFT drop-in entry kept between calls.  A driver that
// calls mfista_imaging_core_nufft repeatedly on one uv coverage (a lambda
// sweep, a series of epochs) would otherwise rebuild the operator (point
// binning, device buffers, FFT tables) and capture the solve graph on every
// call.  An entry is keyed by everything that shapes the device data except
// the visibilities: sizes, regulariser form, FGP iterations, device, and the
// contents of u, v, vis_std and the box mask (compared exactly); a hit
// uploads vis_r / vis_i and runs the captured graph.  At most
// kDropinEntries are kept (least recently used out); a call that finds its
// entry busy (another thread) builds a solver of its own.
// MFISTA_DROPIN_CACHE=0 turns the cache off; mfista_release_cache() frees it.
struct DropinNufft {
  int M = 0, Nx = 0, Ny = 0, form = 0, fgp = 0, device = 0, box = 0;
  std::vector<double> u, v, s;
  std::vector<float> cbox;
  std::unique_ptr<Solver> S;
  NufftOp<double>* op = nullptr;
  bool busy = false;
  bool stale = false;  // its device memory is gone (a reset): never reused, evicted first
  unsigned long long used = 0;
};
constexpr size_t kDropinEntries = 4;
std::mutex g_dropin_mu;
// never destroyed: at process exit the CUDA runtime may already be gone
std::vector<std::unique_ptr<DropinNufft>>& g_dropin = *new std::vector<std::unique_ptr<DropinNufft>>();
unsigned long long g_dropin_clock = 0;

bool dropin_cache_on() {
  const char* c = getenv("MFISTA_DROPIN_CACHE");
  return !(c && c[0] == '0');
}

// the cached solver matching the call, marked busy, or null
DropinNufft* dropin_find(const double* u, const double* v, const double* s, int M, int Nx, int Ny, int form,
                         const float* box, int device) {
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  const size_t nb = box ? (size_t)Nx * Ny : 0;
  for (auto& e : g_dropin) {
    if (e->busy || e->stale || e->M != M || e->Nx != Nx || e->Ny != Ny || e->form != form || e->fgp != g_fgp_iter ||
        e->device != device || e->box != (box ? 1 : 0))
      continue;
    if (memcmp(e->u.data(), u, sizeof(double) * M) || memcmp(e->v.data(), v, sizeof(double) * M) ||
        memcmp(e->s.data(), s, sizeof(double) * M) || (nb && memcmp(e->cbox.data(), box, sizeof(float) * nb)))
      continue;
    // a kept solver whose buffers no longer exist (cudaDeviceReset since)
    // is dropped, not reused
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, e->op->d_vr.p) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      e->stale = true;
      continue;
    }
    e->busy = true;
    e->used = ++g_dropin_clock;
    return e.get();
  }
  return nullptr;
}

// hands a solver back (kept = false: it failed and is dropped)
void dropin_return(DropinNufft* e, bool fresh, bool kept) {
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  if (!fresh) {
    if (kept) {
      e->busy = false;
    } else {
      for (size_t i = 0; i < g_dropin.size(); ++i)
        if (g_dropin[i].get() == e) {
          g_dropin.erase(g_dropin.begin() + i);
          break;
        }
    }
    return;
  }
  std::unique_ptr<DropinNufft> own(e);
  if (!kept) return;
  own->busy = false;
  own->used = ++g_dropin_clock;
  while (g_dropin.size() >= kDropinEntries) {  // least recently used, not busy
    size_t victim = g_dropin.size();
    for (size_t i = 0; i < g_dropin.size(); ++i)
      if (!g_dropin[i]->busy && (victim == g_dropin.size() || g_dropin[i]->stale ||
                                 (!g_dropin[victim]->stale && g_dropin[i]->used < g_dropin[victim]->used)))
        victim = i;
    if (victim == g_dropin.size()) return;  // all busy: do not keep this one
    if (g_dropin[victim]->stale) (void)g_dropin[victim].release();  // see mfista_release_cache
    g_dropin.erase(g_dropin.begin() + victim);
  }
  g_dropin.push_back(std::move(own));
}

}  // namespace

extern "C" void mfista_release_cache(void) {
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  for (size_t i = 0; i < g_dropin.size();) {
    if (g_dropin[i]->busy) {
      ++i;
      continue;
    }
    // a stale solver (its context reset under it) is left alone rather than
    // destroyed: its addresses may belong to new allocations by now
    if (g_dropin[i]->stale) (void)g_dropin[i].release();
    g_dropin.erase(g_dropin.begin() + i);
  }
}

extern "C" int mfista_last_status(void) { return g_status; }
extern "C" int mfista_set_device(int device) {
  set_ok();
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(MFISTA_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e), false);
  return MFISTA_OK;
}
extern "C" int mfista_set_fgp_iter(int n) {
  if (n < 1) return -1;
  int old = g_fgp_iter;
  g_fgp_iter = n;
  return old;
}
extern "C" const char* mfista_last_error(void) { return g_msg.c_str(); }

// ---------------------------------------------------------------------------
// drop-in entry points
// ---------------------------------------------------------------------------
extern "C" void mfista_imaging_core_nufft(double* u_dx, double* v_dy, double* vis_r, double* vis_i,
                                          double* vis_std, int M, int Nx, int Ny, int maxiter, double eps,
                                          double lambda_l1, double lambda_tv, double lambda_tsv, double cinit,
                                          double* xinit, double* xout, int nonneg_flag, int box_flag,
                                          float* cl_box, struct RESULT* mfista_result) {
  set_ok();
  // epsilon = eps * sum|vis|^2 / M  (:923-926)
  double sr = 0, si = 0;
  for (int i = 0; i < M; ++i) sr += vis_r[i] * vis_r[i];
  for (int i = 0; i < M; ++i) si += vis_i[i] * vis_i[i];
  double epsilon = sr + si;
  epsilon *= eps / ((double)M);
  int form;
  if (lambda_tv == 0) form = kFormTSV;
  else if (lambda_tsv == 0) form = kFormTV;
  else {
    printf("You cannot set both of lambda_TV and lambda_TSV positive.\n");
    fail(MFISTA_ERR_BOTH_REG, "lambda_tv and lambda_tsv both non-zero", false);
    return;
  }
  if (maxiter < 0) {
    fail(MFISTA_ERR_ARG, "maxiter must be >= 0", true);
    return;
  }
  bool skip = form == kFormTSV && nonneg_flag != 0 && nonneg_flag != 1;
  if (!quiet()) {
    printf("computing image with MFISTA with NUFFT.\n");
    printf("stop if iter = %d, or Delta_cost < %e\n", maxiter, epsilon);
    if (skip) printf("nonneg_flag must be chosen properly.\n");
  }
  DropinNufft* E = nullptr;
  bool fresh = false;
  try {
    ProbParams p{lambda_l1, lambda_tv, lambda_tsv, cinit, epsilon, maxiter, nonneg_flag, box_flag, 0, 0.0};
    NufftInput in{u_dx, v_dy, vis_r, vis_i, vis_std, nullptr, 1, M, Nx, Ny};
    FinalOut o;
    double ct;
    std::vector<double> xo(skip ? xout : xinit, (skip ? xout : xinit) + (size_t)Nx * Ny);
    const float* box = box_flag == 1 ? cl_box : nullptr;
    if (skip || !dropin_cache_on() || M < 1) {
      run_single([&](Ctx& c) { return new NufftOp<double>(c, in); }, Nx * Ny, Nx, Ny, form, box, p, xo.data(), skip,
                 xo.data(), o, ct);
    } else {
      int dev = 0;
      MF_CK(cudaGetDevice(&dev));
      E = dropin_find(u_dx, v_dy, vis_std, M, Nx, Ny, form, box, dev);
      if (E) {  // same geometry: new visibilities into the kept operator
        MF_CK(cudaMemcpy(E->op->d_vr.p, vis_r, sizeof(double) * M, cudaMemcpyHostToDevice));
        MF_CK(cudaMemcpy(E->op->d_vi.p, vis_i, sizeof(double) * M, cudaMemcpyHostToDevice));
      } else {
        fresh = true;
        E = new DropinNufft;
        E->M = M;
        E->Nx = Nx;
        E->Ny = Ny;
        E->form = form;
        E->fgp = g_fgp_iter;
        E->device = dev;
        E->box = box ? 1 : 0;
        E->u.assign(u_dx, u_dx + M);
        E->v.assign(v_dy, v_dy + M);
        E->s.assign(vis_std, vis_std + M);
        if (box) E->cbox.assign(box, box + (size_t)Nx * Ny);
        E->busy = true;
        E->S.reset(new Solver);
        E->S->precision = MFISTA_FP64;
        E->S->init_common(1, Nx * Ny, Nx, Ny, form, g_fgp_iter, box);
        E->op = new NufftOp<double>(E->S->ctx, in);
        E->S->op.reset(E->op);
        E->S->finish_setup();
      }
      const double t0 = now_s();
      E->S->upload_problems({p}, xo.data());
      E->S->enqueue_solve(false);
      std::vector<FinalOut> ov;
      E->S->fetch(xo.data(), ov);
      ct = now_s() - t0;
      o = ov[0];
      dropin_return(E, fresh, o.status == 0);
      E = nullptr;
    }
    memcpy(xout, xo.data(), sizeof(double) * (size_t)Nx * Ny);
    fill_result(mfista_result, o, M / 2, (double)M, Nx, Ny, Nx * Ny, lambda_l1, lambda_tv, lambda_tsv, maxiter,
                nonneg_flag, ct, skip, cinit);
    if (o.status) fail(o.status, "solver stopped early (status " + std::to_string(o.status) + ")", !quiet());
  } catch (const Error& e) {
    if (E) dropin_return(E, fresh, false);
    fail(e.status, e.what(), true);
  }
}

extern "C" void mfista_imaging_core_fft(int* u_idx, int* v_idx, double* y_r, double* y_i, double* noise_stdev,
                                        int M, int NX, int NY, int maxiter, double eps, double lambda_l1,
                                        double lambda_tv, double lambda_tsv, double cinit, double* xinit,
                                        double* xout, int nonneg_flag, unsigned int fftw_plan_flag, int box_flag,
                                        float* cl_box, struct RESULT* mfista_result) {
  (void)fftw_plan_flag;
  set_ok();
  double epsilon = 0;  // (:715-717)
  for (int i = 0; i < M; ++i) epsilon += y_r[i] * y_r[i] + y_i[i] * y_i[i];
  epsilon *= eps / ((double)M);
  int form;
  if (lambda_tv == 0) form = kFormTSV;
  else if (lambda_tsv == 0) form = kFormTV;
  else {
    printf("You cannot set both of lambda_TV and lambda_TSV positive.\n");
    fail(MFISTA_ERR_BOTH_REG, "lambda_tv and lambda_tsv both non-zero", false);
    return;
  }
  if (maxiter < 0) {
    fail(MFISTA_ERR_ARG, "maxiter must be >= 0", true);
    return;
  }
  bool skip = form == kFormTSV && nonneg_flag != 0 && nonneg_flag != 1;
  if (!quiet()) {
    printf("computing image with MFISTA.\n");
    printf("stop if iter = %d, or Delta_cost < %e\n", maxiter, epsilon);
    if (skip) printf("nonneg_flag must be chosen properly.\n");
  }
  try {
    ProbParams p{lambda_l1, lambda_tv, lambda_tsv, cinit, epsilon, maxiter, nonneg_flag, box_flag, 0, 0.0};
    FftVarInput in{u_idx, v_idx, y_r, y_i, noise_stdev, M, NX, NY};
    FinalOut o;
    double ct;
    std::vector<double> xo(skip ? xout : xinit, (skip ? xout : xinit) + (size_t)NX * NY);
    run_single([&](Ctx& c) { return new FftVarOp<double>(c, in); }, NX * NY, NX, NY, form,
               box_flag == 1 ? cl_box : nullptr, p, xo.data(), skip, xo.data(), o, ct);
    memcpy(xout, xo.data(), sizeof(double) * (size_t)NX * NY);
    fill_result(mfista_result, o, M / 2, (double)M, NX, NY, NX * NY, lambda_l1, lambda_tv, lambda_tsv, maxiter,
                nonneg_flag, ct, skip, cinit);
    if (o.status) fail(o.status, "solver stopped early (status " + std::to_string(o.status) + ")", !quiet());
  } catch (const Error& e) {
    fail(e.status, e.what(), true);
  }
}

extern "C" void mfista_imaging_core_dft(double* y, double* A, int* M, int* N, int NX, int NY, int maxiter,
                                        double eps, double lambda_l1, double lambda_tv, double lambda_tsv,
                                        double cinit, double* xinit, double* xout, int nonneg_flag, int looe_flag,
                                        int box_flag, float* cl_box, struct RESULT* mfista_result) {
  (void)looe_flag;
  set_ok();
  int m = *M, n = *N;
  memcpy(xout, xinit, sizeof(double) * (size_t)n);  // (:552)
  int form;
  if (lambda_tv == 0) form = kFormTSV;
  else if (lambda_tsv == 0) form = kFormTV;
  else {
    printf("You cannot set both of lambda_TV and lambda_TSV positive.\n");
    fail(MFISTA_ERR_BOTH_REG, "lambda_tv and lambda_tsv both non-zero", false);
    return;
  }
  if (maxiter < 0) {
    fail(MFISTA_ERR_ARG, "maxiter must be >= 0", true);
    return;
  }
  bool skip = form == kFormTSV && nonneg_flag != 0 && nonneg_flag != 1;
  if (!quiet()) {
    printf("computing image with MFISTA.\n");
    if (skip) printf("nonneg_flag must be chosen properly.\n");
  }
  try {
    ProbParams p{lambda_l1, lambda_tv, lambda_tsv, cinit, eps, maxiter, nonneg_flag, box_flag, 0, 0.0};
    FinalOut o;
    Solver S;
    S.precision = MFISTA_FP64;
    S.init_common(1, n, NX, NY, form, g_fgp_iter, box_flag == 1 ? cl_box : nullptr);
    DftOp* op = new DftOp(S.ctx, A, y, m, n);
    S.op.reset(op);
    S.finish_setup();
    double t0 = now_s();
    S.upload_problems({p}, xout);
    S.enqueue_solve(skip);
    std::vector<FinalOut> outs;
    std::vector<double> xo(n);
    S.fetch(xo.data(), outs);
    double ct = now_s() - t0;
    o = outs[0];
    memcpy(xout, xo.data(), sizeof(double) * (size_t)n);
    if (!quiet()) printf("summarizing result.\n");
    fill_result(mfista_result, o, m, (double)m, NX, NY, n, lambda_l1, lambda_tv, lambda_tsv, maxiter, nonneg_flag, ct,
                skip, cinit);
    // residual y - A x, owned by the caller (:454)
    mfista_result->residual = (double*)malloc(sizeof(double) * (size_t)std::max(m, 1));
    MF_CK(cudaMemcpy(mfista_result->residual, op->g.resid, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost));
    if (o.status) fail(o.status, "solver stopped early (status " + std::to_string(o.status) + ")", !quiet());
  } catch (const Error& e) {
    fail(e.status, e.what(), true);
  }
}

// ---------------------------------------------------------------------------
// batched plan
// ---------------------------------------------------------------------------
struct mfista_plan_s {
  std::unique_ptr<Solver> S;
  int B = 0, Nx = 0, Ny = 0;
  int form = kFormTSV;
  std::vector<int> m_of;         // points per problem
  std::vector<double> energy;    // sum |vis|^2 per problem
  std::vector<ProbParams> prm;
  double comp_time = 0, t_start = 0;
  int launches = 0;
  std::vector<int> statuses;
};

extern "C" mfista_plan mfista_nufft_plan_create(const double* u_dx, const double* v_dy, const double* vis_r,
                                                const double* vis_i, const double* vis_std, const int* pt_off,
                                                int shared_geometry, int M, int Nx, int Ny, int B, int precision,
                                                int form_tv, int fgp_iter) {
  set_ok();
  try {
    if (B < 1) throw Error(MFISTA_ERR_ARG, "B must be >= 1");
    if (precision != MFISTA_FP32 && precision != MFISTA_FP64) throw Error(MFISTA_ERR_ARG, "precision must be 32 or 64");
    if (!shared_geometry && !pt_off) throw Error(MFISTA_ERR_ARG, "pt_off required without shared geometry");
    if (!shared_geometry) {
      if (pt_off[0] < 0) throw Error(MFISTA_ERR_ARG, "pt_off[0] must be >= 0");
      for (int b = 0; b < B; ++b)
        if (pt_off[b + 1] < pt_off[b]) throw Error(MFISTA_ERR_ARG, "pt_off must not decrease");
      // M > 0 is the length of the concatenated point arrays
      if (M > 0 && pt_off[B] > M) throw Error(MFISTA_ERR_ARG, "pt_off[B] exceeds M, the length of the point arrays");
    }
    std::unique_ptr<mfista_plan_s> P(new mfista_plan_s);
    P->B = B;
    P->Nx = Nx;
    P->Ny = Ny;
    P->form = form_tv ? kFormTV : kFormTSV;
    P->S.reset(new Solver);
    Solver& S = *P->S;
    S.precision = precision;
    S.init_common(B, Nx * Ny, Nx, Ny, P->form, fgp_iter, nullptr);
    NufftInput in{u_dx, v_dy, vis_r, vis_i, vis_std, pt_off, shared_geometry, M, Nx, Ny};
    // FP32 operators carry an FP64 defect correction unless disabled
    const char* nc = getenv("MFISTA_FP32_NO_CORRECTION");
    bool correct = !(nc && nc[0] == '1');
    if (precision == MFISTA_FP32) S.op.reset(new NufftOp<float>(S.ctx, in, correct));
    else S.op.reset(new NufftOp<double>(S.ctx, in));
    S.finish_setup();
    P->m_of.resize(B);
    P->energy.resize(B);
    for (int b = 0; b < B; ++b) {
      int lo = shared_geometry ? 0 : pt_off[b];
      int hi = shared_geometry ? M : pt_off[b + 1];
      double sr = 0, si = 0;
      for (int i = lo; i < hi; ++i) sr += vis_r[i] * vis_r[i];
      for (int i = lo; i < hi; ++i) si += vis_i[i] * vis_i[i];
      P->m_of[b] = hi - lo;
      P->energy[b] = sr + si;
    }
    return P.release();
  } catch (const Error& e) {
    fail(e.status, e.what(), false);
    return nullptr;
  }
}

extern "C" int mfista_plan_set_problems(mfista_plan P, const struct mfista_problem* problems, double eps,
                                        const double* xinit) {
  set_ok();
  if (!P) return fail(MFISTA_ERR_ARG, "null plan", false);
  try {
    P->prm.resize(P->B);
    for (int b = 0; b < P->B; ++b) {
      const mfista_problem& q = problems[b];
      if (q.lambda_tv != 0 && q.lambda_tsv != 0) throw Error(MFISTA_ERR_BOTH_REG, "lambda_tv and lambda_tsv both non-zero");
      if ((P->form == kFormTV) != (q.lambda_tv != 0))
        throw Error(MFISTA_ERR_ARG, "problem regulariser does not match the plan (TV vs TSV)");
      if (P->form == kFormTSV && q.nonneg_flag != 0 && q.nonneg_flag != 1)
        throw Error(MFISTA_ERR_ARG, "nonneg_flag must be 0 or 1");
      if (q.maxiter < 0) throw Error(MFISTA_ERR_ARG, "maxiter must be >= 0");
      double epsilon = P->energy[b];
      epsilon *= eps / ((double)P->m_of[b]);
      P->prm[b] = ProbParams{q.lambda_l1, q.lambda_tv, q.lambda_tsv, q.cinit, epsilon, q.maxiter, q.nonneg_flag, 0, 0, q.target_cost};
    }
    P->S->upload_problems(P->prm, xinit);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_plan_run(mfista_plan P) {
  set_ok();
  if (!P) return fail(MFISTA_ERR_ARG, "null plan", false);
  try {
    P->t_start = now_s();
    P->S->steps_host[0] = 0;
    P->S->steps_host[2] = 0;
    MF_CK(cudaMemcpyAsync(P->S->d_steps.p, P->S->steps_host, sizeof(P->S->steps_host), cudaMemcpyHostToDevice,
                          P->S->stream));
    P->S->enqueue_solve(false);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_plan_fetch(mfista_plan P, double* xout, struct RESULT* results) {
  set_ok();
  if (!P) return fail(MFISTA_ERR_ARG, "null plan", false);
  try {
    std::vector<FinalOut> o;
    P->S->fetch(xout, o);
    P->comp_time = now_s() - P->t_start;
    P->launches = (int)(P->S->fixed_launches + P->S->loop_launches());
    int worst = 0;
    P->statuses.assign(P->B, 0);
    for (int b = 0; b < P->B; ++b) {
      P->statuses[b] = o[b].status;
      const ProbParams& p = P->prm[b];
      if (results)
        fill_result(&results[b], o[b], P->m_of[b] / 2, (double)P->m_of[b], P->Nx, P->Ny, P->Nx * P->Ny, p.lambda_l1,
                    p.lambda_tv, p.lambda_tsv, p.maxiter, p.nonneg, P->comp_time, false, p.cinit);
      if (results) results[b].residual = nullptr;
      if (o[b].status) worst = o[b].status;
    }
    if (worst) return fail(worst, "a problem stopped early (status " + std::to_string(worst) + ")", false);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" void* mfista_plan_stream(mfista_plan P) { return P ? (void*)P->S->stream : nullptr; }

extern "C" int mfista_plan_profile(mfista_plan P, int kernel, int reps, double* ms_per_launch,
                                   double* bytes_per_launch) {
  set_ok();
  if (!P) return fail(MFISTA_ERR_ARG, "null plan", false);
  try {
    double ms = 0, bytes = 0;
    P->S->profile_kernel(kernel, std::max(1, reps), ms, bytes);
    if (ms_per_launch) *ms_per_launch = ms;
    if (bytes_per_launch) *bytes_per_launch = bytes;
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}
extern "C" int mfista_plan_get_shapes(mfista_plan P, int* shapes) {
  set_ok();
  if (!P || !shapes) return fail(MFISTA_ERR_ARG, "null argument", false);
  LaunchShapes sh = P->S->op->shapes();
  shapes[0] = sh.interp_ppw;
  shapes[1] = sh.spread_cluster;
  shapes[2] = sh.rows_per_cta;
  shapes[3] = sh.cols_per_cta;
  return MFISTA_OK;
}

extern "C" int mfista_plan_set_shapes(mfista_plan P, const int* shapes) {
  set_ok();
  if (!P || !shapes) return fail(MFISTA_ERR_ARG, "null argument", false);
  try {
    LaunchShapes sh;
    sh.interp_ppw = shapes[0];
    sh.spread_cluster = shapes[1];
    sh.rows_per_cta = shapes[2];
    sh.cols_per_cta = shapes[3];
    if (sh.spread_cluster && P->S->op->shapes().spread_cluster && !P->S->spread_cluster_fits(sh.spread_cluster))
      throw Error(MFISTA_ERR_ARG, "spread cluster of " + std::to_string(sh.spread_cluster) + " CTAs cannot be resident");
    P->S->apply_shapes(sh);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_plan_tune(mfista_plan P, int reps, int* shapes_out, double* ms_out) {
  set_ok();
  if (!P) return fail(MFISTA_ERR_ARG, "null plan", false);
  try {
    double ms[4] = {0, 0, 0, 0};
    LaunchShapes sh = P->S->tune(std::max(1, reps), ms);
    if (shapes_out) {
      shapes_out[0] = sh.interp_ppw;
      shapes_out[1] = sh.spread_cluster;
      shapes_out[2] = sh.rows_per_cta;
      shapes_out[3] = sh.cols_per_cta;
    }
    if (ms_out)
      for (int k = 0; k < 4; ++k) ms_out[k] = ms[k];
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_plan_kernel_launches(mfista_plan P) { return P ? P->launches : 0; }
extern "C" int mfista_plan_statuses(mfista_plan P, int* status_out) {
  if (!P) return MFISTA_ERR_ARG;
  for (int b = 0; b < P->B; ++b) status_out[b] = b < (int)P->statuses.size() ? P->statuses[b] : 0;
  return MFISTA_OK;
}
extern "C" int mfista_plan_device_loop(mfista_plan P) { return P && !P->S->host_loop ? 1 : 0; }
extern "C" void mfista_plan_destroy(mfista_plan P) { delete P; }

extern "C" int mfista_nufft_batch(const double* u_dx, const double* v_dy, const double* vis_r, const double* vis_i,
                                  const double* vis_std, const int* pt_off, int shared_geometry, int M, int Nx, int Ny,
                                  int B, const struct mfista_problem* problems, double eps, int precision,
                                  int fgp_iter, const double* xinit, double* xout, struct RESULT* results) {
  int form_tv = B > 0 && problems[0].lambda_tv != 0;
  mfista_plan P = mfista_nufft_plan_create(u_dx, v_dy, vis_r, vis_i, vis_std, pt_off, shared_geometry, M, Nx, Ny, B,
                                           precision, form_tv, fgp_iter);
  if (!P) return g_status;
  int st = mfista_plan_set_problems(P, problems, eps, xinit);
  if (st == MFISTA_OK) st = mfista_plan_run(P);
  if (st == MFISTA_OK) st = mfista_plan_fetch(P, xout, results);
  int keep = g_status;
  std::string msg = g_msg;
  mfista_plan_destroy(P);
  g_status = keep;
  g_msg = msg;
  return st;
}

extern "C" int mfista_dft_batch(const double* y, const double* A, int M, int N, int NX, int NY, int B,
                                const struct mfista_problem* problems, double eps, int precision, int fgp_iter,
                                const double* xinit, double* xout, struct RESULT* results) {
  set_ok();
  try {
    if (B < 1) throw Error(MFISTA_ERR_ARG, "B must be >= 1");
    if (precision != MFISTA_FP64 && precision != MFISTA_BF16X3 && precision != MFISTA_BF16X6)
      throw Error(MFISTA_ERR_ARG, "the batched DFT runs in FP64, BF16X3 or BF16X6");
    int form = problems[0].lambda_tv != 0 ? kFormTV : kFormTSV;
    std::vector<ProbParams> prm(B);
    for (int b = 0; b < B; ++b) {
      const mfista_problem& q = problems[b];
      if (q.lambda_tv != 0 && q.lambda_tsv != 0) throw Error(MFISTA_ERR_BOTH_REG, "lambda_tv and lambda_tsv both non-zero");
      if ((form == kFormTV) != (q.lambda_tv != 0)) throw Error(MFISTA_ERR_ARG, "mixed TV / TSV problems");
      if (form == kFormTSV && q.nonneg_flag != 0 && q.nonneg_flag != 1)
        throw Error(MFISTA_ERR_ARG, "nonneg_flag must be 0 or 1");
      if (q.maxiter < 0) throw Error(MFISTA_ERR_ARG, "maxiter must be >= 0");
      prm[b] = ProbParams{q.lambda_l1, q.lambda_tv, q.lambda_tsv, q.cinit, eps, q.maxiter, q.nonneg_flag, 0, 0,
                          q.target_cost};
    }
    Solver S;
    S.precision = MFISTA_FP64;
    S.init_common(B, N, NX, NY, form, fgp_iter, nullptr);
    S.op.reset(new DftOp(S.ctx, A, y, M, N, precision));
    S.finish_setup();
    double t0 = now_s();
    S.upload_problems(prm, xinit);
    S.enqueue_solve(false);
    std::vector<FinalOut> o;
    S.fetch(xout, o);
    if (S.op->device_error()) throw Error(MFISTA_ERR_CUDA, "a tensor-core GEMM wait timed out");
    double ct = now_s() - t0;
    int worst = 0;
    for (int b = 0; b < B; ++b) {
      if (results) {
        fill_result(&results[b], o[b], M, (double)M, NX, NY, N, prm[b].lambda_l1, prm[b].lambda_tv,
                    prm[b].lambda_tsv, prm[b].maxiter, prm[b].nonneg, ct, false, prm[b].cinit);
        results[b].residual = nullptr;
      }
      if (o[b].status) worst = o[b].status;
    }
    if (worst) return fail(worst, "a problem stopped early (status " + std::to_string(worst) + ")", false);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_fft_batch(const int* u_idx, const int* v_idx, const double* y_r, const double* y_i,
                                const double* noise_stdev, int M, int NX, int NY, int B,
                                const struct mfista_problem* problems, double eps, int precision, int fgp_iter,
                                const double* xinit, double* xout, struct RESULT* results) {
  set_ok();
  try {
    if (B < 1 || M < 1) throw Error(MFISTA_ERR_ARG, "B and M must be >= 1");
    if (!u_idx || !v_idx || !y_r || !y_i || !noise_stdev || !problems || !xout)
      throw Error(MFISTA_ERR_ARG, "mfista_fft_batch: null pointer");
    if (precision != MFISTA_FP64 && precision != MFISTA_FP32)
      throw Error(MFISTA_ERR_ARG, "the batched FFT variant runs in FP64 or FP32");
    if (fgp_iter < 1) throw Error(MFISTA_ERR_ARG, "fgp_iter must be >= 1");
    // epsilon scaled as mfista_imaging_core_fft does (c/mfista_fft_lib.c:715-717)
    double energy = 0;
    for (int i = 0; i < M; ++i) energy += y_r[i] * y_r[i] + y_i[i] * y_i[i];
    const double epsilon = energy * (eps / ((double)M));
    int form = problems[0].lambda_tv != 0 ? kFormTV : kFormTSV;
    std::vector<ProbParams> prm(B);
    for (int b = 0; b < B; ++b) {
      const mfista_problem& q = problems[b];
      if (q.lambda_tv != 0 && q.lambda_tsv != 0) throw Error(MFISTA_ERR_BOTH_REG, "lambda_tv and lambda_tsv both non-zero");
      if ((form == kFormTV) != (q.lambda_tv != 0)) throw Error(MFISTA_ERR_ARG, "mixed TV / TSV problems");
      if (form == kFormTSV && q.nonneg_flag != 0 && q.nonneg_flag != 1)
        throw Error(MFISTA_ERR_ARG, "nonneg_flag must be 0 or 1");
      if (q.maxiter < 0) throw Error(MFISTA_ERR_ARG, "maxiter must be >= 0");
      prm[b] = ProbParams{q.lambda_l1, q.lambda_tv, q.lambda_tsv, q.cinit, epsilon, q.maxiter, q.nonneg_flag, 0, 0,
                          q.target_cost};
    }
    Solver S;
    S.precision = precision;
    S.init_common(B, NX * NY, NX, NY, form, fgp_iter, nullptr);
    FftVarInput in{u_idx, v_idx, y_r, y_i, noise_stdev, M, NX, NY};
    if (precision == MFISTA_FP32) S.op.reset(new FftVarOp<float>(S.ctx, in, true));
    else S.op.reset(new FftVarOp<double>(S.ctx, in));
    S.finish_setup();
    double t0 = now_s();
    S.upload_problems(prm, xinit);
    S.enqueue_solve(false);
    std::vector<FinalOut> o;
    S.fetch(xout, o);
    double ct = now_s() - t0;
    int worst = 0;
    for (int b = 0; b < B; ++b) {
      if (results) {
        fill_result(&results[b], o[b], M / 2, (double)M, NX, NY, NX * NY, prm[b].lambda_l1, prm[b].lambda_tv,
                    prm[b].lambda_tsv, prm[b].maxiter, prm[b].nonneg, ct, false, prm[b].cinit);
        results[b].residual = nullptr;
      }
      if (o[b].status) worst = o[b].status;
    }
    if (worst) return fail(worst, "a problem stopped early (status " + std::to_string(worst) + ")", false);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

// ---------------------------------------------------------------------------
// operator-level entry points
// ---------------------------------------------------------------------------
namespace {

template <typename T>
int nufft_apply(const double* u, const double* v, const double* wstd, int M, int Nx, int Ny, const double* x,
                const double* r_r, const double* r_i, double* out_r, double* out_i, double* x_out) {
  Solver S;
  S.precision = sizeof(T) == 4 ? MFISTA_FP32 : MFISTA_FP64;
  S.init_common(1, Nx * Ny, Nx, Ny, kFormTSV, 100, nullptr);
  std::vector<double> zero(std::max(M, 1), 0.0), one(std::max(M, 1), 1.0);
  NufftInput in{u, v, zero.data(), zero.data(), wstd ? wstd : one.data(), nullptr, 1, M, Nx, Ny};
  NufftOp<T>* op = new NufftOp<T>(S.ctx, in);
  S.op.reset(op);
  int slots = std::max({op->chi_slots(), op->tsv_slots(), 1});
  S.d_part.alloc(sizeof(double) * (size_t)kNumQ * slots);
  S.ctx.part.p = S.d_part.as<double>();
  S.ctx.part.slots = slots;
  S.ctx.part.B = 1;
  ProbState st;
  memset(&st, 0, sizeof(st));
  st.active = 1;
  st.need_grad = 1;
  MF_CK(cudaMemcpyAsync(S.ctx.st, &st, sizeof(st), cudaMemcpyHostToDevice, S.stream));
  ProbParams p;
  memset(&p, 0, sizeof(p));
  MF_CK(cudaMemcpyAsync(S.ctx.prm, &p, sizeof(p), cudaMemcpyHostToDevice, S.stream));
  if (x) {
    MF_CK(cudaMemcpyAsync(S.ctx.x, x, sizeof(double) * (size_t)Nx * Ny, cudaMemcpyHostToDevice, S.stream));
    op->forward(S.stream, S.ctx.x, kGateAll, kQChiX, true);
    std::vector<cplx<T>> y2(std::max(M, 1));
    MF_CK(cudaMemcpyAsync(y2.data(), op->d_y2.p, sizeof(cplx<T>) * (size_t)M, cudaMemcpyDeviceToHost, S.stream));
    MF_CK(cudaStreamSynchronize(S.stream));
    // the residual kernel stored (0 - A x) * w * w with w = 1
    for (int k = 0; k < M; ++k) {
      out_r[k] = -(double)y2[k].x;
      out_i[k] = -(double)y2[k].y;
    }
  } else {
    std::vector<cplx<T>> y2(std::max(M, 1));
    for (int k = 0; k < M; ++k) y2[k] = mk<T>((T)r_r[k], (T)r_i[k]);
    MF_CK(cudaMemcpyAsync(op->d_y2.p, y2.data(), sizeof(cplx<T>) * (size_t)M, cudaMemcpyHostToDevice, S.stream));
    op->adjoint(S.stream, nullptr, -1);
    MF_CK(cudaMemcpyAsync(x_out, S.ctx.dfdx, sizeof(double) * (size_t)Nx * Ny, cudaMemcpyDeviceToHost, S.stream));
    MF_CK(cudaStreamSynchronize(S.stream));
  }
  return MFISTA_OK;
}

}  // namespace

extern "C" int mfista_nufft_forward(const double* u_dx, const double* v_dy, int M, int Nx, int Ny, const double* x,
                                    double* out_r, double* out_i, int precision) {
  set_ok();
  try {
    if (precision == MFISTA_FP32)
      return nufft_apply<float>(u_dx, v_dy, nullptr, M, Nx, Ny, x, nullptr, nullptr, out_r, out_i, nullptr);
    return nufft_apply<double>(u_dx, v_dy, nullptr, M, Nx, Ny, x, nullptr, nullptr, out_r, out_i, nullptr);
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_nufft_adjoint(const double* u_dx, const double* v_dy, int M, int Nx, int Ny, const double* r_r,
                                    const double* r_i, double* x_out, int precision) {
  set_ok();
  try {
    if (precision == MFISTA_FP32)
      return nufft_apply<float>(u_dx, v_dy, nullptr, M, Nx, Ny, nullptr, r_r, r_i, nullptr, nullptr, x_out);
    return nufft_apply<double>(u_dx, v_dy, nullptr, M, Nx, Ny, nullptr, r_r, r_i, nullptr, nullptr, x_out);
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_dft_apply(const double* A, int M, int N, const double* X, int B, int transpose, int precision,
                                double* out) {
  set_ok();
  try {
    if (M < 1 || N < 1 || B < 1 || !A || !X || !out) throw Error(MFISTA_ERR_ARG, "bad sizes or null pointer");
    Solver S;
    S.precision = MFISTA_FP64;
    S.init_common(B, N, N, 1, kFormTSV, 100, nullptr);
    std::vector<double> y(M, 0.0);
    DftOp* op = new DftOp(S.ctx, A, y.data(), M, N, precision);
    S.op.reset(op);
    int slots = std::max({op->chi_slots(), op->tsv_slots(), 1});
    S.d_part.alloc(sizeof(double) * (size_t)kNumQ * B * slots);
    S.ctx.part.p = S.d_part.as<double>();
    S.ctx.part.slots = slots;
    S.ctx.part.B = B;
    std::vector<ProbState> st(B);
    for (ProbState& q : st) {
      memset(&q, 0, sizeof(q));
      q.active = 1;
      q.need_grad = 1;
    }
    MF_CK(cudaMemcpyAsync(S.ctx.st, st.data(), sizeof(ProbState) * B, cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemsetAsync(S.ctx.prm, 0, sizeof(ProbParams) * B, S.stream));
    MF_CK(cudaMemsetAsync(S.ctx.xa, 0, sizeof(double) * (size_t)B * N, S.stream));  // anchor 0: the whole product is A x
    if (!transpose) {
      MF_CK(cudaMemcpyAsync(S.ctx.x, X, sizeof(double) * (size_t)B * N, cudaMemcpyHostToDevice, S.stream));
      op->forward(S.stream, S.ctx.x, kGateAll, kQChiX, true);  // stores y - A x with y = 0
      std::vector<double> r((size_t)B * M);
      MF_CK(cudaMemcpyAsync(r.data(), op->g.resid, sizeof(double) * r.size(), cudaMemcpyDeviceToHost, S.stream));
      MF_CK(cudaStreamSynchronize(S.stream));
      for (size_t i = 0; i < r.size(); ++i) out[i] = -r[i];
    } else {
      MF_CK(cudaMemcpyAsync(op->g.resid, X, sizeof(double) * (size_t)B * M, cudaMemcpyHostToDevice, S.stream));
      op->adjoint(S.stream, nullptr, -1);
      MF_CK(cudaMemcpyAsync(out, S.ctx.dfdx, sizeof(double) * (size_t)B * N, cudaMemcpyDeviceToHost, S.stream));
      MF_CK(cudaStreamSynchronize(S.stream));
    }
    if (op->device_error()) throw Error(MFISTA_ERR_CUDA, "a tensor-core GEMM wait timed out");
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_dft_profile(const double* A, int M, int N, int B, int precision, int kernel, int reps,
                                  double* ms_per_launch, double* bytes_per_launch) {
  set_ok();
  try {
    if (M < 1 || N < 1 || B < 1 || !A) throw Error(MFISTA_ERR_ARG, "bad sizes or null pointer");
    Solver S;
    S.precision = MFISTA_FP64;
    S.init_common(B, N, N, 1, kFormTSV, 100, nullptr);
    std::vector<double> y(M, 0.0);
    S.op.reset(new DftOp(S.ctx, A, y.data(), M, N, precision));
    int slots = std::max({S.op->chi_slots(), S.op->tsv_slots(), S.img_blocks(), 1});
    S.d_part.alloc(sizeof(double) * (size_t)kNumQ * B * slots);
    S.ctx.part.p = S.d_part.as<double>();
    S.ctx.part.slots = slots;
    S.ctx.part.B = B;
    MF_CK(cudaMemsetAsync(S.ctx.prm, 0, sizeof(ProbParams) * B, S.stream));
    MF_CK(cudaMemsetAsync(S.ctx.z, 0, sizeof(double) * (size_t)B * N, S.stream));
    double ms = 0, bytes = 0;
    S.profile_kernel(kernel, 1, ms, bytes);  // warm
    S.profile_kernel(kernel, std::max(1, reps), ms, bytes);
    if (S.op->device_error()) throw Error(MFISTA_ERR_CUDA, "a tensor-core GEMM wait timed out");
    if (ms_per_launch) *ms_per_launch = ms;
    if (bytes_per_launch) *bytes_per_launch = bytes;
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_nufft_lipschitz(const double* u_dx, const double* v_dy, const double* vis_std, int M, int Nx,
                                      int Ny, int iters, double* lip_out) {
  set_ok();
  try {
    int n = Nx * Ny;
    std::vector<double> x(n), g(n), fr(M), fi(M), rr(M), ri(M);
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < n; ++i) {
      s ^= s << 13;
      s ^= s >> 7;
      s ^= s << 17;
      x[i] = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    }
    double lam = 0;
    for (int it = 0; it < iters; ++it) {
      double nrm = 0;
      for (double v : x) nrm += v * v;
      nrm = sqrt(nrm);
      for (double& v : x) v /= nrm;
      nufft_apply<double>(u_dx, v_dy, nullptr, M, Nx, Ny, x.data(), nullptr, nullptr, fr.data(), fi.data(), nullptr);
      for (int k = 0; k < M; ++k) {
        double w2 = 1.0 / (vis_std[k] * vis_std[k]);
        rr[k] = fr[k] * w2;
        ri[k] = fi[k] * w2;
      }
      nufft_apply<double>(u_dx, v_dy, nullptr, M, Nx, Ny, nullptr, rr.data(), ri.data(), nullptr, nullptr, g.data());
      lam = 0;
      for (int i = 0; i < n; ++i) lam += x[i] * g[i];
      x = g;
    }
    *lip_out = lam;
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_fgp_prox(const double* b, int NX, int NY, double lambda_l1, double lambda_tv, int iters,
                               int nonneg_flag, int box_flag, const float* cl_box, double* x_out, int precision) {
  set_ok();
  try {
    int n = NX * NY;
    Solver S;
    S.precision = precision == MFISTA_FP32 ? MFISTA_FP32 : MFISTA_FP64;
    S.init_common(1, n, NX, NY, kFormTV, iters, box_flag == 1 ? cl_box : nullptr);
    S.setup_fgp();
    // FGP forms b = dfdx / c + z (minus lambda_l1 / c when nonneg); with c = 1,
    // dfdx = 0 and z = b (lambda_l1 = 0 on the nonneg path) it sees b exactly
    ProbParams p;
    memset(&p, 0, sizeof(p));
    p.lambda_l1 = nonneg_flag == 1 ? 0.0 : lambda_l1;
    p.lambda_tv = lambda_tv;
    p.nonneg = nonneg_flag;
    p.box_flag = box_flag;
    ProbState st;
    memset(&st, 0, sizeof(st));
    st.active = 1;
    st.c = 1.0;
    MF_CK(cudaMemcpyAsync(S.ctx.prm, &p, sizeof(p), cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemcpyAsync(S.ctx.st, &st, sizeof(st), cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemcpyAsync(S.ctx.z, b, sizeof(double) * n, cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemsetAsync(S.ctx.dfdx, 0, sizeof(double) * n, S.stream));
    S.launch_fgp(S.stream);
    MF_CK(cudaMemcpyAsync(x_out, S.ctx.xnew, sizeof(double) * n, cudaMemcpyDeviceToHost, S.stream));
    MF_CK(cudaStreamSynchronize(S.stream));
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

extern "C" int mfista_fgp_profile(int NX, int NY, int B, int iters, int precision, int reps, double* ms_per_launch,
                                  double* bytes_per_launch) {
  set_ok();
  try {
    if (NX < 2 || NY < 2 || B < 1 || iters < 1) throw Error(MFISTA_ERR_ARG, "mfista_fgp_profile: bad sizes");
    const int n = NX * NY;
    Solver S;
    S.precision = precision == MFISTA_FP32 ? MFISTA_FP32 : MFISTA_FP64;
    S.init_common(B, n, NX, NY, kFormTV, iters, nullptr);
    S.setup_fgp();
    // every problem a nonnegative FGP prox of a random image at
    // lambda_tv = 1e-2 (c = 1, dfdx = 0, z = b)
    std::vector<ProbParams> prm(B);
    std::vector<ProbState> st(B);
    std::vector<double> z((size_t)B * n);
    uint64_t r = 0x2545F4914F6CDD1Dull;
    for (double& v : z) {
      r ^= r << 13;
      r ^= r >> 7;
      r ^= r << 17;
      v = (double)(r >> 11) / 9007199254740992.0;
    }
    for (int b = 0; b < B; ++b) {
      memset(&prm[b], 0, sizeof(ProbParams));
      prm[b].lambda_tv = 1e-2;
      prm[b].nonneg = 1;
      memset(&st[b], 0, sizeof(ProbState));
      st[b].active = 1;
      st[b].c = 1.0;
    }
    MF_CK(cudaMemcpyAsync(S.ctx.prm, prm.data(), sizeof(ProbParams) * B, cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemcpyAsync(S.ctx.st, st.data(), sizeof(ProbState) * B, cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemcpyAsync(S.ctx.z, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice, S.stream));
    MF_CK(cudaMemsetAsync(S.ctx.dfdx, 0, sizeof(double) * z.size(), S.stream));
    S.launch_fgp(S.stream);  // warm
    cudaEvent_t e0, e1;
    MF_CK(cudaEventCreate(&e0));
    MF_CK(cudaEventCreate(&e1));
    MF_CK(cudaEventRecord(e0, S.stream));
    const int R = std::max(1, reps);
    for (int k = 0; k < R; ++k) S.launch_fgp(S.stream);
    MF_CK(cudaEventRecord(e1, S.stream));
    MF_CK(cudaEventSynchronize(e1));
    float t = 0;
    MF_CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_per_launch) *ms_per_launch = t / R;
    // compulsory bytes of one prox call: z and dfdx read, xnew written (FP64)
    if (bytes_per_launch) *bytes_per_launch = 24.0 * (double)B * n;
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

// leave-one-out error of DFT solutions (c/looe_lib.c, see looe.cuh)
extern "C" int mfista_dft_looe(const double* y, const double* A, int M, int N, int NX, const double* X, int B,
                               const double* lambda_tsv, double* looe_m, double* looe_std, int* hessian_positive) {
  set_ok();
  try {
    if (M < 2 || N < 1 || NX < 1 || B < 1) throw Error(MFISTA_ERR_ARG, "mfista_dft_looe: needs M >= 2, N, NX, B >= 1");
    if (!y || !A || !X || !looe_m || !looe_std || !hessian_positive)
      throw Error(MFISTA_ERR_ARG, "mfista_dft_looe: null pointer");
    looe::Looe L(y, A, M, N, NX);
    for (int b = 0; b < B; ++b) {
      double out[3];
      L.one(X + (size_t)b * N, lambda_tsv ? lambda_tsv[b] : 0.0, out);
      looe_m[b] = out[0];
      looe_std[b] = out[1];
      hessian_positive[b] = out[2] > 0.5 ? 1 : 0;
    }
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

// movie: frames coupled by a temporal term (matlab/MFISTA_movie_eht.m)
extern "C" int mfista_nufft_movie(const double* u_dx, const double* v_dy, const double* vis_r, const double* vis_i,
                                  const double* vis_std, const int* pt_off, int n_frames, int Nx, int Ny,
                                  const double* t_list, double lambda_l1, double lambda_tsv, double lambda_t,
                                  double cinit, int maxiter, double eps, int nonneg_flag, const double* c_box,
                                  int precision, const double* xinit, double* xout, struct RESULT* results,
                                  double* temporal_cost) {
  set_ok();
  try {
    if (n_frames < 1 || Nx < 1 || Ny < 1) throw Error(MFISTA_ERR_ARG, "mfista_nufft_movie: bad sizes");
    if (!u_dx || !v_dy || !vis_r || !vis_i || !vis_std || !pt_off || !xout)
      throw Error(MFISTA_ERR_ARG, "mfista_nufft_movie: null pointer");
    if (maxiter < 0) throw Error(MFISTA_ERR_ARG, "maxiter must be >= 0");
    if (nonneg_flag != 0 && nonneg_flag != 1) throw Error(MFISTA_ERR_ARG, "nonneg_flag must be 0 or 1");
    if (lambda_t < 0 || lambda_tsv < 0) throw Error(MFISTA_ERR_ARG, "lambda_t and lambda_tsv must be >= 0");
    if (precision != MFISTA_FP64 && precision != MFISTA_FP32)
      throw Error(MFISTA_ERR_ARG, "mfista_nufft_movie: precision must be MFISTA_FP64 or MFISTA_FP32");
    if (pt_off[0] < 0) throw Error(MFISTA_ERR_ARG, "pt_off[0] must be >= 0");
    for (int b = 0; b < n_frames; ++b)
      if (pt_off[b + 1] < pt_off[b]) throw Error(MFISTA_ERR_ARG, "pt_off must not decrease");
    std::vector<double> wt(std::max(n_frames - 1, 0));
    for (int b = 0; b + 1 < n_frames; ++b) {
      const double dt = t_list ? t_list[b + 1] - t_list[b] : 1.0;
      if (!(dt > 0)) throw Error(MFISTA_ERR_ARG, "t_list must increase strictly");
      wt[b] = 1.0 / dt;
    }
    const int N = Nx * Ny;
    Solver S;
    S.precision = precision;
    S.init_common(n_frames, N, Nx, Ny, kFormTSV, 100, nullptr);
    NufftInput in{u_dx, v_dy, vis_r, vis_i, vis_std, pt_off, 0, 0, Nx, Ny};
    if (precision == MFISTA_FP32) S.op.reset(new NufftOp<float>(S.ctx, in, true));
    else S.op.reset(new NufftOp<double>(S.ctx, in));
    S.set_movie(wt, lambda_t);
    if (c_box) S.set_mask(c_box);
    S.finish_setup();
    std::vector<ProbParams> prm(n_frames);
    for (int b = 0; b < n_frames; ++b)
      prm[b] = ProbParams{lambda_l1, 0.0, lambda_tsv, cinit, eps, maxiter, nonneg_flag, 0, 0, 0.0};
    std::vector<double> x0;
    if (xinit) {  // x = (xinit .* c_box) for every frame (MFISTA_movie_eht.m:46)
      x0.resize((size_t)n_frames * N);
      for (int b = 0; b < n_frames; ++b)
        for (int f = 0; f < N; ++f) x0[(size_t)b * N + f] = c_box ? xinit[f] * c_box[f] : xinit[f];
    }
    double t0 = now_s();
    S.upload_problems(prm, xinit ? x0.data() : nullptr);
    S.enqueue_solve(false);
    std::vector<FinalOut> o;
    S.fetch(xout, o);
    const double ct = now_s() - t0;
    double dx = 0.0;
    for (int b = 0; b < n_frames; ++b) dx += o[b].dt_pair;
    if (temporal_cost) *temporal_cost = lambda_t * dx;
    if (results)
      for (int b = 0; b < n_frames; ++b) {
        const int m = pt_off[b + 1] - pt_off[b];
        fill_result(&results[b], o[b], m / 2, (double)m, Nx, Ny, N, lambda_l1, 0.0, lambda_tsv, maxiter, nonneg_flag, ct,
                    false, cinit);
      }
    if (o[0].status) return fail(o[0].status, "the movie stopped early (status " + std::to_string(o[0].status) + ")", false);
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

// forward NUFFT of the reference's C++ build (x2y_nufft), see cpp_nufft.cuh
extern "C" int mfista_cpp_x2y_nufft(const double* u_dx, const double* v_dy, int M, int Nx, int Ny, const double* xin,
                                    double* y_r, double* y_i) {
  set_ok();
  try {
    if (M < 1 || Nx < 12 || Ny < 12) throw Error(MFISTA_ERR_ARG, "mfista_cpp_x2y_nufft: needs M >= 1, Nx, Ny >= 12");
    if (!u_dx || !v_dy || !xin || !y_r || !y_i) throw Error(MFISTA_ERR_ARG, "mfista_cpp_x2y_nufft: null pointer");
    cppnufft::Prep pr(u_dx, v_dy, M, Nx, Ny);
    Solver S;
    S.precision = MFISTA_FP64;
    S.init_common(1, Nx * Ny, Nx, Ny, kFormTSV, 100, nullptr);
    std::vector<double> zero(M, 0.0), one(M, 1.0);
    NufftInput in{u_dx, v_dy, zero.data(), zero.data(), one.data(), nullptr, 1, M, Nx, Ny};
    NufftOp<double>* op = new NufftOp<double>(S.ctx, in);
    S.op.reset(op);
    ProbState st;
    memset(&st, 0, sizeof(st));
    st.active = 1;
    MF_CK(cudaMemcpyAsync(S.ctx.st, &st, sizeof(st), cudaMemcpyHostToDevice, S.stream));
    op->d_e4.upload(pr.e4.data(), pr.e4.size());  // the C++ build's grid correction
    op->geo.e4 = op->d_e4.as<double>();
    MF_CK(cudaMemcpyAsync(S.ctx.x, xin, sizeof(double) * (size_t)Nx * Ny, cudaMemcpyHostToDevice, S.stream));
    op->launch_rows_fwd(S.stream, S.ctx.x, kGateAll, nullptr);
    op->launch_cols_fwd(S.stream, kGateAll);
    DevMem d_mx, d_my, d_yn, d_e1, d_e2x, d_e2y, d_out;
    d_mx.upload(pr.mx.data(), M);
    d_my.upload(pr.my.data(), M);
    d_yn.upload(pr.yneg.data(), M);
    d_e1.upload(pr.e1.data(), M);
    d_e2x.upload(pr.e2x.data(), pr.e2x.size());
    d_e2y.upload(pr.e2y.data(), pr.e2y.size());
    d_out.alloc(sizeof(double) * 2 * (size_t)M);
    cppnufft::k_cpp_interp<<<cdiv(M, 8), 256, 0, S.stream>>>(
        op->d_grid.as<cplx<double>>(), Nx, Ny, d_mx.as<int>(), d_my.as<int>(), d_yn.as<int>(), d_e1.as<double>(),
        d_e2x.as<double>(), d_e2y.as<double>(), M, 1.0 / (4.0 * (double)Nx * (double)Ny), d_out.as<double>(),
        d_out.as<double>() + M);
    MF_LAUNCH_CK();
    MF_CK(cudaMemcpyAsync(y_r, d_out.p, sizeof(double) * M, cudaMemcpyDeviceToHost, S.stream));
    MF_CK(cudaMemcpyAsync(y_i, d_out.as<double>() + M, sizeof(double) * M, cudaMemcpyDeviceToHost, S.stream));
    MF_CK(cudaStreamSynchronize(S.stream));
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

// ---------------------------------------------------------------------------
// the reference's C++ build (c++/mfista_nufft_lib.cpp, c++/mfista_fft_lib.cpp)
// ---------------------------------------------------------------------------
namespace {

// sort_input (c++/mfista_nufft_lib.cpp:550-641): the points ordered by their
// rounded grid row of v, then of u, with std::sort and the reference's
// comparator; the five arrays are permuted in place.
void cpp_sort_input(int M, int Nx, int Ny, double* u, double* v, double* vr, double* vi, double* vs) {
  const int mrx = 2 * Nx, mry = 2 * Ny;
  std::vector<size_t> idx(M);
  for (int i = 0; i < M; ++i) idx[i] = (size_t)i;
  std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    const double va = round(v[a] * mry / (2 * M_PI)), vb = round(v[b] * mry / (2 * M_PI));
    if (va == vb) return round(u[a] * mrx / (2 * M_PI)) < round(u[b] * mrx / (2 * M_PI));
    return va < vb;
  });
  std::vector<double> tmp(M);
  for (double* arr : {u, v, vr, vi, vs}) {
    for (int i = 0; i < M; ++i) tmp[i] = arr[i];
    for (int i = 0; i < M; ++i) arr[i] = tmp[idx[i]];
  }
}

// calc_costs_nufft (c++/mfista_nufft_lib.cpp:931-998): the fields it sets
void fill_costs_cpp(RESULT* r, const FinalOut& o, int M, int nx, int ny, double l1, double ltv, double ltsv) {
  r->sq_error = o.sq_error;
  r->M = M;
  r->N = nx * ny;
  r->NX = nx;
  r->NY = ny;
  r->lambda_l1 = l1;
  r->lambda_tv = ltv;
  r->lambda_tsv = ltsv;
  r->mean_sq_error = o.sq_error / (double)M;
  r->l1cost = o.l1cost;
  r->N_active = (int)llround(o.n_active);
  double fc = o.sq_error / 2;
  if (l1 > 0) fc += l1 * o.l1cost;
  if (ltsv > 0) {
    r->tsvcost = o.regcost;
    fc += ltsv * o.regcost;
  }
  r->finalcost = fc;
}

// summary (costs) of the C++-build NUFFT problem at x0, no iterations
void cpp_costs_at(const double* u, const double* v, const double* vr, const double* vi, const double* vs, int M,
                  int Nx, int Ny, const ProbParams& p, const double* x0, FinalOut& out) {
  Solver S;
  S.precision = MFISTA_FP64;
  S.init_common(1, Nx * Ny, Nx, Ny, kFormTSV, 100, nullptr);
  S.op.reset(new cppnufft::CppNufftOp(S.ctx, u, v, vr, vi, vs, M, Nx, Ny));
  S.finish_setup();
  S.upload_problems({p}, x0);
  S.enqueue_solve(true);
  std::vector<FinalOut> o;
  S.fetch(nullptr, o);
  out = o[0];
}

}  // namespace

extern "C" int mfista_cpp_y2x_nufft(const double* u_dx, const double* v_dy, int M, int Nx, int Ny,
                                    const double* yin_r, const double* yin_i, double* xout) {
  set_ok();
  try {
    if (M < 1 || Nx < 12 || Ny < 12) throw Error(MFISTA_ERR_ARG, "mfista_cpp_y2x_nufft: needs M >= 1, Nx, Ny >= 12");
    if (!u_dx || !v_dy || !yin_r || !yin_i || !xout) throw Error(MFISTA_ERR_ARG, "mfista_cpp_y2x_nufft: null pointer");
    Solver S;
    S.precision = MFISTA_FP64;
    S.init_common(1, Nx * Ny, Nx, Ny, kFormTSV, 100, nullptr);
    std::vector<double> zero(M, 0.0), one(M, 1.0);
    cppnufft::CppNufftOp* op = new cppnufft::CppNufftOp(S.ctx, u_dx, v_dy, zero.data(), zero.data(), one.data(), M,
                                                        Nx, Ny);
    S.op.reset(op);
    std::vector<double2> y(M);
    for (int k = 0; k < M; ++k) y[k] = make_double2(yin_r[k], yin_i[k]);
    MF_CK(cudaMemcpyAsync(op->y2(), y.data(), sizeof(double2) * (size_t)M, cudaMemcpyHostToDevice, S.stream));
    ProbState st;
    memset(&st, 0, sizeof(st));
    st.active = 1;
    MF_CK(cudaMemcpyAsync(S.ctx.st, &st, sizeof(st), cudaMemcpyHostToDevice, S.stream));
    op->adjoint_into(S.stream, S.ctx.dfdx, nullptr, -1, kGateAll);
    MF_CK(cudaMemcpyAsync(xout, S.ctx.dfdx, sizeof(double) * (size_t)Nx * Ny, cudaMemcpyDeviceToHost, S.stream));
    MF_CK(cudaStreamSynchronize(S.stream));
    return MFISTA_OK;
  } catch (const Error& e) {
    return fail(e.status, e.what(), false);
  }
}

// mfista_imaging_core_nufft of the C++ build (c++/mfista_nufft_lib.cpp:1016-1074):
// RESULT from calc_costs_nufft (M = M, not M/2), TSV form only, the caller's
// u/v/vis arrays sorted in place, first-iteration backtracking factor 10.
extern "C" void mfista_cpp_imaging_core_nufft(double* u_dx, double* v_dy, double* vis_r, double* vis_i,
                                              double* vis_std, int M, int Nx, int Ny, int maxiter, double eps,
                                              double lambda_l1, double lambda_tv, double lambda_tsv, double cinit,
                                              double* xinit, double* xout, int nonneg_flag, int box_flag,
                                              float* cl_box, struct RESULT* mfista_costs) {
  set_ok();
  try {
    if (maxiter < 0) throw Error(MFISTA_ERR_ARG, "maxiter must be >= 0");
    double epsilon = 0;
    for (int i = 0; i < M; ++i) epsilon += vis_r[i] * vis_r[i] + vis_i[i] * vis_i[i];
    epsilon *= eps / ((double)M);
    const int N = Nx * Ny;
    // costs at xinit (:1037-1040)
    ProbParams p0{lambda_l1, 0.0, lambda_tsv, cinit, epsilon, 0, 1, 0, 0, 0.0};
    FinalOut o;
    cpp_costs_at(u_dx, v_dy, vis_r, vis_i, vis_std, M, Nx, Ny, p0, xinit, o);
    fill_costs_cpp(mfista_costs, o, M, Nx, Ny, lambda_l1, lambda_tv, lambda_tsv);
    if (lambda_tv != 0) {
      printf("We have not implemented TV option.\n");
      fail(MFISTA_ERR_ARG, "the C++ build has no TV form", false);
      return;
    }
    cpp_sort_input(M, Nx, Ny, u_dx, v_dy, vis_r, vis_i, vis_std);
    double t0 = now_s();
    if (nonneg_flag != 0 && nonneg_flag != 1) {
      // the C++ core returns 0 iterations without writing xout (:789-795)
      printf("nonneg_flag must be chosen properly.\n");
      cpp_costs_at(u_dx, v_dy, vis_r, vis_i, vis_std, M, Nx, Ny, p0, xout, o);
      mfista_costs->comp_time = now_s() - t0;
      mfista_costs->ITER = 0;
      mfista_costs->Lip_const = cinit;
    } else {
      ProbParams p{lambda_l1, 0.0, lambda_tsv, cinit, epsilon, maxiter, nonneg_flag, box_flag, 0, 0.0};
      Solver S;
      S.precision = MFISTA_FP64;
      S.eta_first = 10.0;
      S.init_common(1, N, Nx, Ny, kFormTSV, 100, box_flag == 1 ? cl_box : nullptr);
      S.op.reset(new cppnufft::CppNufftOp(S.ctx, u_dx, v_dy, vis_r, vis_i, vis_std, M, Nx, Ny));
      S.finish_setup();
      t0 = now_s();
      S.upload_problems({p}, xinit);
      S.enqueue_solve(maxiter == 0);
      std::vector<FinalOut> oo;
      S.fetch(xout, oo);
      o = oo[0];
      mfista_costs->comp_time = now_s() - t0;
      mfista_costs->ITER = o.iters;
      mfista_costs->Lip_const = maxiter == 0 ? cinit : o.lip;
      if (o.status) fail(o.status, "solver stopped early (status " + std::to_string(o.status) + ")", !quiet());
    }
    mfista_costs->nonneg = nonneg_flag;
    mfista_costs->maxiter = maxiter;
    fill_costs_cpp(mfista_costs, o, M, Nx, Ny, lambda_l1, lambda_tv, lambda_tsv);
  } catch (const Error& e) {
    fail(e.status, e.what(), true);
  }
}

// mfista_imaging_core_fft of the C++ build (c++/mfista_fft_lib.cpp:425-485):
// the C library's TSV solve; the TV form is not implemented there.
extern "C" void mfista_cpp_imaging_core_fft(int* u_idx, int* v_idx, double* y_r, double* y_i, double* noise_stdev,
                                            int M, int NX, int NY, int maxiter, double eps, double lambda_l1,
                                            double lambda_tv, double lambda_tsv, double cinit, double* xinit,
                                            double* xout, int nonneg_flag, unsigned int fftw_plan_flag, int box_flag,
                                            float* cl_box, struct RESULT* mfista_result) {
  if (lambda_tv != 0) {
    set_ok();
    printf("We have not implemented TV option.\n");
    fail(MFISTA_ERR_ARG, "the C++ build has no TV form", false);
    return;
  }
  mfista_imaging_core_fft(u_idx, v_idx, y_r, y_i, noise_stdev, M, NX, NY, maxiter, eps, lambda_l1, lambda_tv,
                          lambda_tsv, cinit, xinit, xout, nonneg_flag, fftw_plan_flag, box_flag, cl_box,
                          mfista_result);
}
