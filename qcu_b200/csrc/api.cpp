// The C ABI: qcu.h (drop-in) and qcu_ext.h (extension).  Every entry point
// catches internal exceptions and turns them into a recorded last error.
#include <cstring>

#include "batch.h"
#include "mrhs.h"
#include "dd.h"
#include "mg.h"
#include "nn.h"
#include "solver.h"

// the library is built with hidden visibility; only the C ABI is exported
#pragma GCC visibility push(default)
#include "../../include/qcu.h"
#include "../../include/qcu_ext.h"
#pragma GCC visibility pop

namespace qcu {
int last_error(char *buf, int len);
void clover_dslash_noalloc(void *out, const void *in, const void *gauge, const int latt[4], int parity);
int noalloc_max_vh();
}

using namespace qcu;

struct qcuGauge_s {
  GaugeHandle *h;
};
struct qcuNN_s {
  NNet *n;
};
struct qcuMG_s {
  MG *m;
};

#define QCU_API_BEGIN \
  clear_last_error(); \
  try {
#define QCU_API_END                                \
  return 0;                                        \
  }                                                \
  catch (const qcu::Error &e) {                    \
    set_last_error(e.code, e.what());              \
    return e.code;                                 \
  }                                                \
  catch (const std::exception &e) {                \
    set_last_error(3, e.what());                   \
    return 3;                                      \
  }                                                \
  catch (...) {                                    \
    set_last_error(3, "unknown internal error");   \
    return 3;                                      \
  }

static bool single_rank(const QcuParam *grid) {
  require(grid != nullptr, "grid pointer is null");
  for (int d = 0; d < 4; d++)
    if (grid->lattice_size[d] != 1) return false;
  return true;
}

static int legacy_dslash_call(void *out, void *in, void *gauge, QcuParam *param, int parity, int clover) {
  QCU_API_BEGIN
  require(param != nullptr, "param pointer is null");
  legacy_dslash(out, in, gauge, param->lattice_size, parity, clover);
  QCU_API_END
}

extern "C" {

// ---------------------------------------------------------------- qcu.h
void dslashQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity) {
  legacy_dslash_call(fermion_out, fermion_in, gauge, param, parity, 0);
}

void dslashCloverQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity) {
  legacy_dslash_call(fermion_out, fermion_in, gauge, param, parity, 1);
}

void mpiDslashQcu(void *, void *, void *, QcuParam *, int, QcuParam *) {}
void mpiBistabCgQcu(void *, QcuParam *, QcuParam *) {}

void ncclDslashQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity, QcuParam *grid) {
  clear_last_error();
  bool one = true;
  try {
    one = single_rank(grid);
    if (!one) {
      // this rank's sub-lattice; faces exchanged with the neighbouring ranks
      // over the communicator set up by qcuCommInit (src/nccl_wilson_dslash.cu:3-19)
      require(param != nullptr, "param pointer is null");
      dd_dslash_nccl(fermion_out, fermion_in, gauge, param->lattice_size, parity, grid->lattice_size);
    }
  } catch (const qcu::Error &e) {
    set_last_error(e.code, e.what());
    return;
  } catch (const std::exception &e) {
    set_last_error(3, e.what());
    return;
  }
  if (one) legacy_dslash_call(fermion_out, fermion_in, gauge, param, parity, 0);
}

void ncclBistabCgQcu(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, QcuParam *grid) {
  clear_last_error();
  GaugeHandle *G = nullptr;
  try {
    require(param != nullptr, "param pointer is null");
    if (!single_rank(grid)) {
      // this rank's part of the solve over the grid: qcu's kappa, start,
      // criterion and iteration cap, inner products summed over all ranks
      dd_solve(fermion_out, fermion_in, gauge, param->lattice_size, grid->lattice_size, false, 0.125, 1e-9, 1000,
               23333);
      return;
    }
    G = gauge_load(gauge, param->lattice_size, 1.0, 0.0);
    SolveParams p;
    p.kappa = 0.125;   // include/define.h:69
    p.tol = 1e-9;      // include/define.h:68, absolute on ||r||^2
    p.abs_tol = 1;
    p.maxiter = 1000;  // include/define.h:67
    p.precision = 64;
    p.delta = 0.0;
    p.x0_mode = 2;     // random start, include/lattice_bistabcg.h:108-109
    p.x0_seed = 23333;
    solve(*G, fermion_out, fermion_in, p);
  } catch (const qcu::Error &e) {
    set_last_error(e.code, e.what());
  } catch (const std::exception &e) {
    set_last_error(3, e.what());
  }
  delete G;
}

// ---------------------------------------------------------------- qcu_ext.h
int qcuGetLastError(char *msg, int len) { return last_error(msg, len); }
int qcuVersion(void) { return 1; }

int qcuGaugeLoad(qcuGauge *h, const void *gauge, const int latt[4], double t_boundary, double clover_coeff) {
  QCU_API_BEGIN
  require(h != nullptr, "handle pointer is null");
  *h = nullptr;
  GaugeHandle *G = gauge_load(gauge, latt, t_boundary, clover_coeff);
  *h = new qcuGauge_s{G};
  QCU_API_END
}

int qcuGaugeFree(qcuGauge h) {
  QCU_API_BEGIN
  if (h) {
    delete h->h;
    delete h;
  }
  QCU_API_END
}

int qcuDslash(qcuGauge h, void *out, const void *in, int parity, int use_clover, int precision) {
  QCU_API_BEGIN
  require(h != nullptr, "null gauge handle");
  handle_dslash(*h->h, out, in, parity, use_clover, precision);
  QCU_API_END
}

int qcuMatPC(qcuGauge h, void *out, const void *in, double kappa, int use_clover) {
  QCU_API_BEGIN
  require(h != nullptr, "null gauge handle");
  handle_mpc(*h->h, out, in, kappa, use_clover);
  QCU_API_END
}

int qcuMat(qcuGauge h, void *out, const void *in, double kappa, int use_clover) {
  QCU_API_BEGIN
  require(h != nullptr, "null gauge handle");
  handle_mat(*h->h, out, in, kappa, use_clover);
  QCU_API_END
}

void qcuInvertParamDefault(qcuInvertParam *p) {
  if (!p) return;
  SolveParams d;
  p->kappa = d.kappa;
  p->tol = d.tol;
  p->maxiter = d.maxiter;
  p->precision = d.precision;
  p->delta = d.delta;
  p->abs_tol = d.abs_tol;
  p->x0_mode = d.x0_mode;
  p->x0_seed = d.x0_seed;
  p->use_clover = d.use_clover;
  p->chunk = d.chunk;
  p->solver = d.solver;
  p->inner_iters = d.inner_iters;
  p->inner_tol = d.inner_tol;
  p->gcr_k = d.gcr_k;
  p->gauge_precision = d.gauge_precision;
  p->precond = d.precond;
  p->nn = nullptr;
  p->mg = nullptr;
}

static SolveParams solve_params(const qcuInvertParam *p) {
  SolveParams s;
  s.kappa = p->kappa;
  s.tol = p->tol;
  s.maxiter = p->maxiter;
  s.precision = p->precision;
  s.delta = p->delta;
  s.abs_tol = p->abs_tol;
  s.x0_mode = p->x0_mode;
  s.x0_seed = p->x0_seed;
  s.use_clover = p->use_clover;
  s.chunk = p->chunk;
  s.solver = p->solver;
  s.inner_iters = p->inner_iters;
  s.inner_tol = p->inner_tol;
  s.gcr_k = p->gcr_k;
  s.gauge_precision = p->gauge_precision;
  s.precond = p->precond;
  s.nn = p->nn ? p->nn->n : nullptr;
  s.mg = p->mg ? p->mg->m : nullptr;
  require(s.tol > 0, "tol must be positive");
  require(s.delta >= 0 && s.delta < 1, "delta must be in [0, 1)");
  return s;
}

static void fill_result(const SolveInfo &info, qcuInvertResult *r) {
  r->iterations = info.iterations;
  r->reliable_updates = info.updates;
  r->status = info.status;
  r->restarts = info.restarts;
  r->true_residual = info.true_residual;
  r->iter_residual2 = info.iter_residual2;
  r->seconds = info.seconds;
  r->fallback = info.fallback;
}

int qcuInvert(qcuGauge h, void *x, const void *b, const qcuInvertParam *p, qcuInvertResult *r) {
  QCU_API_BEGIN
  require(h != nullptr && p != nullptr, "null handle or parameter pointer");
  const SolveInfo info = solve(*h->h, x, b, solve_params(p));
  if (r) fill_result(info, r);
  QCU_API_END
}

int qcuInvertBatch(const qcuBatchSystem *systems, int n_systems, const qcuInvertParam *p, qcuInvertResult *results,
                   qcuBatchTune *tune) {
  QCU_API_BEGIN
  require(systems != nullptr && p != nullptr && n_systems > 0, "null systems/parameter pointer or no systems");
  std::vector<BatchSystem> sys(n_systems);
  for (int i = 0; i < n_systems; i++) {
    require(systems[i].gauge != nullptr, "batch: null gauge handle");
    sys[i].G = systems[i].gauge->h;
    sys[i].nrhs = systems[i].nrhs;
    sys[i].kappa = systems[i].kappa;
    sys[i].use_clover = systems[i].use_clover;
    sys[i].x = systems[i].x;
    sys[i].b = systems[i].b;
  }
  BatchTune t;
  const std::vector<SolveInfo> info = solve_batch(sys, solve_params(p), &t);
  if (results)
    for (size_t r = 0; r < info.size(); r++) fill_result(info[r], results + r);
  if (tune) {
    tune->dslash_threads = t.dslash_threads;
    tune->dslash_rhs = t.dslash_rhs;
    tune->blas_sites = t.blas_sites;
    tune->mma = t.mma;
  }
  QCU_API_END
}

int qcuBatchDslashTime(const qcuBatchSystem *systems, int n_systems, int precision, int gauge_precision,
                       qcuBatchTune *tune, int iters, double *ms) {
  QCU_API_BEGIN
  require(systems != nullptr && ms != nullptr && n_systems > 0, "null systems/ms pointer or no systems");
  std::vector<BatchSystem> sys(n_systems);
  for (int i = 0; i < n_systems; i++) {
    require(systems[i].gauge != nullptr, "batch: null gauge handle");
    sys[i].G = systems[i].gauge->h;
    sys[i].nrhs = systems[i].nrhs;
    sys[i].kappa = systems[i].kappa;
    sys[i].use_clover = systems[i].use_clover;
    sys[i].x = systems[i].x;
    sys[i].b = systems[i].b;
  }
  SolveParams p;
  p.precision = precision;
  p.gauge_precision = gauge_precision;
  BatchTune t, chosen;
  const bool force = tune != nullptr && tune->dslash_threads > 0;
  if (force) {
    t.dslash_threads = tune->dslash_threads;
    t.dslash_rhs = tune->dslash_rhs;
    t.blas_sites = tune->blas_sites;
    t.mma = tune->mma;
  }
  solve_batch(sys, p, &chosen, force ? &t : nullptr, nullptr, ms, iters);
  if (tune) {
    tune->dslash_threads = chosen.dslash_threads;
    tune->dslash_rhs = chosen.dslash_rhs;
    tune->blas_sites = chosen.blas_sites;
    tune->mma = chosen.mma;
  }
  QCU_API_END
}

int qcuDslashMultiTC(qcuGauge h, void *out, const void *in, int nrhs, int parity) {
  QCU_API_BEGIN
  require(h != nullptr, "null gauge handle");
  handle_dslash_mrhs(*h->h, out, in, nrhs, parity);
  QCU_API_END
}

int qcuDslashMultiTCTime(qcuGauge h, int nrhs, int parity, int iters, double *ms) {
  QCU_API_BEGIN
  require(h != nullptr && ms != nullptr, "null gauge handle or ms pointer");
  *ms = handle_dslash_mrhs_time(*h->h, nrhs, parity, iters);
  QCU_API_END
}

int qcuBatchApplyMatPC(const qcuBatchSystem *systems, int n_systems, int precision, int gauge_precision,
                       const qcuBatchTune *tune, double *dots) {
  QCU_API_BEGIN
  require(systems != nullptr && tune != nullptr && dots != nullptr && n_systems > 0,
          "null systems/tune/dots pointer or no systems");
  std::vector<BatchSystem> sys(n_systems);
  for (int i = 0; i < n_systems; i++) {
    require(systems[i].gauge != nullptr, "batch: null gauge handle");
    sys[i].G = systems[i].gauge->h;
    sys[i].nrhs = systems[i].nrhs;
    sys[i].kappa = systems[i].kappa;
    sys[i].use_clover = systems[i].use_clover;
    sys[i].x = systems[i].x;
    sys[i].b = systems[i].b;
  }
  SolveParams p;
  p.precision = precision;
  p.gauge_precision = gauge_precision;
  BatchTune t;
  t.dslash_threads = tune->dslash_threads;
  t.dslash_rhs = tune->dslash_rhs;
  t.blas_sites = tune->blas_sites;
  t.mma = tune->mma;
  solve_batch(sys, p, nullptr, &t, dots);
  QCU_API_END
}

int qcuGaugeRandom(void *gauge, const int latt[4], int kind, double eps, unsigned long long seed) {
  QCU_API_BEGIN
  require(gauge != nullptr, "gauge pointer is null");
  require(kind >= 0 && kind <= 2, "gauge kind must be 0 (Haar), 1 (smooth) or 2 (unit)");
  const Geom g = make_geom(latt);
  Context &ctx = context();
  QCU_CUDA(cudaDeviceSynchronize());
  launch_gauge_random(g, gauge, kind, eps, seed, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  QCU_API_END
}

int qcuFermionRandom(void *psi, long long n, int kind, unsigned long long seed) {
  QCU_API_BEGIN
  require(psi != nullptr && n >= 0, "bad fermion buffer");
  require(kind == 0 || kind == 1, "fermion kind must be 0 (normal) or 1 (uniform)");
  Context &ctx = context();
  QCU_CUDA(cudaDeviceSynchronize());
  if (n > 0) launch_fermion_random(psi, n, kind, seed, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  QCU_API_END
}

int dslashCloverQcuNoAlloc(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity) {
  QCU_API_BEGIN
  require(param != nullptr, "param pointer is null");
  clover_dslash_noalloc(fermion_out, fermion_in, gauge, param->lattice_size, parity);
  QCU_API_END
}

int qcuNoAllocMaxSites(void) { return noalloc_max_vh(); }

int qcuCommUniqueId(void *id) {
  QCU_API_BEGIN
  dd_unique_id(id);
  QCU_API_END
}

int qcuCommInit(const void *id, int nranks, int rank) {
  QCU_API_BEGIN
  dd_comm_init(id, nranks, rank);
  QCU_API_END
}

int qcuCommFree(void) {
  QCU_API_BEGIN
  dd_comm_free();
  QCU_API_END
}

int qcuDDPlan(const int latt[4], const int grid[4], int rank, int *plan) {
  QCU_API_BEGIN
  require(plan != nullptr, "null plan buffer");
  const DDPlan p = dd_plan(latt, grid, rank);
  int k = 0;
  plan[k++] = p.nranks;
  plan[k++] = p.rank;
  for (int d = 0; d < 4; d++) plan[k++] = p.coord[d];
  for (int d = 0; d < 4; d++) plan[k++] = p.fwd[d];
  for (int d = 0; d < 4; d++) plan[k++] = p.bwd[d];
  for (int d = 0; d < 4; d++) plan[k++] = p.face[d];
  QCU_API_END
}

int qcuDDSchedule(const int latt[4], const int grid[4], int rank, int *ops, int *n_ops) {
  QCU_API_BEGIN
  require(ops != nullptr && n_ops != nullptr, "null schedule buffer");
  const std::vector<DDOp> s = dd_schedule(dd_plan(latt, grid, rank));
  for (size_t i = 0; i < s.size(); i++) {
    ops[5 * i] = s[i].kind;
    ops[5 * i + 1] = s[i].dir;
    ops[5 * i + 2] = s[i].slot;
    ops[5 * i + 3] = s[i].peer;
    ops[5 * i + 4] = s[i].count;
  }
  *n_ops = (int)s.size();
  QCU_API_END
}

int qcuDslashDDEmulate(void *out_all, const void *in_all, const void *gauge_all, const int latt[4], int parity,
                       const int grid[4]) {
  QCU_API_BEGIN
  dd_dslash_emulate(out_all, in_all, gauge_all, latt, parity, grid);
  QCU_API_END
}

int qcuBistabCgDDEmulate(void *x_all, const void *b_all, const void *gauge_all, const int latt[4], const int grid[4],
                         int *iterations, double *r2) {
  QCU_API_BEGIN
  const DDSolveResult r = dd_solve(x_all, b_all, gauge_all, latt, grid, true, 0.125, 1e-9, 1000, 23333);
  if (iterations) *iterations = r.iterations;
  if (r2) *r2 = r.r2;
  QCU_API_END
}

int qcuNNCreate(qcuNN *net, unsigned long long seed, double init_scale) {
  QCU_API_BEGIN
  require(net != nullptr, "null network pointer");
  *net = new qcuNN_s{nn_create(seed, init_scale)};
  QCU_API_END
}

int qcuNNFree(qcuNN net) {
  QCU_API_BEGIN
  if (net) {
    nn_free(net->n);
    delete net;
  }
  QCU_API_END
}

int qcuNNNumParams(void) { return nn_nparam(); }

int qcuNNGetWeights(qcuNN net, float *w) {
  QCU_API_BEGIN
  require(net && w, "null argument");
  nn_get(*net->n, w);
  QCU_API_END
}

int qcuNNSetWeights(qcuNN net, const float *w) {
  QCU_API_BEGIN
  require(net && w, "null argument");
  nn_set(*net->n, w);
  QCU_API_END
}

int qcuNNSetTensorCores(qcuNN net, int on) {
  QCU_API_BEGIN
  require(net != nullptr, "null network");
  nn_set_tensor_cores(*net->n, on);
  QCU_API_END
}

int qcuNNApply(qcuNN net, qcuGauge h, void *out, const void *in) {
  QCU_API_BEGIN
  require(net && h && out && in, "null argument");
  nn_apply_pyq(*net->n, *h->h, out, in);
  QCU_API_END
}

int qcuNNTrainStep(qcuNN net, qcuGauge h, const void *r, const void *e, int batch, double lr, double *loss,
                   float *grad) {
  QCU_API_BEGIN
  require(net && h && r && e && batch > 0, "bad arguments");
  const double l = nn_train_step(*net->n, *h->h, r, e, batch, lr, grad);
  if (loss) *loss = l;
  QCU_API_END
}

void qcuMGParamDefault(qcuMGParam *p) {
  if (!p) return;
  const MGParams d;
  for (int k = 0; k < 4; k++) p->geo_block_size[k] = d.geo_block_size[k];
  p->n_vec = d.n_vec;
  p->setup_maxiter = d.setup_maxiter;
  p->coarse_tol = d.coarse_tol;
  p->coarse_maxiter = d.coarse_maxiter;
  p->nu_pre = d.nu_pre;
  p->nu_post = d.nu_post;
  p->gcr_k = d.gcr_k;
}

int qcuMGCreate(qcuMG *mg, qcuGauge h, double kappa, const qcuMGParam *p, double *setup_seconds) {
  QCU_API_BEGIN
  require(mg != nullptr && h != nullptr, "null argument");
  MGParams q;
  if (p) {
    for (int k = 0; k < 4; k++) q.geo_block_size[k] = p->geo_block_size[k];
    q.n_vec = p->n_vec;
    q.setup_maxiter = p->setup_maxiter;
    q.coarse_tol = p->coarse_tol;
    q.coarse_maxiter = p->coarse_maxiter;
    q.nu_pre = p->nu_pre;
    q.nu_post = p->nu_post;
    q.gcr_k = p->gcr_k;
  }
  MG *m = mg_create(*h->h, kappa, q);
  if (setup_seconds) *setup_seconds = mg_setup_seconds(*m);
  *mg = new qcuMG_s{m};
  QCU_API_END
}

int qcuMGFree(qcuMG mg) {
  QCU_API_BEGIN
  if (mg) {
    mg_free(mg->m);
    delete mg;
  }
  QCU_API_END
}

int qcuMGInvert(qcuMG mg, void *x, const void *b, double tol, int maxiter, qcuMGResult *r) {
  QCU_API_BEGIN
  require(mg != nullptr, "null multigrid");
  const MGInfo i = mg_solve(*mg->m, x, b, tol, maxiter);
  if (r) {
    r->outer = i.outer;
    r->coarse_iters = i.coarse_iters;
    r->status = i.status;
    r->true_residual = i.true_residual;
    r->seconds = i.seconds;
  }
  QCU_API_END
}

int qcuMGCheck(qcuMG mg, double *orth_err, double *galerkin_err) {
  QCU_API_BEGIN
  require(mg && orth_err && galerkin_err, "null argument");
  mg_check(*mg->m, orth_err, galerkin_err);
  QCU_API_END
}

long long qcuKernelLaunches(void) { return launch_count(); }

void *qcuGetStream(void) {
  try {
    return (void *)context().stream;
  } catch (...) {
    return nullptr;
  }
}

int qcuBenchDslash(qcuGauge h, int precision, int gauge_precision, int use_clover, int iters, double *ms_per_call) {
  QCU_API_BEGIN
  require(h != nullptr && ms_per_call != nullptr && iters > 0, "bad arguments");
  GaugeHandle &G = *h->h;
  require(!use_clover || G.has_clover, "no clover term loaded");
  const int kind = precision == 64 ? SOA64 : precision == 32 ? SOA32 : precision == 16 ? SOA16 : -1;
  require(kind >= 0, "precision must be 64, 32 or 16");
  if (gauge_precision == 0) gauge_precision = precision;
  const int gkind = gauge_precision == 64 ? GSOA64 : gauge_precision == 32 ? GSOA32 : gauge_precision == 16 ? GSOA16 : -1;
  require(gkind == (kind == SOA64 ? GSOA64 : kind == SOA32 ? GSOA32 : GSOA16) || (kind == SOA32 && gkind == GSOA16),
          "unsupported spinor/link precision pair");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  const int Vh = G.g.Vh;
  Spinor a, b;
  a.alloc(kind, Vh);
  b.alloc(kind, Vh);
  DevBuf tmp;
  tmp.ensure(spinor_bytes(AOS64, Vh));
  launch_fermion_random(tmp.p, (int64_t)Vh * 12, 0, 12345, ctx.stream);
  launch_convert(AOS64, kind, Vh, tmp.p, nullptr, a.data.p, a.norm.as<float>(), ctx.stream);
  launch_convert(AOS64, kind, Vh, tmp.p, nullptr, b.data.p, b.norm.as<float>(), ctx.stream);
  DslashArgs d;
  d.gauge = gkind == GSOA64 ? G.g64.p : (gkind == GSOA32 ? G.g32.p : G.g16.p);
  d.t_bc = G.t_bc;
  d.a = 1.0;
  auto run = [&](int i) {
    const int par = i & 1;
    const Spinor &in = par ? a : b;
    Spinor &out = par ? b : a;
    d.in = in.data.p;
    d.in_norm = in.norm.as<float>();
    d.out = out.data.p;
    d.out_norm = out.norm.as<float>();
    d.parity = par;
    d.clover = use_clover ? G.clover_inv(kind, par) : nullptr;
    launch_dslash(kind, gkind, kind == SOA64 ? CSOA64 : CSOA32, G.g, d, ctx, ctx.stream);
  };
  for (int i = 0; i < 3; i++) run(i);
  cudaEvent_t e0, e1;
  QCU_CUDA(cudaEventCreate(&e0));
  QCU_CUDA(cudaEventCreate(&e1));
  QCU_CUDA(cudaEventRecord(e0, ctx.stream));
  for (int i = 0; i < iters; i++) run(i);
  QCU_CUDA(cudaEventRecord(e1, ctx.stream));
  QCU_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  QCU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_per_call = (double)ms / iters;
  QCU_API_END
}

}  // extern "C"
