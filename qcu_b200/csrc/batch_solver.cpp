// Batched solver driver: flexible GCR per right-hand side in FP64 around one
// inner BiCGSTAB that advances all right-hand sides of all lattices of the
// batch together (batch.h).
//
// Per outer step every kernel is one launch over the whole batch; the inner
// solve is one CUDA graph (init, a device-side WHILE loop over the batched
// BiCGSTAB iteration, the conversion of the result), captured once per call
// and replayed once per outer step.  The host reads the per-rhs states three
// times per outer step to form the GCR coefficients, as the single-rhs GCR
// does; a right-hand side that has converged (or broken down, or used its
// iterations) drops out of every later launch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>

#include "batch.h"

namespace qcu {

namespace {

struct RhsBufs {
  Spinor v[BV_N];
  Spinor W[GCR_MAXK], Z[GCR_MAXK];
  Spinor be, bo, xe, aux;  // FP64 source / solution halves
};

struct BatchCache {
  std::vector<std::unique_ptr<RhsBufs>> rhs;
  DevBuf desc, tiles[BT_N], groups[2], st, partials, active, coef;
  SolverState *st_host = nullptr;
  int *active_host = nullptr;
  BatchCoef *coef_host = nullptr;
  std::map<std::string, BatchTune> tuned;
  BatchCache() {
    QCU_CUDA(cudaMallocHost(&st_host, sizeof(SolverState) * BATCH_MAX_RHS));
    QCU_CUDA(cudaMallocHost(&active_host, sizeof(int) * BATCH_MAX_RHS));
    QCU_CUDA(cudaMallocHost(&coef_host, sizeof(BatchCoef) * BATCH_MAX_RHS));
    memset(coef_host, 0, sizeof(BatchCoef) * BATCH_MAX_RHS);
  }
};
BatchCache &cache() { return per_device<BatchCache>(context()); }

// Tile table over "units" (a rhs, or a group of rhs sharing a lattice):
// every unit's sites in blocks of `sites`; tiles sorted by the position of
// their block within the unit's lattice, units of the same position adjacent,
// so rhs sharing a lattice read the same links at the same time and lattices
// of different volume are spread over the whole grid.
std::vector<int2> make_tiles(const std::vector<int> &unit_vh, int sites) {
  size_t total = 0;
  for (int v : unit_vh) total += (v + sites - 1) / sites;
  require(total < (size_t)INT32_MAX, "batch too large");
  struct Key {
    double f;
    int u, b;
  };
  std::vector<Key> keys;
  keys.reserve(total);
  for (int u = 0; u < (int)unit_vh.size(); u++) {
    const int n = (unit_vh[u] + sites - 1) / sites;
    for (int b = 0; b < n; b++) keys.push_back({(b + 0.5) / n, u, b});
  }
  std::stable_sort(keys.begin(), keys.end(), [](const Key &x, const Key &y) { return x.f < y.f; });
  std::vector<int2> t(total);
  for (size_t i = 0; i < total; i++) t[i] = make_int2(keys[i].u, keys[i].b);
  return t;
}

}  // namespace

std::vector<SolveInfo> solve_batch(const std::vector<BatchSystem> &sys, const SolveParams &prm, BatchTune *tune_out,
                                   const BatchTune *force_tune, double *apply_dots, double *dslash_ms,
                                   int dslash_iters) {
  const auto t0 = std::chrono::steady_clock::now();
  require(!sys.empty(), "batch: no systems");
  require(prm.maxiter > 0 && prm.inner_iters > 0 && prm.gcr_k > 0, "batch: maxiter, inner_iters, gcr_k must be > 0");
  require(!prm.abs_tol && prm.x0_mode == 0, "batch: relative tolerance and a zero initial guess only");
  require(prm.precond == 0, "batch: the network preconditioner is available in single solves");
  const int kind = kind_of_precision(prm.precision);
  int gkind = kind == SOA64 ? GSOA64 : (kind == SOA32 ? GSOA32 : GSOA16);  // 16-bit spinors: 16-bit links
  if (prm.gauge_precision) {
    require(prm.gauge_precision == 16 && kind == SOA32, "batch: gauge_precision 16 is available with precision 32");
    gkind = GSOA16;
  }
  // expand the systems into right-hand sides
  struct Rhs {
    const BatchSystem *s;
    int j;
  };
  std::vector<Rhs> rl;
  for (const BatchSystem &s : sys) {
    require(s.G != nullptr && s.x != nullptr && s.b != nullptr, "batch: null gauge or spinor pointer");
    require(s.nrhs > 0, "batch: every system needs nrhs > 0");
    require(s.kappa > 0, "batch: kappa must be positive");
    require(!s.use_clover || s.G->has_clover, "batch: clover requested but the gauge handle has no clover term");
    for (int j = 0; j < s.nrhs; j++) rl.push_back({&s, j});
  }
  const int R = (int)rl.size();
  require(R <= BATCH_MAX_RHS, "batch: at most " + std::to_string(BATCH_MAX_RHS) + " right-hand sides");
  const int m = std::min(prm.gcr_k, GCR_MAXK);
  const int clov_any = std::any_of(sys.begin(), sys.end(), [](const BatchSystem &s) { return s.use_clover != 0; });

  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  cudaStream_t st = ctx.stream;
  BatchCache &c = cache();
  int sms = 0;
  QCU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
  QCU_CUDA(cudaDeviceSynchronize());  // inputs written on any stream are complete

  // ---- buffers and sources
  while ((int)c.rhs.size() < R) c.rhs.push_back(std::make_unique<RhsBufs>());
  std::vector<SolveInfo> info(R);
  std::vector<double> bb(R), tol2(R);
  std::vector<int> Vh(R), verified(R, 0);
  int *act = c.active_host;
  for (int r = 0; r < R; r++) {
    const BatchSystem &s = *rl[r].s;
    RhsBufs &B = *c.rhs[r];
    const int vh = s.G->g.Vh;
    Vh[r] = vh;
    for (int k = 0; k < BV_N; k++)  // the inner x stays FP32 under 16-bit spinors
      B.v[k].alloc(k >= BV_INNER_N ? SOA64 : (k == BV_X && kind == SOA16 ? SOA32 : kind), vh);
    for (int k = 0; k < m; k++) {
      B.W[k].alloc(SOA64, vh);
      B.Z[k].alloc(SOA64, vh);
    }
    for (Spinor *q : {&B.be, &B.bo, &B.xe, &B.aux}) q->alloc(SOA64, vh);
    Dsl d64{*s.G, ctx, SOA64};
    const size_t full = 2 * spinor_bytes(AOS64, vh);
    const void *b = static_cast<const char *>(s.b) + full * rl[r].j;
    bb[r] = prepare_source(d64, b, s.kappa, s.use_clover != 0, B.be, B.bo, B.v[BV_BP], B.aux, B.v[BV_TMP64]);
    tol2[r] = prm.tol * prm.tol * bb[r];
    QCU_CUDA(cudaMemsetAsync(B.v[BV_X64].data.p, 0, spinor_bytes(SOA64, vh), st));
    act[r] = bb[r] > 0.0;
    info[r].status = bb[r] > 0.0 ? ST_RUNNING : ST_CONVERGED;
    verified[r] = bb[r] == 0.0;
  }

  // ---- descriptors, tile tables, states
  std::vector<RhsDesc> desc(R);
  for (int r = 0; r < R; r++) {
    const BatchSystem &s = *rl[r].s;
    const GaugeHandle &G = *s.G;
    RhsBufs &B = *c.rhs[r];
    RhsDesc &d = desc[r];
    d = RhsDesc{};
    d.g = G.g;
    d.kappa = s.kappa;
    d.k2 = s.kappa * s.kappa;
    d.t_bc = G.t_bc;
    d.gin = gkind == GSOA64 ? G.g64.p : (gkind == GSOA32 ? G.g32.p : G.g16.p);
    d.g64 = G.g64.p;
    for (int p = 0; p < 2; p++) {
      d.cin[p] = s.use_clover ? G.clover_inv(kind, p) : nullptr;
      d.c64[p] = s.use_clover ? G.clover_inv(SOA64, p) : nullptr;
    }
    for (int k = 0; k < BV_N; k++) {
      d.v[k] = B.v[k].data.p;
      d.vn[k] = B.v[k].norm.as<float>();
    }
    for (int k = 0; k < m; k++) {
      d.W[k] = B.W[k].data.p;
      d.Z[k] = B.Z[k].data.p;
    }
  }
  // partials: enough for the finest table any candidate uses (32 sites per tile)
  size_t max_tiles = 0;
  for (int r = 0; r < R; r++) max_tiles += (Vh[r] + 31) / 32;
  c.partials.ensure(std::max(max_tiles, (size_t)R * BATCH_POST_GRID) * RED_MAXV * sizeof(double));
  c.st.ensure(sizeof(SolverState) * BATCH_MAX_RHS);
  c.active.ensure(sizeof(int) * BATCH_MAX_RHS);
  c.coef.ensure(sizeof(BatchCoef) * BATCH_MAX_RHS);
  c.desc.ensure(sizeof(RhsDesc) * R);

  std::ostringstream key;
  key << kind << "/" << gkind;
  for (int r = 0; r < R; r++) key << ":" << Vh[r] << (rl[r].s->use_clover ? "c" : "");
  const auto found = c.tuned.find(key.str());
  bool need_tune = found == c.tuned.end() && kind != SOA64;
  BatchTune tune;
  if (found != c.tuned.end()) tune = found->second;
  // QCU_BATCH_TUNE="threads,rhs,blas_sites,mma" fixes the tunables (no autotuning)
  if (const char *fix = getenv("QCU_BATCH_TUNE")) {
    BatchTune f;
    require(sscanf(fix, "%d,%d,%d,%d", &f.dslash_threads, &f.dslash_rhs, &f.blas_sites, &f.mma) == 4,
            "QCU_BATCH_TUNE must be threads,rhs,blas_sites,mma");
    require(f.blas_sites >= 128 && f.blas_sites % 128 == 0, "QCU_BATCH_TUNE: blas_sites must be a multiple of 128");
    require(f.dslash_rhs >= 1 && f.dslash_rhs <= BATCH_MAX_NR, "QCU_BATCH_TUNE: rhs per group out of range");
    tune = f;
    need_tune = false;
  }
  if (force_tune) {
    require(force_tune->blas_sites >= 128 && force_tune->blas_sites % 128 == 0,
            "batch: blas_sites must be a multiple of 128");
    require(force_tune->dslash_rhs >= 1 && force_tune->dslash_rhs <= BATCH_MAX_NR, "batch: rhs per group out of range");
    tune = *force_tune;
    need_tune = false;
  }
  const bool tune_log = getenv("QCU_TUNE_LOG") != nullptr;
  if (kind == SOA64) tune.dslash_threads = 128, tune.dslash_rhs = 1, tune.mma = 0;

  // rhs groups of the inner dslash (tune.dslash_rhs consecutive rhs of one
  // system; unused slots repeat the first) and of the FP64 dslash (one each)
  auto make_groups = [&](int nr) {
    std::vector<RhsGroup> gs;
    std::vector<int> gvh;
    int r0 = 0;
    for (const BatchSystem &s : sys) {
      for (int j = 0; j < s.nrhs; j += nr) {
        RhsGroup gp{};
        gp.n = std::min(nr, s.nrhs - j);
        for (int k = 0; k < BATCH_MAX_NR; k++) gp.rhs[k] = r0 + j + std::min(k, gp.n - 1);
        gs.push_back(gp);
        gvh.push_back(s.G->g.Vh);
      }
      r0 += s.nrhs;
    }
    return std::make_pair(gs, gvh);
  };
  BatchArgs A[BT_N];
  auto build_tables = [&]() {
    const int sites[BT_N] = {tune.dslash_threads, tune.blas_sites, 128};
    const auto g_in = make_groups(tune.dslash_rhs), g_one = make_groups(1);
    const std::vector<RhsGroup> *grp[BT_N] = {&g_in.first, nullptr, &g_one.first};
    const std::vector<int> *units[BT_N] = {&g_in.second, &Vh, &g_one.second};
    for (int t = 0; t < BT_N; t++) {
      const std::vector<int2> tiles = make_tiles(*units[t], sites[t]);
      int off = 0;
      for (int r = 0; r < R; r++) {  // per-rhs partials: one per block of its lattice
        desc[r].ntile[t] = (Vh[r] + sites[t] - 1) / sites[t];
        desc[r].poff[t] = off;
        off += desc[r].ntile[t];
      }
      c.tiles[t].ensure(sizeof(int2) * tiles.size());
      QCU_CUDA(cudaMemcpyAsync(c.tiles[t].p, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, st));
      BatchArgs &a = A[t];
      a.d = c.desc.as<RhsDesc>();
      a.tiles = c.tiles[t].as<int2>();
      a.groups = nullptr;
      if (grp[t]) {
        DevBuf &gb = c.groups[t == BT_DSLASH ? 0 : 1];
        gb.ensure(sizeof(RhsGroup) * grp[t]->size());
        QCU_CUDA(cudaMemcpyAsync(gb.p, grp[t]->data(), sizeof(RhsGroup) * grp[t]->size(), cudaMemcpyHostToDevice,
                                 st));
        a.groups = gb.as<RhsGroup>();
        a.ngroups = (int)grp[t]->size();
      }
      a.st = c.st.as<SolverState>();
      a.partials = c.partials.as<double>();
      a.active = c.active.as<int>();
      a.coef = c.coef.as<BatchCoef>();
      a.nrhs = R;
      a.table = t;
      a.ntiles = (int)tiles.size();
      a.tile_sites = sites[t];
      a.sms = sms;
      QCU_CUDA(cudaStreamSynchronize(st));  // the host tables die with this iteration
    }
    QCU_CUDA(cudaMemcpyAsync(c.desc.p, desc.data(), sizeof(RhsDesc) * R, cudaMemcpyHostToDevice, st));
    QCU_CUDA(cudaStreamSynchronize(st));
  };
  build_tables();
  for (int r = 0; r < R; r++) {
    SolverState s0{};
    s0.inner_mode = 1;  // stop at inner_tol or inner_iters
    s0.inner_rel2 = prm.inner_tol * prm.inner_tol;
    s0.maxiter = prm.inner_iters;
    c.st_host[r] = s0;
  }
  QCU_CUDA(cudaMemcpyAsync(c.st.p, c.st_host, sizeof(SolverState) * R, cudaMemcpyHostToDevice, st));
  auto upload_active = [&]() {
    QCU_CUDA(cudaMemcpyAsync(c.active.p, act, sizeof(int) * R, cudaMemcpyHostToDevice, st));
  };
  auto read_states = [&]() {
    QCU_CUDA(cudaMemcpyAsync(c.st_host, c.st.p, sizeof(SolverState) * R, cudaMemcpyDeviceToHost, st));
    QCU_CUDA(cudaStreamSynchronize(st));
    return c.st_host;
  };
  auto upload_coef = [&]() {
    QCU_CUDA(cudaMemcpyAsync(c.coef.p, c.coef_host, sizeof(BatchCoef) * R, cudaMemcpyHostToDevice, st));
  };
  upload_active();

  // ---- operators
  auto inner_dsl = [&](const BDslOp &op) { launch_bdslash(kind, gkind, A[BT_DSLASH], op, tune, st); };
  const BatchTune tune64;  // 128 threads, one rhs per thread
  auto dsl64 = [&](const BDslOp &op) { launch_bdslash(SOA64, GSOA64, A[BT_DSLASH64], op, tune64, st); };
  // r64 = bp - M_pc x64 and |r64|^2 per active rhs (FP64)
  auto true_residual = [&]() {
    BDslOp o0;
    o0.in = BV_X64, o0.out = BV_TMP64, o0.parity = 0, o0.clover = clov_any, o0.gate = BG_ACTIVE;
    dsl64(o0);
    BDslOp o1 = o0;
    o1.in = BV_TMP64, o1.out = BV_R64, o1.parity = 1, o1.a0 = 0, o1.ak2 = 1, o1.x1 = BV_BP, o1.b1 = 1,
    o1.x2 = BV_X64, o1.b2 = -1, o1.red = RED_NORM, o1.fin = FIN_STORE;
    dsl64(o1);
  };

  // ---- autotune, once per batch shape: block size (and the tensor-core
  //      path) of the inner dslash and the BLAS tile size, timed on the fields
  //      of this batch (r = r64 of the zero initial guess)
  if (need_tune) {
    const long long launches0 = launch_count();
    true_residual();
    launch_binit(kind, A[BT_BLAS], st);
    auto time_it = [&](auto &&fn) {
      cudaEvent_t e0, e1;
      QCU_CUDA(cudaEventCreate(&e0));
      QCU_CUDA(cudaEventCreate(&e1));
      fn();
      QCU_CUDA(cudaEventRecord(e0, st));
      for (int i = 0; i < 5; i++) fn();
      QCU_CUDA(cudaEventRecord(e1, st));
      QCU_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      QCU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return (double)ms / 5;
    };
    BDslOp op;
    op.in = BV_R, op.out = BV_TMP, op.parity = 0, op.clover = clov_any;
    BatchTune best = tune;
    double tbest = 1e30;
    // (sites per tile, rhs per group, tensor-core path)
    const int cand[][3] = {{64, 1, 0},  {128, 1, 0}, {256, 1, 0}, {64, 2, 0},
                           {128, 2, 0}, {64, 4, 0},  {128, 4, 0}, {32, 8, 1}};
    for (const auto &cd : cand) {
      tune.dslash_threads = cd[0];
      tune.dslash_rhs = cd[1];
      tune.mma = cd[2];
      double ms = 1e30;
      try {
        build_tables();
        ms = time_it([&]() { inner_dsl(op); });
      } catch (const Error &) {
        cudaGetLastError();  // variant not available for this storage
      }
      if (tune_log) fprintf(stderr, "qcu batch tune: dslash threads %d rhs %d mma %d: %.4f ms\n", cd[0], cd[1], cd[2], ms);
      if (ms < tbest) {
        tbest = ms;
        best.dslash_threads = cd[0];
        best.dslash_rhs = cd[1];
        best.mma = cd[2];
      }
    }
    tune = best;
    tbest = 1e30;
    for (int bs : {128, 256, 512}) {
      tune.blas_sites = bs;
      build_tables();
      const double ms = time_it([&]() { launch_bsupdate(kind, A[BT_BLAS], st); });
      if (tune_log) fprintf(stderr, "qcu batch tune: blas sites %d: %.4f ms\n", bs, ms);
      if (ms < tbest) {
        tbest = ms;
        best.blas_sites = bs;
      }
    }
    tune = best;
    build_tables();
    c.tuned[key.str()] = tune;
    set_launch_count(launches0);  // tuning launches are not part of the solve
  }
  if (tune_out) *tune_out = tune;

  // ---- timing mode: the inner hopping kernel alone, on the odd halves of b
  if (dslash_ms) {
    require(dslash_iters >= 1, "batch dslash timing: iters must be positive");
    for (int r = 0; r < R; r++) {
      const size_t half = spinor_bytes(AOS64, Vh[r]);
      const void *bo = static_cast<const char *>(rl[r].s->b) + 2 * half * rl[r].j + half;
      RhsBufs &B = *c.rhs[r];
      launch_convert(AOS64, kind, Vh[r], bo, nullptr, B.v[BV_P].data.p, B.v[BV_P].norm.as<float>(), st);
    }
    BDslOp d0;
    d0.in = BV_P, d0.out = BV_TMP, d0.parity = 0, d0.clover = clov_any, d0.gate = BG_ALWAYS;
    for (int i = 0; i < 3; i++) inner_dsl(d0);
    cudaEvent_t e0, e1;
    QCU_CUDA(cudaEventCreate(&e0));
    QCU_CUDA(cudaEventCreate(&e1));
    QCU_CUDA(cudaEventRecord(e0, st));
    for (int i = 0; i < dslash_iters; i++) inner_dsl(d0);
    QCU_CUDA(cudaEventRecord(e1, st));
    QCU_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    QCU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *dslash_ms = (double)ms / dslash_iters;
    for (int r = 0; r < R; r++) info[r].status = ST_CONVERGED;
    return info;
  }

  // ---- apply mode: the inner operator of the batched solve, once, as an
  //      operator (the kernels and launch shapes the inner iteration uses)
  if (apply_dots) {
    for (int r = 0; r < R; r++) {
      const size_t half = spinor_bytes(AOS64, Vh[r]);
      const void *bo = static_cast<const char *>(rl[r].s->b) + 2 * half * rl[r].j + half;
      RhsBufs &B = *c.rhs[r];
      for (int k : {BV_P, BV_RT})
        launch_convert(AOS64, kind, Vh[r], bo, nullptr, B.v[k].data.p, B.v[k].norm.as<float>(), st);
    }
    // tmp = [A_e^-1] D_eo p;  v = p - kappa^2 [A_o^-1] D_oe tmp  with <rt, v> (rt = p),
    // then the same with the other fused reduction: t = M_pc p with <t, p>, |t|^2
    BDslOp d0;
    d0.in = BV_P, d0.out = BV_TMP, d0.parity = 0, d0.clover = clov_any, d0.gate = BG_ALWAYS;
    BDslOp d1 = d0;
    d1.in = BV_TMP, d1.out = BV_V, d1.parity = 1, d1.a0 = 0, d1.ak2 = -1, d1.x1 = BV_P, d1.b1 = 1,
    d1.red = RED_DOT_RT, d1.fin = FIN_STORE, d1.rt = BV_RT;
    inner_dsl(d0);
    inner_dsl(d1);
    SolverState *S = read_states();
    for (int r = 0; r < R; r++) apply_dots[5 * r] = S[r].sums[0], apply_dots[5 * r + 1] = S[r].sums[1];
    BDslOp d2 = d1;
    d2.out = BV_T, d2.red = RED_TS_TT, d2.rt = -1;
    inner_dsl(d0);
    inner_dsl(d2);
    S = read_states();
    for (int r = 0; r < R; r++)
      for (int k = 0; k < 3; k++) apply_dots[5 * r + 2 + k] = S[r].sums[k];
    for (int r = 0; r < R; r++) {
      const size_t half = spinor_bytes(AOS64, Vh[r]);
      char *x = static_cast<char *>(rl[r].s->x) + 2 * half * rl[r].j;
      RhsBufs &B = *c.rhs[r];
      launch_convert(kind, AOS64, Vh[r], B.v[BV_TMP].data.p, B.v[BV_TMP].norm.as<float>(), x, nullptr, st);
      launch_convert(kind, AOS64, Vh[r], B.v[BV_V].data.p, B.v[BV_V].norm.as<float>(), x + half, nullptr, st);
      info[r].status = ST_CONVERGED;
    }
    QCU_CUDA(cudaStreamSynchronize(st));
    return info;
  }

  // ---- inner solve graph: init, WHILE(batched BiCGSTAB iteration), z = x
  cudaGraph_t g = nullptr;
  cudaGraphExec_t inner = nullptr;
  const long long launches_before_capture = launch_count();
  {
    const auto mode = cudaStreamCaptureModeThreadLocal;
    QCU_CUDA(cudaGraphCreate(&g, 0));
    try {
      QCU_CUDA(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode));
      launch_binit(kind, A[BT_BLAS], st);
      QCU_CUDA(cudaStreamEndCapture(st, &g));
      cudaGraphNode_t init_node;
      size_t n = 1;
      QCU_CUDA(cudaGraphGetNodes(g, &init_node, &n));
      require(n == 1, "batch inner graph: unexpected init capture");
      cudaGraphConditionalHandle h;
      QCU_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t loop;
      QCU_CUDA(cudaGraphAddNode(&loop, g, &init_node, 1, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      QCU_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode));
      launch_bpupdate(kind, A[BT_BLAS], st);
      BDslOp d0;
      d0.parity = 0, d0.clover = clov_any, d0.gate = BG_NOT_DONE;
      BDslOp d1 = d0;
      d1.parity = 1, d1.a0 = 0, d1.ak2 = -1, d1.b1 = 1;
      d0.in = BV_P, d0.out = BV_TMP;  // v = M_pc p, <rt, v> -> alpha
      d1.in = BV_TMP, d1.out = BV_V, d1.x1 = BV_P, d1.red = RED_DOT_RT, d1.fin = FIN_ALPHA, d1.rt = BV_RT;
      inner_dsl(d0);
      inner_dsl(d1);
      launch_bsupdate(kind, A[BT_BLAS], st);
      d0.in = BV_S;  // t = M_pc s, <t, s>, |t|^2 -> omega
      d1.out = BV_T, d1.x1 = BV_S, d1.red = RED_TS_TT, d1.fin = FIN_OMEGA, d1.rt = -1;
      inner_dsl(d0);
      inner_dsl(d1);
      launch_bxrupdate(kind, A[BT_BLAS], st);
      launch_bloop_cond(A[BT_BLAS], h, (unsigned)prm.inner_iters + 2u, st);
      QCU_CUDA(cudaStreamEndCapture(st, &body));
      QCU_CUDA(cudaStreamBeginCaptureToGraph(st, g, &loop, nullptr, 1, mode));
      launch_bxout(kind, A[BT_BLAS], st);
      QCU_CUDA(cudaStreamEndCapture(st, &g));
      QCU_CUDA(cudaGraphInstantiate(&inner, g, 0));
    } catch (...) {
      cudaStreamCaptureStatus cs;
      if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t junk;
        cudaStreamEndCapture(st, &junk);
      }
      cudaGetLastError();
      cudaGraphDestroy(g);
      set_launch_count(launches_before_capture);
      throw;
    }
    cudaGraphDestroy(g);
    set_launch_count(launches_before_capture);  // replays are counted from the iteration counts
  }

  // ---- outer flexible GCR, all active rhs in step
  BDslOp w0;  // w = M_pc z
  w0.in = BV_Z, w0.out = BV_TMP64, w0.parity = 0, w0.clover = clov_any, w0.gate = BG_ACTIVE;
  BDslOp w1 = w0;
  w1.in = BV_TMP64, w1.out = BV_W, w1.parity = 1, w1.a0 = 0, w1.ak2 = -1, w1.x1 = BV_Z, w1.b1 = 1;
  std::vector<double> nw((size_t)R * GCR_MAXK, 0.0);  // |W_j|^2 per rhs
  auto any_active = [&]() { return std::any_of(act, act + R, [](int a) { return a != 0; }); };
  auto out_ptr = [&](int r) {
    const size_t full = 2 * spinor_bytes(AOS64, Vh[r]);
    return static_cast<void *>(static_cast<char *>(rl[r].s->x) + full * rl[r].j);
  };
  try {
    for (;;) {
      while (any_active()) {
        true_residual();
        SolverState *S = read_states();
        for (int r = 0; r < R; r++) {
          if (!act[r]) continue;
          const double rr = S[r].sums[0];
          if (!(rr == rr)) info[r].status = ST_NAN, act[r] = 0;
          else if (rr <= tol2[r]) info[r].status = ST_CONVERGED, act[r] = 0;
          else if (info[r].iterations >= prm.maxiter) info[r].status = ST_MAXITER, act[r] = 0;
        }
        upload_active();
        for (int k = 0; k < m && any_active(); k++) {
          QCU_CUDA(cudaGraphLaunch(inner, st));
          dsl64(w0);
          dsl64(w1);
          if (k > 0) {
            launch_bgcr_multidot(A[BT_BLAS], k, st);
            S = read_states();
            for (int r = 0; r < R; r++) {
              if (!act[r]) continue;
              for (int j = 0; j < k; j++) {
                c.coef_host[r].beta[2 * j] = S[r].sums[2 * j] / nw[(size_t)r * GCR_MAXK + j];
                c.coef_host[r].beta[2 * j + 1] = S[r].sums[2 * j + 1] / nw[(size_t)r * GCR_MAXK + j];
              }
            }
            upload_coef();
          } else {
            S = read_states();
          }
          int passes = 1;
          for (int r = 0; r < R; r++)
            if (act[r]) {
              info[r].iterations += S[r].iter;
              passes = std::max(passes, S[r].iter + 1);
            }
          note_launch(2 + 8LL * passes);  // the inner graph's kernels
          launch_bgcr_orth(A[BT_BLAS], k, st);
          S = read_states();
          for (int r = 0; r < R; r++) {
            if (!act[r]) continue;
            const double ww = S[r].sums[0];
            if (!(ww > 0.0) || !(ww < 1e300)) {
              info[r].status = ww == ww ? ST_BREAKDOWN : ST_NAN;
              act[r] = 0;
              continue;
            }
            nw[(size_t)r * GCR_MAXK + k] = ww;
            c.coef_host[r].alpha[0] = S[r].sums[1] / ww;
            c.coef_host[r].alpha[1] = S[r].sums[2] / ww;
          }
          upload_active();
          upload_coef();
          launch_bgcr_update(A[BT_BLAS], k, st);
          S = read_states();
          for (int r = 0; r < R; r++) {
            if (!act[r]) continue;
            info[r].iter_residual2 = S[r].sums[0];
            info[r].updates++;
            if (S[r].sums[0] <= tol2[r]) info[r].status = ST_CONVERGED, act[r] = 0;  // verified below
            else if (info[r].iterations >= prm.maxiter) info[r].status = ST_MAXITER, act[r] = 0;
          }
          upload_active();
        }
      }
      // full-system FP64 true residual of every newly converged rhs (and its
      // solution written out); a rhs whose preconditioned residual met its
      // target but whose full residual did not resumes with a tighter target
      bool resumed = false;
      for (int r = 0; r < R; r++) {
        if (verified[r] || info[r].status != ST_CONVERGED) continue;
        const BatchSystem &s = *rl[r].s;
        RhsBufs &B = *c.rhs[r];
        Dsl d64{*s.G, ctx, SOA64};
        const double rr = finish_solution(d64, s.kappa, s.use_clover != 0, B.be, B.bo, B.v[BV_X64], B.xe, B.aux,
                                          B.v[BV_TMP64], out_ptr(r));
        info[r].true_residual = std::sqrt(rr / bb[r]);
        verified[r] = 1;
        if (info[r].true_residual > prm.tol) {
          if (info[r].restarts < 12 && info[r].iterations < prm.maxiter) {
            tol2[r] *= 0.25 * (prm.tol * prm.tol * bb[r]) / std::max(rr, 1e-300);
            info[r].restarts++;
            info[r].status = ST_RUNNING;
            verified[r] = 0;
            act[r] = 1;
            resumed = true;
          } else {
            info[r].status = ST_MAXITER;
          }
        }
      }
      if (!resumed) break;
      upload_active();
    }
  } catch (...) {
    cudaGraphExecDestroy(inner);
    throw;
  }
  cudaGraphExecDestroy(inner);

  // ---- solutions of rhs that stopped without converging, and zero sources
  for (int r = 0; r < R; r++) {
    if (verified[r] && bb[r] > 0.0) continue;
    if (bb[r] == 0.0) {
      QCU_CUDA(cudaMemsetAsync(out_ptr(r), 0, 2 * spinor_bytes(AOS64, Vh[r]), st));
      continue;
    }
    const BatchSystem &s = *rl[r].s;
    RhsBufs &B = *c.rhs[r];
    Dsl d64{*s.G, ctx, SOA64};
    const double rr = finish_solution(d64, s.kappa, s.use_clover != 0, B.be, B.bo, B.v[BV_X64], B.xe, B.aux,
                                      B.v[BV_TMP64], out_ptr(r));
    info[r].true_residual = std::sqrt(rr / bb[r]);
  }
  QCU_CUDA(cudaStreamSynchronize(st));
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (auto &i : info) i.seconds = secs;
  return info;
}

}  // namespace qcu
