// Operator application and the BiCGSTAB driver.
//
// The algorithm is qcu's even-odd preconditioned BiCGSTAB
// (include/lattice_bistabcg.h:101-132,221-340): b'_o = b_o + kappa D_oe b_e,
// solve (1 - kappa^2 D_oe D_eo) x_o = b'_o, then x_e = b_e + kappa D_eo x_o,
// extended with the clover term (A_p^-1 applied after each hop) and with an
// inner precision below FP64 corrected by reliable updates: the FP64 true
// residual b' - M_pc x64 replaces the iterated one whenever the latter has
// dropped by `delta`, and always before convergence is declared.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "gcr.h"
#include "nn.h"
#include "solver.h"
#include "mg.h"

namespace qcu {

int kind_of_precision(int prec) {
  switch (prec) {
    case 64: return SOA64;
    case 32: return SOA32;
    case 16: return SOA16;
  }
  throw Error(1, "precision must be 64, 32 or 16");
}
static int gkind_of(int kind) { return kind == SOA64 ? GSOA64 : (kind == SOA32 ? GSOA32 : GSOA16); }
static int ckind_of(int kind) { return kind == SOA64 ? CSOA64 : CSOA32; }

GaugeHandle *gauge_load(const void *gauge_pyq, const int latt[4], double t_bc, double clover_coeff) {
  require(gauge_pyq != nullptr, "gauge pointer is null");
  require(t_bc == 1.0 || t_bc == -1.0, "t boundary must be +1 or -1");
  Context &ctx = context();
  QCU_CUDA(cudaDeviceSynchronize());  // the field may still be in flight on another stream (an async copy)
  auto *G = new GaugeHandle();
  try {
    for (int d = 0; d < 4; d++) G->latt[d] = latt[d];
    G->g = make_geom(latt);
    G->t_bc = t_bc;
    const int Vh = G->g.Vh;
    G->g64.ensure(gauge_bytes(GSOA64, Vh));
    G->g32.ensure(gauge_bytes(GSOA32, Vh));
    G->g16.ensure(gauge_bytes(GSOA16, Vh));
    launch_gauge_pack(GSOA64, G->g, gauge_pyq, G->g64.p, ctx.stream);
    launch_gauge_pack(GSOA32, G->g, gauge_pyq, G->g32.p, ctx.stream);
    launch_gauge_pack(GSOA16, G->g, gauge_pyq, G->g16.p, ctx.stream);
    if (clover_coeff != 0.0) {
      G->has_clover = true;
      G->clover_coeff = clover_coeff;
      DevBuf bad;
      bad.ensure(sizeof(int));
      QCU_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx.stream));
      for (int p = 0; p < 2; p++) {
        G->A64[p].ensure(clover_bytes(CSOA64, Vh));
        G->Ainv64[p].ensure(clover_bytes(CSOA64, Vh));
        G->Ainv32[p].ensure(clover_bytes(CSOA32, Vh));
        launch_clover_build(G->g, gauge_pyq, p, clover_coeff, G->A64[p].p, G->Ainv64[p].p, bad.as<int>(), ctx.stream);
        launch_clover_to32(Vh, G->Ainv64[p].p, G->Ainv32[p].p, ctx.stream);
      }
      int nbad = 0;
      QCU_CUDA(cudaMemcpyAsync(&nbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
      QCU_CUDA(cudaStreamSynchronize(ctx.stream));
      require(nbad == 0, "clover term is singular on " + std::to_string(nbad) + " site blocks");
    }
    QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  } catch (...) {
    delete G;
    throw;
  }
  return G;
}

// ---------------------------------------------------------------- workspace
namespace {
struct Workspace {
  Spinor be, bo, bp, x64, r64, tmp64, xe, aux;  // FP64
  Spinor r, rt, p, v, s, t, tmp, x;             // inner precision (x: FP64 or FP32)
  void prepare(int kind, int Vh) {
    for (Spinor *q : {&be, &bo, &bp, &x64, &r64, &tmp64, &xe, &aux}) q->alloc(SOA64, Vh);
    for (Spinor *q : {&r, &rt, &p, &v, &s, &t, &tmp}) q->alloc(kind, Vh);
    x.alloc(kind == SOA64 ? SOA64 : SOA32, Vh);
  }
};
Workspace &workspace() { return per_device<Workspace>(context()); }
}  // namespace

void Dsl::operator()(int par, const Spinor &in, Spinor &out, bool clover, double a, const Spinor *x1, double b1,
                     const Spinor *x2, double b2, int red, int fin, const Spinor *rt, int gate) {
  DslashArgs d;
  d.in = in.data.p;
  d.in_norm = in.norm.as<float>();
  d.out = out.data.p;
  d.out_norm = out.norm.as<float>();
  if (x1) {
    d.x1 = x1->data.p;
    d.x1_norm = x1->norm.as<float>();
    d.b1 = b1;
  }
  if (x2) {
    d.x2 = x2->data.p;
    d.x2_norm = x2->norm.as<float>();
    d.b2 = b2;
  }
  if (rt) {
    d.rt = rt->data.p;
    d.rt_norm = rt->norm.as<float>();
  }
  const int gk = gkind >= 0 ? gkind : gkind_of(kind);
  d.gauge = gk == GSOA64 ? G.g64.p : (gk == GSOA32 ? G.g32.p : G.g16.p);
  d.clover = clover ? G.clover_inv(kind, par) : nullptr;
  d.parity = par;
  d.t_bc = G.t_bc;
  d.a = a;
  d.red = red;
  d.fin = fin;
  d.gate = gate;
  launch_dslash(kind, gk, ckind_of(kind), G.g, d, ctx, ctx.stream);
}

static VecSet make_vecset(Workspace &w) {
  VecSet vs;
  vs.r = w.r.data.p;
  vs.rn = w.r.norm.as<float>();
  vs.rt = w.rt.data.p;
  vs.rtn = w.rt.norm.as<float>();
  vs.p = w.p.data.p;
  vs.pn = w.p.norm.as<float>();
  vs.v = w.v.data.p;
  vs.vn = w.v.norm.as<float>();
  vs.s = w.s.data.p;
  vs.sn = w.s.norm.as<float>();
  vs.t = w.t.data.p;
  vs.tn = w.t.norm.as<float>();
  vs.x = w.x.data.p;
  vs.xn = w.x.norm.as<float>();
  vs.x64 = w.x64.data.p;
  vs.r64 = w.r64.data.p;
  return vs;
}

static SolverState read_state(Context &ctx) {
  QCU_CUDA(cudaMemcpyAsync(ctx.st_host, ctx.st, sizeof(SolverState), cudaMemcpyDeviceToHost, ctx.stream));
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  return *ctx.st_host;
}

static double dots_norm2(Context &ctx, int kind, int Vh, void *a, float *an) {
  launch_dots(kind, Vh, a, an, a, an, ctx, ctx.stream);
  return read_state(ctx).sums[2];
}

double prepare_source(Dsl &d64, const void *b_pyq, double kappa, bool clov, Spinor &be, Spinor &bo, Spinor &bp,
                      Spinor &aux, Spinor &tmp64) {
  Context &ctx = d64.ctx;
  const GaugeHandle &G = d64.G;
  const int Vh = G.g.Vh;
  cudaStream_t st = ctx.stream;
  const char *b = static_cast<const char *>(b_pyq);
  launch_convert(AOS64, SOA64, Vh, b, nullptr, be.data.p, nullptr, st);
  launch_convert(AOS64, SOA64, Vh, b + spinor_bytes(AOS64, Vh), nullptr, bo.data.p, nullptr, st);
  if (clov) {
    launch_clover_apply(SOA64, Vh, G.Ainv64[0].p, be.data.p, aux.data.p, st);
    d64(1, aux, tmp64, false, kappa, &bo, 1.0);
    launch_clover_apply(SOA64, Vh, G.Ainv64[1].p, tmp64.data.p, bp.data.p, st);
  } else {
    d64(1, be, bp, false, kappa, &bo, 1.0);
  }
  return dots_norm2(ctx, SOA64, Vh, be.data.p, nullptr) + dots_norm2(ctx, SOA64, Vh, bo.data.p, nullptr);
}

double finish_solution(Dsl &d64, double kappa, bool clov, Spinor &be, Spinor &bo, Spinor &xo, Spinor &xe,
                       Spinor &aux, Spinor &tmp64, void *x_pyq) {
  Context &ctx = d64.ctx;
  const GaugeHandle &G = d64.G;
  const int Vh = G.g.Vh;
  cudaStream_t st = ctx.stream;
  // x_e = A_e^-1 (b_e + kappa D_eo x_o)
  d64(0, xo, tmp64, false, kappa, &be, 1.0);
  if (clov) launch_clover_apply(SOA64, Vh, G.Ainv64[0].p, tmp64.data.p, xe.data.p, st);
  else launch_convert(SOA64, SOA64, Vh, tmp64.data.p, nullptr, xe.data.p, nullptr, st);
  // full-system FP64 true residual: r_p = b_p - A_p x_p + kappa D x_{1-p}
  double rr = 0;
  for (int p = 0; p < 2; p++) {
    Spinor &xp_ = p ? xo : xe;
    Spinor &bpar = p ? bo : be;
    const Spinor *ax = &xp_;
    if (clov) {
      launch_clover_apply(SOA64, Vh, G.A64[p].p, xp_.data.p, aux.data.p, st);
      ax = &aux;
    }
    d64(p, p ? xe : xo, tmp64, false, kappa, &bpar, 1.0, ax, -1.0, RED_NORM, FIN_STORE);
    rr += read_state(ctx).sums[0];
  }
  if (x_pyq) {
    char *x = static_cast<char *>(x_pyq);
    launch_convert(SOA64, AOS64, Vh, xe.data.p, nullptr, x, nullptr, st);
    launch_convert(SOA64, AOS64, Vh, xo.data.p, nullptr, x + spinor_bytes(AOS64, Vh), nullptr, st);
  }
  return rr;
}

// one BiCGSTAB iteration (plus the gated reliable-update sequence)
static void enqueue_iteration(Dsl &dP, Dsl &d64, Workspace &w, const VecSet &vs, double kappa, bool clov) {
  Context &ctx = dP.ctx;
  const int Vh = dP.G.g.Vh, kind = dP.kind;
  const double k2 = kappa * kappa;
  launch_pupdate(kind, Vh, vs, ctx.st, GATE_NOT_DONE, ctx.stream);
  dP(0, w.p, w.tmp, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_NOT_DONE);
  dP(1, w.tmp, w.v, clov, -k2, &w.p, 1.0, nullptr, 0, RED_DOT_RT, FIN_ALPHA, &w.rt, GATE_NOT_DONE);
  launch_supdate(kind, Vh, vs, ctx.st, GATE_NOT_DONE, ctx.stream);
  dP(0, w.s, w.tmp, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_NOT_DONE);
  dP(1, w.tmp, w.t, clov, -k2, &w.s, 1.0, nullptr, 0, RED_TS_TT, FIN_OMEGA, nullptr, GATE_NOT_DONE);
  launch_xrupdate(kind, Vh, vs, ctx, GATE_NOT_DONE, ctx.stream);
  // reliable update: x64 += x; r64 = b' - M_pc x64 (FP64); r = r64
  launch_xfold(w.x.kind, Vh, vs, ctx.st, GATE_UPDATE, ctx.stream);
  d64(0, w.x64, w.tmp64, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_UPDATE);
  d64(1, w.tmp64, w.r64, clov, k2, &w.bp, 1.0, &w.x64, -1.0, RED_NORM, FIN_RTRUE, nullptr, GATE_UPDATE);
  launch_rconv(kind, Vh, vs, ctx, GATE_UPDATE, ctx.stream);
}

// Inner preconditioner solve of the GCR outer loop: BiCGSTAB in the inner
// precision on M_pc z = r64, from zero, until |r| <= inner_tol |r64| or
// inner_iters iterations.  The whole solve (init, iterations, conversion of the
// result to FP64) is one captured graph, replayed once per GCR step: stopping
// is decided on the device (gated launches), so the host never waits on it.
static cudaGraphExec_t capture_inner_solve(Dsl &dP, Workspace &w, const VecSet &vs, double kappa, bool clov,
                                           int iters, Spinor &z_out, long long &nodes) {
  Context &ctx = dP.ctx;
  const int Vh = dP.G.g.Vh, kind = dP.kind;
  const double k2 = kappa * kappa;
  cudaStream_t st = ctx.stream;
  cudaGraph_t graph;
  const long long before = launch_count();
  QCU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    launch_init(kind, Vh, vs, ctx, st);
    for (int k = 0; k < iters; k++) {
      launch_pupdate(kind, Vh, vs, ctx.st, GATE_NOT_DONE, st);
      dP(0, w.p, w.tmp, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_NOT_DONE);
      dP(1, w.tmp, w.v, clov, -k2, &w.p, 1.0, nullptr, 0, RED_DOT_RT, FIN_ALPHA, &w.rt, GATE_NOT_DONE);
      launch_supdate(kind, Vh, vs, ctx.st, GATE_NOT_DONE, st);
      dP(0, w.s, w.tmp, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_NOT_DONE);
      dP(1, w.tmp, w.t, clov, -k2, &w.s, 1.0, nullptr, 0, RED_TS_TT, FIN_OMEGA, nullptr, GATE_NOT_DONE);
      launch_xrupdate(kind, Vh, vs, ctx, GATE_NOT_DONE, st);
    }
    launch_convert(w.x.kind, SOA64, Vh, w.x.data.p, w.x.norm.as<float>(), z_out.data.p, nullptr, st);
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    throw;
  }
  QCU_CUDA(cudaStreamEndCapture(st, &graph));
  nodes = launch_count() - before;
  set_launch_count(before);
  cudaGraphExec_t exec;
  QCU_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  QCU_CUDA(cudaGraphDestroy(graph));
  return exec;
}

// The same inner solve as a graph with a conditional WHILE node: init, then
// the iteration body repeated on the device until the solver state says done
// (converged, breakdown, or inner_iters reached; a guard counter bounds the
// loop in any case), then the conversion.  No empty launches after
// convergence and no host involvement.  `iters_out` is not known at capture
// time: the caller reads st->iter after each replay.
static cudaGraphExec_t capture_inner_solve_while(Dsl &dP, Workspace &w, const VecSet &vs, double kappa, bool clov,
                                                 int iters, Spinor &z_out, long long &per_iter) {
  Context &ctx = dP.ctx;
  const int Vh = dP.G.g.Vh, kind = dP.kind;
  const double k2 = kappa * kappa;
  cudaStream_t st = ctx.stream;
  const auto mode = cudaStreamCaptureModeThreadLocal;
  const long long before = launch_count();
  cudaGraph_t g = nullptr;
  QCU_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphExec_t exec = nullptr;
  try {
    QCU_CUDA(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode));
    launch_init(kind, Vh, vs, ctx, st);
    QCU_CUDA(cudaStreamEndCapture(st, &g));
    cudaGraphNode_t init_node;
    size_t n = 1;
    QCU_CUDA(cudaGraphGetNodes(g, &init_node, &n));
    require(n == 1, "inner solve graph: unexpected init capture");
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
    const long long body0 = launch_count();
    launch_pupdate(kind, Vh, vs, ctx.st, GATE_NOT_DONE, st);
    dP(0, w.p, w.tmp, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_NOT_DONE);
    dP(1, w.tmp, w.v, clov, -k2, &w.p, 1.0, nullptr, 0, RED_DOT_RT, FIN_ALPHA, &w.rt, GATE_NOT_DONE);
    launch_supdate(kind, Vh, vs, ctx.st, GATE_NOT_DONE, st);
    dP(0, w.s, w.tmp, clov, 1.0, nullptr, 0, nullptr, 0, RED_NONE, FIN_STORE, nullptr, GATE_NOT_DONE);
    dP(1, w.tmp, w.t, clov, -k2, &w.s, 1.0, nullptr, 0, RED_TS_TT, FIN_OMEGA, nullptr, GATE_NOT_DONE);
    launch_xrupdate(kind, Vh, vs, ctx, GATE_NOT_DONE, st);
    launch_loop_cond(ctx.st, h, (unsigned)iters + 2u, st);
    per_iter = launch_count() - body0;  // kernels per pass of the loop body
    QCU_CUDA(cudaStreamEndCapture(st, &body));
    QCU_CUDA(cudaStreamBeginCaptureToGraph(st, g, &loop, nullptr, 1, mode));
    launch_convert(w.x.kind, SOA64, Vh, w.x.data.p, w.x.norm.as<float>(), z_out.data.p, nullptr, st);
    QCU_CUDA(cudaStreamEndCapture(st, &g));
    QCU_CUDA(cudaGraphInstantiate(&exec, g, 0));
  } catch (...) {
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk;
      cudaStreamEndCapture(st, &junk);
    }
    cudaGetLastError();
    cudaGraphDestroy(g);
    set_launch_count(before);
    throw;
  }
  cudaGraphDestroy(g);
  set_launch_count(before);  // replays are counted from the iteration count
  return exec;
}

namespace {
struct GcrSpace {
  Spinor W[GCR_MAXK], Z[GCR_MAXK], znew, wnew, zin;
  void prepare(int m, int Vh) {
    for (int j = 0; j < m; j++) {
      W[j].alloc(SOA64, Vh);
      Z[j].alloc(SOA64, Vh);
    }
    znew.alloc(SOA64, Vh);
    wnew.alloc(SOA64, Vh);
    zin.alloc(SOA64, Vh);
  }
};
GcrSpace &gcr_space() { return per_device<GcrSpace>(context()); }
}  // namespace

// Flexible GCR(m) on M_pc in FP64 with the inner solve above as right
// preconditioner: x64/r64 advance until the recursive |r|^2 <= tol2.
static void run_gcr(Dsl &dP, Dsl &d64, Workspace &w, const VecSet &vs, const SolveParams &prm, double tol2,
                    SolveInfo &info) {
  Context &ctx = dP.ctx;
  const int Vh = dP.G.g.Vh;
  const bool clov = prm.use_clover != 0;
  const double kappa = prm.kappa, k2 = kappa * kappa;
  const int m = std::max(1, std::min(prm.gcr_k, GCR_MAXK));
  cudaStream_t st = ctx.stream;
  GcrSpace &gs = gcr_space();
  gs.prepare(m, Vh);
  // inner solver settings stay constant across the GCR steps
  SolverState init{};
  init.inner_mode = 1;
  init.inner_rel2 = prm.inner_tol * prm.inner_tol;
  init.maxiter = prm.inner_iters;
  *ctx.st_host = init;
  QCU_CUDA(cudaMemcpyAsync(ctx.st, ctx.st_host, sizeof(SolverState), cudaMemcpyHostToDevice, st));
  // preconditioner: 0 inner solve z = BiCGSTAB(r); 1 z = N(r) (network);
  // 2 z = N(r) + BiCGSTAB(r - M_pc N(r)); 3 the same with N the multigrid's
  // coarse-grid correction.  The inner solve reads `rin`.
  const int pc = prm.precond;
  require(pc >= 0 && pc <= 3, "solve: precond must be 0, 1, 2 or 3");
  require(pc == 0 || pc == 3 || prm.nn != nullptr, "solve: the network preconditioner needs a network");
  require(pc != 3 || prm.mg != nullptr, "solve: precond 3 needs a multigrid");
  if (pc == 1 || pc == 2) nn_prepare(*prm.nn, Vh);
  if (pc == 3) mg_require_compatible(*prm.mg, dP.G, kappa, prm.use_clover);
  VecSet vin = vs;
  vin.r64 = pc >= 2 ? w.aux.data.p : w.r64.data.p;
  long long nodes = 0;  // 0: device-side WHILE loop (launches counted from the iteration count)
  long long per_iter = 8;  // kernels per pass of the WHILE body (measured at capture)
  cudaGraphExec_t inner = nullptr;
  if (pc != 1) {
    try {
      inner = capture_inner_solve_while(dP, w, vin, kappa, clov, prm.inner_iters, gs.zin, per_iter);
    } catch (const Error &) {
      // conditional graph nodes unavailable: fixed-length capture with gated iterations
      inner = capture_inner_solve(dP, w, vin, kappa, clov, prm.inner_iters, gs.zin, nodes);
    }
  }
  GcrArgs a;
  a.w = gs.wnew.data.p;
  a.z = pc == 0 ? gs.zin.data.p : gs.znew.data.p;
  for (int j = 0; j < m; j++) {
    a.W[j] = gs.W[j].data.p;
    a.Z[j] = gs.Z[j].data.p;
  }
  a.x = w.x64.data.p;
  a.r = w.r64.data.p;
  double nw[GCR_MAXK] = {};  // |W_j|^2
  // Stagnation: a cycle (m outer steps, started from the FP64 true residual)
  // that lowers the best true |r|^2 by less than 1 % counts as stalled;
  // QCU_GCR_STALL_CYCLES such cycles in a row (default 3) end the GCR solve
  // with ST_STALLED, and solve() lets plain FP64 BiCGSTAB finish from x64.
  // (0 declares the stall after the first cycle: the host-side way the tests
  // drive the fallback.)
  const char *stall_env = getenv("QCU_GCR_STALL_CYCLES");
  const int stall_limit = stall_env ? std::max(0, atoi(stall_env)) : 3;
  double best = 0.0;
  int stalled = 0;
  try {
    for (int cycle = 0; info.iterations < prm.maxiter; cycle++) {
      // true residual at the start of every cycle
      d64(0, w.x64, w.tmp64, clov, 1.0);
      d64(1, w.tmp64, w.r64, clov, k2, &w.bp, 1.0, &w.x64, -1.0, RED_NORM, FIN_STORE);
      double rr = read_state(ctx).sums[0];
      if (!(rr == rr)) {
        info.status = ST_NAN;
        break;
      }
      if (rr <= tol2) {
        info.status = ST_CONVERGED;
        break;
      }
      if (cycle > 0) {
        if (rr > 0.99 * best) stalled++;
        else stalled = 0;
        if (stalled >= stall_limit) {
          info.status = ST_STALLED;
          break;
        }
      }
      best = cycle == 0 ? rr : std::min(best, rr);
      for (int k = 0; k < m && rr > tol2 && info.iterations < prm.maxiter; k++) {
        if (pc == 1 || pc == 2) nn_apply_soa64(*prm.nn, dP.G, w.r64.data.p, gs.znew.data.p, st);
        if (pc == 3) mg_coarse_odd(*prm.mg, ctx, w.r64.data.p, gs.znew.data.p);
        if (pc == 2) {  // what the first stage leaves: aux = r - M_pc z
          d64(0, gs.znew, w.tmp64, clov, 1.0);
          d64(1, w.tmp64, w.aux, clov, k2, &w.r64, 1.0, &gs.znew, -1.0);
        } else if (pc == 3) {  // the same after the minimal-residual multiple: aux = M_pc z, then r - alpha aux
          d64(0, gs.znew, w.tmp64, clov, 1.0);
          d64(1, w.tmp64, w.aux, clov, -k2, &gs.znew, 1.0);
          mg_minres_scale(*prm.mg, ctx, gs.znew.data.p, w.aux.data.p, w.r64.data.p);
        }
        if (pc != 1) {
          QCU_CUDA(cudaGraphLaunch(inner, st));
          if (nodes) note_launch(nodes);
        }
        if (pc >= 2) launch_axpby(SOA64, Vh, 1.0, gs.zin.data.p, nullptr, 1.0, gs.znew.data.p, nullptr, st);
        Spinor &zk = pc == 0 ? gs.zin : gs.znew;
        // w = M_pc z
        d64(0, zk, w.tmp64, clov, 1.0);
        d64(1, w.tmp64, gs.wnew, clov, -k2, &zk, 1.0);
        a.k = k;
        if (k > 0) {
          launch_gcr_multidot(Vh, a, ctx, st);
          const SolverState S = read_state(ctx);
          for (int j = 0; j < k; j++) {
            // |W_j|^2 was stored when W_j was made
            a.beta[2 * j] = S.sums[2 * j] / nw[j];
            a.beta[2 * j + 1] = S.sums[2 * j + 1] / nw[j];
          }
          info.iterations += pc == 1 ? 1 : S.iter;  // inner iterations of this step
          if (pc != 1 && !nodes) note_launch(2 + per_iter * std::max(S.iter, 1));
        } else {
          const int it = pc == 1 ? 1 : read_state(ctx).iter;
          info.iterations += it;
          if (pc != 1 && !nodes) note_launch(2 + per_iter * std::max(it, 1));
        }
        launch_gcr_orth(Vh, a, ctx, st);
        SolverState S = read_state(ctx);
        const double ww = S.sums[0];
        if (!(ww > 0.0) || !(ww < 1e300)) {
          info.status = ww == ww ? ST_BREAKDOWN : ST_NAN;
          rr = -1;
          break;
        }
        nw[k] = ww;
        a.alpha[0] = S.sums[1] / ww;
        a.alpha[1] = S.sums[2] / ww;
        launch_gcr_update(Vh, a, ctx, st);
        rr = read_state(ctx).sums[0];
        info.iter_residual2 = rr;
        info.updates++;  // outer (FP64) steps
      }
      if (rr < 0) break;
    }
  } catch (...) {
    if (inner) cudaGraphExecDestroy(inner);
    throw;
  }
  if (inner) cudaGraphExecDestroy(inner);
  if (pc == 3) note_launch(mg_take_launches(*prm.mg, ctx));
  if (info.status == ST_RUNNING && info.iterations >= prm.maxiter) info.status = ST_MAXITER;
}

// BiCGSTAB on M_pc in the inner precision with reliable updates; x64 advances
// until the FP64 true |r|^2 <= tol2 (or a stop condition).  Returns the state.
static SolverState run_bicgstab(Dsl &dP, Dsl &d64, Workspace &w, const VecSet &vs, const SolveParams &prm, double tol2,
                                int maxiter) {
  Context &ctx = dP.ctx;
  const int Vh = dP.G.g.Vh, kind = dP.kind;
  const bool clov = prm.use_clover != 0;
  const double kappa = prm.kappa;
  cudaStream_t st = ctx.stream;
  const int chunk = prm.chunk > 0 ? prm.chunk : (Vh >= (1 << 18) ? 8 : (Vh >= (1 << 14) ? 16 : 32));
  const bool use_graph = getenv("QCU_NO_GRAPH") == nullptr;
  // r64 = b' - M_pc x64
  d64(0, w.x64, w.tmp64, clov, 1.0);
  d64(1, w.tmp64, w.r64, clov, kappa * kappa, &w.bp, 1.0, &w.x64, -1.0, RED_NORM, FIN_RTRUE);
  SolverState init{};
  init.tol2 = tol2;
  init.delta2 = prm.delta * prm.delta;
  init.maxiter = maxiter;
  *ctx.st_host = init;
  QCU_CUDA(cudaMemcpyAsync(ctx.st, ctx.st_host, sizeof(SolverState), cudaMemcpyHostToDevice, st));
  launch_init(kind, Vh, vs, ctx, st);
  SolverState S = read_state(ctx);
  if (!S.done) {
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;
    if (use_graph) {
      cudaGraph_t graph;
      const long long before = launch_count();
      QCU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        for (int k = 0; k < chunk; k++) enqueue_iteration(dP, d64, w, vs, kappa, clov);
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        throw;
      }
      QCU_CUDA(cudaStreamEndCapture(st, &graph));
      nodes = launch_count() - before;  // captured, not run: counted per replay below
      set_launch_count(before);
      QCU_CUDA(cudaGraphInstantiate(&exec, graph, 0));
      QCU_CUDA(cudaGraphDestroy(graph));
    }
    // every iteration advances st->iter, and the iteration that reaches
    // maxiter sets done, so this loop ends after at most maxiter/chunk + 1
    // passes; the cap below only guards against a logic error
    const long long max_passes = (long long)maxiter / chunk + 8;
    try {
      for (long long pass = 0;; pass++) {
        require(pass < max_passes, "solver did not terminate within maxiter (internal error)");
        if (exec) {
          QCU_CUDA(cudaGraphLaunch(exec, st));
          note_launch(nodes);
        } else {
          for (int k = 0; k < chunk; k++) enqueue_iteration(dP, d64, w, vs, kappa, clov);
        }
        S = read_state(ctx);
        if (S.done) break;
      }
    } catch (...) {
      if (exec) cudaGraphExecDestroy(exec);
      throw;
    }
    if (exec) cudaGraphExecDestroy(exec);
  }
  // fold whatever the inner solution still holds (after a NaN the inner
  // partial solution is discarded: x64 is the last good FP64 iterate)
  if (S.status != ST_NAN) launch_xfold(w.x.kind, Vh, vs, ctx.st, GATE_ALWAYS, st);
  return S;
}

SolveInfo solve(GaugeHandle &G, void *x_pyq, const void *b_pyq, const SolveParams &prm) {
  require(x_pyq != nullptr && b_pyq != nullptr, "solve: null spinor pointer");
  require(prm.kappa > 0, "solve: kappa must be positive");
  require(prm.maxiter > 0, "solve: maxiter must be positive");
  require(!prm.use_clover || G.has_clover, "solve: clover requested but the gauge handle has no clover term");
  require(prm.solver == 0 || prm.solver == 1, "solve: solver must be 0 (BiCGSTAB) or 1 (GCR)");
  require(prm.solver == 0 || (prm.inner_iters > 0 && prm.gcr_k > 0 && !prm.abs_tol),
          "solve: GCR needs inner_iters > 0, gcr_k > 0 and a relative tolerance");
  const auto t0 = std::chrono::steady_clock::now();
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  const int kind = kind_of_precision(prm.precision);
  const int Vh = G.g.Vh;
  const bool clov = prm.use_clover != 0;
  const double kappa = prm.kappa;
  Workspace &w = workspace();
  w.prepare(kind, Vh);
  Dsl dP{G, ctx, kind}, d64{G, ctx, SOA64}, dF{G, ctx, SOA64};  // dF: the FP64 fallback's operator
  if (prm.gauge_precision) {
    require(prm.gauge_precision == 16 && kind == SOA32, "solve: gauge_precision 16 is available with precision 32");
    dP.gkind = GSOA16;
  }
  // reduction partials sized once, before any graph capture bakes the pointer in
  ctx.ensure_partials((size_t)std::max((Vh + DSLASH_BLOCK - 1) / DSLASH_BLOCK, MAX_REDUCE_BLOCKS));
  const size_t half = spinor_bytes(AOS64, Vh);
  char *xp = static_cast<char *>(x_pyq);
  cudaStream_t st = ctx.stream;
  QCU_CUDA(cudaDeviceSynchronize());  // inputs written on any stream are complete

  const double bb = prepare_source(d64, b_pyq, kappa, clov, w.be, w.bo, w.bp, w.aux, w.tmp64);
  SolveInfo info;
  if (bb == 0.0) {
    QCU_CUDA(cudaMemsetAsync(x_pyq, 0, 2 * half, st));
    QCU_CUDA(cudaStreamSynchronize(st));
    info.status = ST_CONVERGED;
    return info;
  }
  double tol2 = prm.abs_tol ? prm.tol : prm.tol * prm.tol * bb;

  // initial guess
  if (prm.x0_mode == 1) launch_convert(AOS64, SOA64, Vh, xp + half, nullptr, w.x64.data.p, nullptr, st);
  else if (prm.x0_mode == 2) launch_uniform_soa64(Vh, w.x64.data.p, prm.x0_seed, st);
  else QCU_CUDA(cudaMemsetAsync(w.x64.data.p, 0, spinor_bytes(SOA64, Vh), st));

  VecSet vs = make_vecset(w);
  for (int restart = 0;; restart++) {
    if (prm.solver == 1 && !info.fallback) {
      info.status = ST_RUNNING;
      run_gcr(dP, d64, w, vs, prm, tol2, info);
      if (prm.precond == 1 || prm.precond == 2) nn_check(*prm.nn);
      if ((info.status == ST_STALLED || info.status == ST_BREAKDOWN || info.status == ST_NAN) &&
          info.iterations < prm.maxiter) {
        // the plain solver finishes: FP64 BiCGSTAB from the last FP64 iterate
        // (from zero if that iterate is not finite), judged as always by the
        // FP64 true residual
        if (info.status == ST_NAN) QCU_CUDA(cudaMemsetAsync(w.x64.data.p, 0, spinor_bytes(SOA64, Vh), st));
        info.fallback = 1;
        w.prepare(SOA64, Vh);
        vs = make_vecset(w);
        info.restarts++;
        continue;
      }
    } else {
      SolveParams pb = prm;
      if (info.fallback) pb.delta = 0.0;  // plain: the true residual is recomputed at the end
      const SolverState S = run_bicgstab(info.fallback ? dF : dP, d64, w, vs, pb, tol2, prm.maxiter - info.iterations);
      info.iterations += S.iter;
      info.updates += S.nupdates;
      info.status = S.status;
      info.iter_residual2 = S.rr;
      // BiCGSTAB breakdown (rho, <rt,v> or <t,t> vanishing) or a non-finite
      // inner value: restart from the FP64 iterate with a fresh shadow residual
      if ((S.status == ST_BREAKDOWN || S.status == ST_NAN) && info.restarts < 8 && info.iterations < prm.maxiter) {
        info.restarts++;
        continue;
      }
    }
    const double rr = finish_solution(d64, kappa, clov, w.be, w.bo, w.x64, w.xe, w.aux, w.tmp64, nullptr);
    info.true_residual = std::sqrt(rr / bb);
    const bool relative_ok = prm.abs_tol || info.true_residual <= prm.tol;
    if (info.status != ST_CONVERGED || relative_ok || restart >= 12 || info.iterations >= prm.maxiter) {
      if (info.status == ST_CONVERGED && !relative_ok) info.status = ST_MAXITER;
      break;
    }
    // the preconditioned residual met tol2 but the full one did not: tighten and resume from x64
    tol2 *= 0.25 * (prm.tol * prm.tol * bb) / std::max(rr, 1e-300);
    info.restarts++;
  }
  launch_convert(SOA64, AOS64, Vh, w.xe.data.p, nullptr, xp, nullptr, st);
  launch_convert(SOA64, AOS64, Vh, w.x64.data.p, nullptr, xp + half, nullptr, st);
  QCU_CUDA(cudaStreamSynchronize(st));
  info.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return info;
}

// ---------------------------------------------------------------- operators on a handle
void handle_dslash(GaugeHandle &G, void *out, const void *in, int par, int use_clover, int precision) {
  require(out && in, "dslash: null spinor pointer");
  require(par == 0 || par == 1, "parity must be 0 or 1");
  require(!use_clover || G.has_clover, "dslash: no clover term loaded");
  const bool links16 = precision == 3216;  // FP32 spinors with 16-bit links (the FP32 inner operator)
  const int kind = kind_of_precision(links16 ? 32 : precision);
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  Workspace &w = workspace();
  const int Vh = G.g.Vh;
  w.aux.alloc(SOA64, Vh);
  w.tmp64.alloc(SOA64, Vh);
  w.r.alloc(kind, Vh);
  w.tmp.alloc(kind, Vh);
  Spinor &a = kind == SOA64 ? w.aux : w.r, &b = kind == SOA64 ? w.tmp64 : w.tmp;
  QCU_CUDA(cudaDeviceSynchronize());
  Dsl d{G, ctx, kind, links16 ? GSOA16 : -1};
  launch_convert(AOS64, kind, Vh, in, nullptr, a.data.p, a.norm.as<float>(), ctx.stream);
  d(par, a, b, use_clover != 0, 1.0);
  launch_convert(kind, AOS64, Vh, b.data.p, b.norm.as<float>(), out, nullptr, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
}

void handle_mpc(GaugeHandle &G, void *out, const void *in, double kappa, int use_clover) {
  require(out && in, "mpc: null spinor pointer");
  require(!use_clover || G.has_clover, "mpc: no clover term loaded");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  Workspace &w = workspace();
  const int Vh = G.g.Vh;
  w.aux.alloc(SOA64, Vh);
  w.tmp64.alloc(SOA64, Vh);
  w.r64.alloc(SOA64, Vh);
  QCU_CUDA(cudaDeviceSynchronize());
  Dsl d64{G, ctx, SOA64};
  launch_convert(AOS64, SOA64, Vh, in, nullptr, w.aux.data.p, nullptr, ctx.stream);
  d64(0, w.aux, w.tmp64, use_clover != 0, 1.0);
  d64(1, w.tmp64, w.r64, use_clover != 0, -kappa * kappa, &w.aux, 1.0);
  launch_convert(SOA64, AOS64, Vh, w.r64.data.p, nullptr, out, nullptr, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
}

void handle_mat(GaugeHandle &G, void *out, const void *in, double kappa, int use_clover) {
  require(out && in, "mat: null spinor pointer");
  require(!use_clover || G.has_clover, "mat: no clover term loaded");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  Workspace &w = workspace();
  const int Vh = G.g.Vh;
  for (Spinor *q : {&w.be, &w.bo, &w.tmp64, &w.aux}) q->alloc(SOA64, Vh);
  QCU_CUDA(cudaDeviceSynchronize());
  Dsl d64{G, ctx, SOA64};
  const size_t half = spinor_bytes(AOS64, Vh);
  launch_convert(AOS64, SOA64, Vh, in, nullptr, w.be.data.p, nullptr, ctx.stream);
  launch_convert(AOS64, SOA64, Vh, static_cast<const char *>(in) + half, nullptr, w.bo.data.p, nullptr, ctx.stream);
  for (int p = 0; p < 2; p++) {
    Spinor &xp = p ? w.bo : w.be;
    const Spinor *ax = &xp;
    if (use_clover) {
      launch_clover_apply(SOA64, Vh, G.A64[p].p, xp.data.p, w.aux.data.p, ctx.stream);
      ax = &w.aux;
    }
    d64(p, p ? w.be : w.bo, w.tmp64, false, -kappa, ax, 1.0);
    launch_convert(SOA64, AOS64, Vh, w.tmp64.data.p, nullptr, static_cast<char *>(out) + p * half, nullptr,
                   ctx.stream);
  }
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
}

// ---------------------------------------------------------------- legacy direct path
void legacy_dslash(void *out, const void *in, const void *gauge, const int latt[4], int parity, int clover) {
  require(out && in && gauge, "dslash: null pointer argument");
  require(parity == 0 || parity == 1, "parity must be 0 or 1");
  const Geom g = make_geom(latt);
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  QCU_CUDA(cudaDeviceSynchronize());
  DslashArgs d;
  d.in = in;
  d.out = out;
  d.gauge = gauge;
  d.parity = parity;
  d.t_bc = 1.0;
  d.a = 1.0;
  if (clover && ctx.legacy_clover == nullptr) {  // this device's scratch, reused across calls, never freed
    ctx.legacy_clover = new DevBuf();
    ctx.legacy_bad = new DevBuf();
  }
  DevBuf *cl = ctx.legacy_clover, *bad = ctx.legacy_bad;
  if (clover) {
    // qcu builds the clover of the output parity with unit normalisation on
    // every call (src/nccl_clover_dslash.cu:27-61)
    cl->ensure(clover_bytes(CSOA64, g.Vh));
    bad->ensure(sizeof(int));
    QCU_CUDA(cudaMemsetAsync(bad->p, 0, sizeof(int), ctx.stream));
    launch_clover_build(g, gauge, parity, 1.0, nullptr, cl->p, bad->as<int>(), ctx.stream);
    d.clover = cl->p;
  }
  launch_dslash(AOS64, GAOS64, CSOA64, g, d, ctx, ctx.stream);
  QCU_CUDA(cudaStreamSynchronize(ctx.stream));
  if (clover) {
    int nbad = 0;
    QCU_CUDA(cudaMemcpy(&nbad, bad->p, sizeof(int), cudaMemcpyDeviceToHost));
    require(nbad == 0, "clover term is singular on " + std::to_string(nbad) + " site blocks");
  }
}

}  // namespace qcu
