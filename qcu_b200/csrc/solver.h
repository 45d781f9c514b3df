// Gauge handles, operator application and the BiCGSTAB driver.
#pragma once
#include "internal.h"

namespace qcu {

// A gauge field resident on the device in every storage the kernels use,
// plus (optionally) the clover term and its inverse on both parities.
struct GaugeHandle {
  int latt[4];
  Geom g;
  double t_bc = 1.0;
  DevBuf g64, g32, g16;
  bool has_clover = false;
  double clover_coeff = 0.0;
  DevBuf A64[2], Ainv64[2], Ainv32[2];
  const void *gauge(int kind) const {
    return kind == SOA64 ? g64.p : (kind == SOA32 ? g32.p : g16.p);
  }
  const void *clover_inv(int kind, int par) const {
    if (!has_clover) return nullptr;
    return kind == SOA64 ? Ainv64[par].p : Ainv32[par].p;
  }
};

GaugeHandle *gauge_load(const void *gauge_pyq, const int latt[4], double t_bc, double clover_coeff);

struct SolveParams {
  double kappa = 0.125;
  double tol = 1e-10;       // relative: ||b - M x|| <= tol ||b|| (full system, FP64)
  int maxiter = 10000;
  int precision = 64;       // inner precision: 64, 32, 16
  double delta = 0.1;       // reliable update when |r| < delta * max|r| since the last one (0: at the end only)
  int abs_tol = 0;          // 1: qcu's criterion, iterated ||r_pc||^2 < tol
  int x0_mode = 0;          // 0 zero, 1 caller's x, 2 uniform(0,1] from x0_seed
  uint64_t x0_seed = 0;
  int use_clover = 0;
  int chunk = 0;            // iterations per captured graph (0: automatic)
  int solver = 0;           // 0 BiCGSTAB (reliable updates), 1 flexible GCR with an inner BiCGSTAB
  int inner_iters = 16;     // GCR: iterations of the inner solve per step
  double inner_tol = 0.1;   // GCR: inner solve stops at |r| <= inner_tol |r_outer|
  int gcr_k = 8;            // GCR: directions kept before a restart (<= 16)
  int gauge_precision = 0;  // 0: links stored like the spinors; 16 with precision 32: 16-bit links
  int precond = 0;          // GCR: 0 inner BiCGSTAB, 1 network, 2 network then inner BiCGSTAB,
                            // 3 multigrid coarse-grid correction then inner BiCGSTAB
  struct NNet *nn = nullptr;
  struct MG *mg = nullptr;  // precond 3: built on the same handle and kappa
};

struct SolveInfo {
  int iterations = 0;
  int updates = 0;           // BiCGSTAB: reliable updates; GCR: outer steps
  int status = 0;
  int restarts = 0;
  double true_residual = 0;  // ||b - M x|| / ||b||, FP64, full two-parity system
  double iter_residual2 = 0; // last iterated ||r_pc||^2
  double seconds = 0;
  int fallback = 0;          // GCR stalled or broke down; plain FP64 BiCGSTAB finished
};

// x, b: full two-parity spinors, PyQuda layout, complex128, device
SolveInfo solve(GaugeHandle &G, void *x, const void *b, const SolveParams &p);

int kind_of_precision(int prec);

// One hopping-term application on a handle's fields in a given storage:
//   out = a * [Ainv_par] D_{par <- 1-par} in + b1 x1 + b2 x2 (+ fused reduction)
struct Dsl {
  const GaugeHandle &G;
  Context &ctx;
  int kind;
  int gkind = -1;  // gauge storage; -1: the one matching the spinor kind
  void operator()(int par, const Spinor &in, Spinor &out, bool clover, double a, const Spinor *x1 = nullptr,
                  double b1 = 0, const Spinor *x2 = nullptr, double b2 = 0, int red = RED_NONE, int fin = FIN_STORE,
                  const Spinor *rt = nullptr, int gate = GATE_ALWAYS);
};

// b (PyQuda full spinor, device) -> be, bo (FP64 internal) and the even-odd
// source bp = A_o^-1 (b_o + kappa D_oe A_e^-1 b_e); returns |b|^2.
// (include/lattice_bistabcg.h:101-106 for the Wilson case)
double prepare_source(Dsl &d64, const void *b_pyq, double kappa, bool clov, Spinor &be, Spinor &bo, Spinor &bp,
                      Spinor &aux, Spinor &tmp64);
// x_e = A_e^-1 (b_e + kappa D_eo x_o) and the full-system FP64 true |b - M x|^2;
// also writes x (PyQuda layout) when x_pyq is not null
// (include/lattice_bistabcg.h:313-332 for the Wilson case)
double finish_solution(Dsl &d64, double kappa, bool clov, Spinor &be, Spinor &bo, Spinor &xo, Spinor &xe,
                       Spinor &aux, Spinor &tmp64, void *x_pyq);

// out = D_{par <- 1-par} in on PyQuda-layout half spinors (optionally A^-1 D),
// computed in the given storage precision (64, 32, 16; 3216 = FP32 spinors with
// 16-bit links) on the packed gauge
void handle_dslash(GaugeHandle &G, void *out, const void *in, int par, int use_clover, int precision);
// out = M_pc in (odd parity, PyQuda-layout half spinors)
void handle_mpc(GaugeHandle &G, void *out, const void *in, double kappa, int use_clover);
// out = M in on full PyQuda spinors (M = A - kappa D, A = 1 for Wilson)
void handle_mat(GaugeHandle &G, void *out, const void *in, double kappa, int use_clover);

// legacy single dslash straight on PyQuda buffers (no packing, no allocation)
void legacy_dslash(void *out, const void *in, const void *gauge, const int latt[4], int parity, int clover);

}  // namespace qcu
