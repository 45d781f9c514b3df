// Batched solves: many right-hand sides, on one or several lattices of
// uneven volume, advanced together.
//
// Every batched kernel runs over a tile table: tile k = (rhs, block b of that
// rhs's sites).  One launch covers all right-hand sides of all lattices; a
// right-hand side's scalars live in its own SolverState, its reductions end
// in the last block of its own tiles (per-rhs ticket), and converged
// right-hand sides drop out of every launch on their own (gates).  Tiles are
// ordered so that the right-hand sides sharing a lattice visit the same
// sites at the same time: the links they all read come from DRAM once and
// from L2 for the others.
#pragma once
#include <vector>

#include "gcr.h"
#include "solver.h"

namespace qcu {

constexpr int BATCH_MAX_RHS = 64;
constexpr int BATCH_MAX_NR = 8;  // right-hand sides per dslash group
constexpr int BATCH_POST_GRID = 148 * 8;  // largest grid of a kernel that reduces once per block

// right-hand sides of one system that the dslash advances together: one
// thread per site computes all of them, decoding each link once
struct RhsGroup {
  int n;
  int rhs[BATCH_MAX_NR];
};

// per-rhs vectors (roles); the first group is stored in the inner precision
enum BVec {
  BV_R = 0, BV_RT, BV_P, BV_V, BV_S, BV_T, BV_TMP, BV_X,  // inner precision (x: FP32 under 16-bit spinors)
  BV_R64, BV_Z, BV_TMP64, BV_W, BV_X64, BV_BP,          // FP64
  BV_N
};
constexpr int BV_INNER_N = BV_R64;

struct RhsDesc {
  Geom g;
  int ntile[3];  // tiles of this rhs in each tile table (BatchTable)
  int poff[3];   // offset of its partials (in tiles) in each table
  double kappa, k2, t_bc;
  const void *gin, *g64;        // links: inner storage, FP64
  const void *cin[2], *c64[2];  // inverse clover per output parity (inner, FP64); null without clover
  void *v[BV_N];
  float *vn[BV_N];              // per-site norms of 16-bit spinors (null otherwise)
  void *W[GCR_MAXK], *Z[GCR_MAXK];
};

// GCR coefficients of one step for every rhs, written by the host
struct BatchCoef {
  double beta[2 * GCR_MAXK];
  double alpha[2];
};

enum BatchGate { BG_ALWAYS = 0, BG_NOT_DONE = 1, BG_ACTIVE = 2 };
// tile tables: the inner dslash (tuned block size), the BLAS kernels (tuned
// tile size), the FP64 dslash (128 sites per tile)
enum BatchTable { BT_DSLASH = 0, BT_BLAS = 1, BT_DSLASH64 = 2, BT_N = 3 };

struct BatchArgs {
  const RhsDesc *d = nullptr;     // [nrhs]
  const int2 *tiles = nullptr;    // [ntiles] (rhs, block); dslash tables: (group, block)
  const RhsGroup *groups = nullptr;  // dslash tables: the groups tiles refer to
  int ngroups = 0;
  SolverState *st = nullptr;      // [nrhs]
  double *partials = nullptr;     // [tiles of the finest table][RED_MAXV]
  const int *active = nullptr;    // [nrhs]
  const BatchCoef *coef = nullptr;  // [nrhs]
  int nrhs = 0;
  int table = 0;                  // BatchTable of `tiles`
  int ntiles = 0;
  int tile_sites = 128;           // sites per tile
  int sms = 148;                  // SMs of the device (grid of the persistent kernels)
};

// One batched hopping-term application:
//   v[out] = a * [A^-1] D_{par <- 1-par} v[in] + b1 v[x1] + b2 v[x2]
// with a = a0 + ak kappa + ak2 kappa^2 of each rhs, and an optional fused
// reduction (the RedKind of the single-rhs kernel) finalised per rhs.
struct BDslOp {
  int in = -1, out = -1, x1 = -1, x2 = -1, rt = -1;
  int parity = 0;
  double a0 = 1, ak = 0, ak2 = 0, b1 = 0, b2 = 0;
  int red = RED_NONE, fin = FIN_STORE, gate = BG_ALWAYS;
  int clover = 0;  // apply the inverse clover of rhs that have one
};

// tunables chosen per batch shape by the autotuner
struct BatchTune {
  int dslash_threads = 128;  // sites per dslash tile: 64, 128 or 256 (one thread each); 32 for the tensor-core path
  int dslash_rhs = 1;        // right-hand sides per dslash thread: 1, 2 or 4 (8 rhs per warp: tensor cores)
  int blas_sites = 256;      // sites per BLAS tile (128 threads each)
  int mma = 0;               // tensor-core contraction for the inner dslash: 1 3xTF32 (FP32-accurate), 2 TF32
};

void launch_bdslash(int kind, int gkind, const BatchArgs &a, const BDslOp &op, const BatchTune &t, cudaStream_t s);
// inner BiCGSTAB iteration, batched (gates: BG_NOT_DONE on each rhs's state)
void launch_bpupdate(int kind, const BatchArgs &a, cudaStream_t s);
void launch_bsupdate(int kind, const BatchArgs &a, cudaStream_t s);
void launch_bxrupdate(int kind, const BatchArgs &a, cudaStream_t s);
// r = rt = r64 (inner precision), p = v = x = 0; FIN_INIT per rhs; inactive rhs start done
void launch_binit(int kind, const BatchArgs &a, cudaStream_t s);
// z = x (inner solution to FP64), active rhs only
void launch_bxout(int kind, const BatchArgs &a, cudaStream_t s);
// WHILE condition over all rhs states (guard: at most cap passes)
void launch_bloop_cond(const BatchArgs &a, cudaGraphConditionalHandle h, unsigned cap, cudaStream_t s);
// outer GCR step, FP64, active rhs only
void launch_bgcr_multidot(const BatchArgs &a, int k, cudaStream_t s);
void launch_bgcr_orth(const BatchArgs &a, int k, cudaStream_t s);
void launch_bgcr_update(const BatchArgs &a, int k, cudaStream_t s);

// one system of a batched solve: nrhs full spinors (PyQuda layout,
// contiguous, device) solved on one gauge handle
struct BatchSystem {
  GaugeHandle *G = nullptr;
  int nrhs = 0;
  double kappa = 0;
  int use_clover = 0;
  void *x = nullptr;
  const void *b = nullptr;
};

// Flexible GCR(gcr_k) per rhs in FP64, preconditioned by a batched inner
// BiCGSTAB (precision 16 with 16-bit links, 32 with 32- or 16-bit links, or
// 64) over all rhs of all systems,
// captured once as a CUDA graph with a device-side WHILE loop.  One SolveInfo
// per rhs, in system order.
// force_tune: use these tunables (no autotuning).  apply_dots: instead of
// solving, apply the batched inner operator once per rhs (apply mode, below)
// and write 5 doubles per rhs there.
// dslash_ms: instead of solving, time the inner hopping kernel (first half of
// M_pc on the odd halves of b, dslash_iters launches, CUDA events) and write
// the mean time per launch there.
std::vector<SolveInfo> solve_batch(const std::vector<BatchSystem> &sys, const SolveParams &prm, BatchTune *tune_out,
                                   const BatchTune *force_tune = nullptr, double *apply_dots = nullptr,
                                   double *dslash_ms = nullptr, int dslash_iters = 0);

}  // namespace qcu
