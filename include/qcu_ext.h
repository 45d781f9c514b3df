/*
 * qcu_ext.h -- additive extension ABI of the B200 implementation.
 *
 * qcu's own ABI (qcu.h) fixes kappa = 0.125, an absolute tolerance, FP64,
 * periodic boundaries and rebuilds everything on every call.  These entry
 * points expose the same path with its parameters: a gauge field (and clover
 * term) loaded once and kept on the device, any kappa, a relative FP64
 * true-residual tolerance, an inner precision of 64/32/16 bits with reliable
 * updates, the t boundary phase, and solver statistics.
 *
 * Same data conventions as qcu.h: device pointers, complex128, PyQuda layout,
 * lattice {Lx, Ly, Lz, Lt}, parity = output parity.  Every function returns
 * 0 on success and a non-zero code on error (1 bad argument, 2 CUDA error,
 * 3 internal), with the message available from qcuGetLastError().
 */
#ifndef QCU_B200_QCU_EXT_H
#define QCU_B200_QCU_EXT_H

#include "qcu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qcuGauge_s *qcuGauge;
typedef struct qcuNN_s *qcuNN;  /* learned preconditioner (see qcuNNCreate) */
typedef struct qcuMG_s *qcuMG;  /* two-level multigrid (see qcuMGCreate) */

/* last error of the calling thread: returns its code, copies the message */
int qcuGetLastError(char *msg, int len);
int qcuVersion(void);

/* Load a gauge field (PyQuda layout) onto the device as reconstruct-12
 * storage in FP64, FP32 and 16-bit fixed point.  t_boundary = +1 periodic, -1 antiperiodic
 * in time (applied in the stencil, so the links stay SU(3)).  clover_coeff
 * != 0 also builds the clover term A = 1 - coeff/8 sum_{mu<nu} gamma_mu
 * gamma_nu (Q_munu - Q_munu^dag) and its inverse on both parities; coeff =
 * kappa*csw is the Sheikholeslami-Wohlert term, coeff = 1 is qcu's clover
 * (src/clover_dslash.cu:826-835). */
int qcuGaugeLoad(qcuGauge *h, const void *gauge, const int latt[4], double t_boundary, double clover_coeff);
int qcuGaugeFree(qcuGauge h);

/* half spinors: out(parity) = [A_parity^{-1}] D_{parity <- 1-parity} in, computed
 * with the field stored in `precision` bits (64, 32, or 16 = int16 fixed point + per-site
 * norm; accumulation in FP64 resp. FP32), or 3216 = FP32 spinors with 16-bit links;
 * input and output stay complex128 */
int qcuDslash(qcuGauge h, void *out, const void *in, int parity, int use_clover, int precision);
/* odd-parity Schur operator M_pc = 1 - kappa^2 [A_o^-1] D_oe [A_e^-1] D_eo */
int qcuMatPC(qcuGauge h, void *out, const void *in, double kappa, int use_clover);
/* full operator on full spinors, M = A - kappa D (A = 1 for Wilson) */
int qcuMat(qcuGauge h, void *out, const void *in, double kappa, int use_clover);

typedef struct {
  double kappa;
  double tol;            /* stop when ||b - M x|| <= tol ||b|| (FP64, full system) */
  int maxiter;
  int precision;         /* inner precision: 64, 32 or 16 (int16 + per-site norm) */
  double delta;          /* reliable update threshold (0.1 typical; 0 = only at the end) */
  int abs_tol;           /* 1: qcu's test, iterated ||r_o||^2 < tol */
  int x0_mode;           /* 0 zero, 1 use x on input, 2 uniform (0,1] from x0_seed */
  unsigned long long x0_seed;
  int use_clover;
  int chunk;             /* iterations per captured CUDA graph (0 = automatic) */
  int solver;            /* 0 BiCGSTAB with reliable updates; 1 flexible GCR (FP64) whose
                            preconditioner is an inner BiCGSTAB in `precision` */
  int inner_iters;       /* GCR: inner iterations per step */
  double inner_tol;      /* GCR: inner stop at |r| <= inner_tol |r_outer| */
  int gcr_k;             /* GCR: directions kept before a restart (<= 16) */
  int gauge_precision;   /* 0: links stored like the spinors; 16 (with precision 32): FP32
                            spinors and 16-bit links in the inner operator */
  int precond;           /* GCR preconditioner: 0 inner BiCGSTAB; 1 the network `nn`;
                            2 the network, then the inner BiCGSTAB on what it leaves;
                            3 the multigrid `mg`'s coarse-grid correction, then the inner
                            BiCGSTAB on what it leaves (mg built on this handle and kappa) */
  qcuNN nn;
  qcuMG mg;
} qcuInvertParam;

typedef struct {
  int iterations;
  int reliable_updates;  /* BiCGSTAB: reliable updates; GCR: outer steps */
  int status;            /* 1 converged, 2 max iterations, 3 breakdown, 4 NaN/Inf */
  int restarts;
  double true_residual;  /* ||b - M x|| / ||b||, recomputed in FP64 at the end */
  double iter_residual2; /* last iterated ||r_o||^2 */
  double seconds;
  int fallback;          /* 1: the GCR solve stalled or broke down, and plain FP64 BiCGSTAB,
                            started from its last FP64 iterate, finished the solve */
} qcuInvertResult;

void qcuInvertParamDefault(qcuInvertParam *p);
/* x, b: full spinors.  Even-odd preconditioned BiCGSTAB on the odd sites. */
int qcuInvert(qcuGauge h, void *x, const void *b, const qcuInvertParam *p, qcuInvertResult *r);

/* One system of a batched solve: nrhs right-hand sides on one gauge handle.
 * x and b hold nrhs full spinors back to back ([nrhs][2][Vh][4][3]
 * complex128, PyQuda layout, device). */
typedef struct {
  qcuGauge gauge;
  int nrhs;
  double kappa;
  int use_clover;
  void *x;
  const void *b;
} qcuBatchSystem;

/* Tunables the batched solver chose for this batch shape (autotuned on the
 * first solve of a shape, reused afterwards). */
typedef struct {
  int dslash_threads;  /* sites per block of the inner dslash (64, 128, 256) */
  int dslash_rhs;      /* right-hand sides each dslash thread computes (1, 2, 4) */
  int blas_sites;      /* sites per block of the vector kernels */
  int mma;             /* 1: the inner dslash uses the tensor-core contraction */
} qcuBatchTune;

/* Batched solve of every right-hand side of every system (at most 64 in
 * total; lattices may differ in size): flexible GCR(gcr_k) in FP64 per
 * right-hand side around one inner BiCGSTAB (precision 16 -- 16-bit spinors
 * and links --, 32 -- with 16-bit links when gauge_precision is 16 -- or 64)
 * that advances all right-hand
 * sides together, one kernel launch per step for the whole batch, captured
 * as one CUDA graph.  Uses kappa/use_clover of each system (the param's are
 * ignored), tol, maxiter (inner iterations per rhs), precision,
 * gauge_precision, inner_iters, inner_tol and gcr_k; x0_mode must be 0 and
 * abs_tol 0.  results: one per right-hand side, in system order (may be
 * null); tune: optional. */
int qcuInvertBatch(const qcuBatchSystem *systems, int n_systems, const qcuInvertParam *p, qcuInvertResult *results,
                   qcuBatchTune *tune);

/* Timing of the batched solver's inner hopping kernel (no counterpart in
 * qcu): the odd halves of every b_j are stored in the inner precision and the
 * kernel of the first half of M_pc runs `iters` times on them; *ms = mean
 * device time per launch (CUDA events).  tune: null or dslash_threads <= 0 =
 * let the autotuner choose (the choice is written back); else that shape. */
int qcuBatchDslashTime(const qcuBatchSystem *systems, int n_systems, int precision, int gauge_precision,
                       qcuBatchTune *tune, int iters, double *ms);

/* Multi-right-hand-side hopping term on the tcgen05 tensor cores (no
 * counterpart in qcu, whose dslash takes one spinor): out_j = D_{parity <-
 * 1-parity} in_j for j < nrhs (1..128), in/out = nrhs half spinors back to
 * back ([nrhs][Vh][4][3] complex128, PyQuda layout, device).  Per site and
 * hop one tensor-core product serves every right-hand side: spinors are
 * rounded to FP16 once, B = real form of (1 -+ gamma_mu) x U in FP16 (from the
 * 16-bit links), FP32 accumulation; the result is rounded to FP16 (about
 * 1e-3 relative, against 1e-6 for the FP32 hop).  Two FP16 work fields of
 * Vh x 48 x (64 or 128) bytes are kept per device for reuse (the library's
 * memory pool). */
int qcuDslashMultiTC(qcuGauge h, void *out, const void *in, int nrhs, int parity);
/* its kernel alone, on resident seeded multi-rhs fields: *ms = mean device
 * time per application over `iters` launches (CUDA events) */
int qcuDslashMultiTCTime(qcuGauge h, int nrhs, int parity, int iters, double *ms);

/* Operator check of the batched solver's inner kernels (no counterpart in
 * qcu, whose solver takes one right-hand side).  For every right-hand side j
 * of every system, the odd half b_o of b_j is stored in the inner precision
 * (precision / gauge_precision as for qcuInvertBatch), and the batched
 * hopping kernels of the inner solve, launched with the tunables `tune`
 * (sites per block, right-hand sides per thread, tensor-core mode 0/1/2),
 * compute, written to x_j as complex128:
 *   even half  [A_e^-1] D_eo b_o                       (first half of M_pc)
 *   odd half   M_pc b_o = b_o - kappa^2 [A_o^-1] D_oe [A_e^-1] D_eo b_o
 * with both fused reductions of the inner iteration:
 *   dots[5i+0..1] = <b_o, M_pc b_o>, dots[5i+2..3] = <M_pc b_o, b_o>,
 *   dots[5i+4] = |M_pc b_o|^2                          (rhs i in system order).
 * Clover is applied for systems with use_clover. */
int qcuBatchApplyMatPC(const qcuBatchSystem *systems, int n_systems, int precision, int gauge_precision,
                       const qcuBatchTune *tune, double *dots);

/* seeded generators, PyQuda layout complex128 on the device.
 * gauge kind: 0 Haar SU(3), 1 exp(i eps H) reunitarised, 2 unit links.
 * fermion kind: 0 complex normal N(0,1) per component, 1 uniform (0,1]. */
int qcuGaugeRandom(void *gauge, const int latt[4], int kind, double eps, unsigned long long seed);
int qcuFermionRandom(void *psi, long long n_complex, int kind, unsigned long long seed);

/* dslashCloverQcu for callers that cannot allocate device memory.  This entry
 * point has no counterpart in the reference.  Callers such as a framework
 * whose caching allocator already holds its device-memory budget, a job under
 * a hard device-memory cap, or a latency-critical path cannot afford a
 * cudaMalloc; this variant keeps the inverse clover field it needs in a
 * static device array (18 MiB, held by every GPU that loads the library) and
 * allocates nothing.  Same arguments and result as dslashCloverQcu; returns 0
 * on success, non-zero with qcuGetLastError() set otherwise.
 *  - at most qcuNoAllocMaxSites() = 32768 sites per parity (a 16^4 lattice);
 *    larger lattices are rejected with an error;
 *  - the driver reserves the array on a device when the library's device code
 *    is first used there (lazy module loading, the CUDA 12 default; at load
 *    time under CUDA_MODULE_LOADING=EAGER): under a hard memory cap, make the
 *    first call early;
 *  - every call synchronises the device and runs on the legacy default
 *    stream: make no call while a stream of the process is being captured;
 *    a call cannot be captured;
 *  - all calls share the scratch: calls that overlap on the GPU race. */
int dslashCloverQcuNoAlloc(void *fermion_out, void *fermion_in, void *gauge, QcuParam *param, int parity);
int qcuNoAllocMaxSites(void);

/* ---- Several GPUs: ncclDslashQcu with grid != {1,1,1,1} (qcu's domain
 * decomposition, src/nccl_wilson_dslash.cu:3-19, include/lattice_dslash.h:11-197).
 * Every rank (one process per GPU) passes its local sub-lattice in PyQuda
 * layout, `param` = the local lattice size (every extent even) and `grid` =
 * ranks per direction; rank r sits at qcu's grid coordinate
 * (include/lattice_set.h:89-95: t fastest, rank = ((gx*Gy+gy)*Gz+gz)*Gt+gt).
 * Faces of half spinors are exchanged with NCCL point-to-point over a
 * communicator made once per device: one rank calls qcuCommUniqueId, the id
 * (128 bytes) reaches every rank by the launcher's own means (MPI, a
 * torch.distributed broadcast, ...), then each rank calls qcuCommInit with
 * its rank.  NCCL (libnccl.so.2) is loaded on first use. */
int qcuCommUniqueId(void *id);
int qcuCommInit(const void *id, int nranks, int rank);
int qcuCommFree(void);
/* this rank's plan: [nranks, rank, coord[4], fwd[4], bwd[4], face[4]] (22
 * ints; face = sites of one parity on the face of each partitioned direction,
 * 0 elsewhere); needs no GPU */
int qcuDDPlan(const int latt[4], const int grid[4], int rank, int *plan);
/* the face exchange this rank carries out, in order: n_ops entries of 5 ints
 * (kind 0 send / 1 recv, direction, slot, peer rank, complex count); slot 0
 * of a direction is the low face (sent to the backward rank, received from
 * the forward one), slot 1 the high face (sent forward, received from
 * backward); at most 16 entries; needs no GPU */
int qcuDDSchedule(const int latt[4], const int grid[4], int rank, int *ops, int *n_ops);
/* every rank of `grid` at once in this process on the current GPU, faces
 * exchanged by device copies following each rank's schedule: the same
 * kernels as ncclDslashQcu without a second GPU.  *_all hold the ranks'
 * local fields back to back in rank order. */
int qcuDslashDDEmulate(void *out_all, const void *in_all, const void *gauge_all, const int latt[4], int parity,
                       const int grid[4]);
/* ncclBistabCgQcu's solve over `grid` for every rank at once in this process
 * (full spinors and gauges back to back in rank order): qcu's kappa 0.125,
 * random start (seed 23333, each element fixed by its global site, so the
 * start equals the single-GPU one on the global lattice) and stop on the
 * grid-wide iterated ||r_o||^2 < 1e-9 or 1000 iterations.  Reports the
 * iterations and the final ||r_o||^2. */
int qcuBistabCgDDEmulate(void *x_all, const void *b_all, const void *gauge_all, const int latt[4], const int grid[4],
                         int *iterations, double *r2);

/* Learned preconditioner: a gauge-equivariant parallel-transport network
 * approximating M_pc^{-1} on the odd sites.  Two layers, 4 -> 16 -> 4
 * colour-vector channels (12 complex -> 48 -> 12 per site); each layer sums
 * the identity and the 8 link transports of its input, each mixed by a
 * complex channel matrix.  FP32 arithmetic, FP32 master weights with a bf16
 * copy used for inference.  Weights are qcuNNNumParams() floats (complex
 * pairs, layer 1 [9][16][4] then layer 2 [9][4][16]).  Starts as the identity
 * plus noise of scale init_scale. */
int qcuNNCreate(qcuNN *net, unsigned long long seed, double init_scale);
int qcuNNFree(qcuNN net);
int qcuNNNumParams(void);
int qcuNNGetWeights(qcuNN net, float *w);
int qcuNNSetWeights(qcuNN net, const float *w);
/* out = N(in) on odd-parity half spinors (complex128 PyQuda layout).
 * Inference (this call and the GCR preconditioner) runs each layer's channel
 * mixing on the tensor cores: tcgen05 BF16 MMAs with FP32 accumulators in
 * tensor memory, the parallel transports rounded to bf16 as the A operand;
 * qcuNNSetTensorCores(net, 0) selects the FP32 FMA layers instead. */
int qcuNNApply(qcuNN net, qcuGauge h, void *out, const void *in);
int qcuNNSetTensorCores(qcuNN net, int on);
/* One training step on a batch of (residual r_i, error e_i) odd half spinors
 * ([batch][Vh][4][3] complex128): loss = mean_i |N(r_i) - e_i|^2 / |e_i|^2,
 * gradients by the hand-written backward kernels, then an Adam step with
 * learning rate lr (lr = 0: gradient only).  grad (optional, host) receives
 * dL/dW* as qcuNNNumParams() floats. */
int qcuNNTrainStep(qcuNN net, qcuGauge h, const void *r, const void *e, int batch, double lr, double *loss,
                   float *grad);

/* Two-level adaptive aggregation multigrid for the full operator
 * M = A - kappa D (Wilson, or clover when the handle has a clover term).
 * No counterpart in qcu, whose src/multgrid.cu is empty; the parameters are
 * those PyQuda passes to QUDA's multigrid (python/PyQuda/pyquda/dslash/
 * general.py:121-230), the defaults its Wilson and clover dslash classes use
 * (dslash/wilson.py:24) with two levels and fewer near-null vectors.
 * Set-up: n_vec near-null vectors (each the error left by setup_maxiter
 * iterations of FP32 BiCGSTAB on M y = M v0, v0 Gaussian), orthonormalised
 * on every aggregate of geo_block_size sites and chirality, and the Galerkin
 * coarse operator P^dag M P (2 n_vec complex degrees of freedom per
 * aggregate).  Solve: FP64 flexible GCR(gcr_k) on the full system, each step
 * preconditioned by nu_pre MR steps, the coarse correction (FP32 BiCGSTAB to
 * coarse_tol, at most coarse_maxiter iterations) and nu_post MR steps. */
typedef struct {
  int geo_block_size[4]; /* aggregate extents x (full), y, z, t; the x extent even, the
                            product a multiple of 32 and at most 512, each dividing the lattice */
  int n_vec;             /* near-null vectors, 1..16 */
  int setup_maxiter;
  double coarse_tol;
  int coarse_maxiter;
  int nu_pre;
  int nu_post;
  int gcr_k;             /* outer GCR directions kept before a restart, 1..32 */
} qcuMGParam;
typedef struct {
  int outer;             /* outer GCR steps (one two-level cycle each) */
  int coarse_iters;      /* coarse BiCGSTAB iterations, summed */
  int status;            /* 1 converged, 2 max outer steps, 3 breakdown, 4 NaN/Inf */
  double true_residual;  /* ||b - M x|| / ||b||, FP64 */
  double seconds;
} qcuMGResult;
void qcuMGParamDefault(qcuMGParam *p);
/* the gauge handle must outlive the multigrid; set-up runs on the current device */
int qcuMGCreate(qcuMG *mg, qcuGauge h, double kappa, const qcuMGParam *p, double *setup_seconds);
int qcuMGFree(qcuMG mg);
/* x, b: full spinors (PyQuda layout, complex128, device); x starts from zero;
 * stops at ||b - M x|| <= tol ||b|| or maxiter outer steps */
int qcuMGInvert(qcuMG mg, void *x, const void *b, double tol, int maxiter, qcuMGResult *r);
/* set-up checks on a seeded coarse vector c: |P^dag P c - c| / |c| and
 * |A_c c - P^dag M P c| / |P^dag M P c| */
int qcuMGCheck(qcuMG mg, double *orth_err, double *galerkin_err);

/* number of kernels this library has launched in this process (graph
 * replays count every node) */
long long qcuKernelLaunches(void);

/* the library's CUDA stream on the current device (for event timing) */
void *qcuGetStream(void);

/* Kernel timing: `iters` back-to-back applications of the internal-layout
 * hopping term (spinor precision 64/32/16, link precision 0 = same or 16 with
 * FP32 spinors, optionally with the clover inverse) on random input,
 * alternating parities, timed with CUDA events on the library stream.
 * Returns the mean milliseconds per application. */
int qcuBenchDslash(qcuGauge h, int precision, int gauge_precision, int use_clover, int iters, double *ms_per_call);

#ifdef __cplusplus
}
#endif

#endif
