// Solver state kept in device memory, and the block/grid reduction used by
// every kernel that produces an inner product.
//
// A reduction never waits on other blocks: each block writes its partial
// sums, bumps a ticket, and the block that draws the last ticket sums the
// partials in a fixed order (deterministic) and applies the BiCGSTAB scalar
// recurrence for that step ("finalize").  Scalars therefore never leave the
// GPU during a solve; the host only polls `done` between chunks of iterations.
#pragma once
#include "cplx.cuh"

namespace qcu {

enum SolverStatus { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXITER = 2, ST_BREAKDOWN = 3, ST_NAN = 4, ST_STALLED = 5 };

constexpr int RED_MAXV = 40;  // largest number of doubles one reduction produces (partials stride)

struct SolverState {
  double rho[2], rho_prev[2], alpha[2], omega[2], beta[2];
  double rr;       // iterated ||r||^2 of the current inner residual
  double rr_max;   // largest true ||r||^2 since the last reliable update
  double rr_true;  // last FP64 true ||r||^2
  double tol2;     // stop when the FP64 true ||r||^2 <= tol2
  double delta2;   // reliable update when rr <= delta2 * rr_max (0: only at the end)
  double inner_rel2;  // inner mode: stop when rr <= inner_rel2 * rr(start)
  double sums[RED_MAXV];  // result of the last FIN_STORE reduction
  int iter, maxiter, done, update, status, nupdates;
  int inner_mode;  // 1: a preconditioner solve (no reliable updates, stops on inner_rel2)
  unsigned ticket;
  unsigned loop_guard;  // body executions of a device-side WHILE loop since the last init
};

// gate modes: which kernels of a captured iteration actually run
enum Gate { GATE_ALWAYS = 0, GATE_NOT_DONE = 1, GATE_UPDATE = 2 };

__device__ __forceinline__ bool gate_open(const SolverState *st, int gate) {
  if (gate == GATE_ALWAYS || st == nullptr) return true;
  volatile const SolverState *v = st;
  if (gate == GATE_NOT_DONE) return v->done == 0;
  return v->update != 0 && v->done == 0;
}

enum FinOp {
  FIN_STORE = 0,  // sums -> st->sums
  FIN_ALPHA,      // alpha = rho / <rt, v>
  FIN_OMEGA,      // omega = <t, s> / <t, t>
  FIN_XR,         // rho_prev = rho; rho = <rt, r>; rr = |r|^2; iteration bookkeeping
  FIN_RTRUE,      // rr_true = |r64|^2
  FIN_RCONV,      // rho = <rt, r>; rr = rr_max = rr_true; end of a reliable update
  FIN_INIT        // rho = <rt, r>; rr = rr_max = rr_true = |r|^2; scalars reset
};

__device__ __forceinline__ bool bad_number(double v) { return !(v == v) || v > 1e300 || v < -1e300; }

__device__ inline void finalize(SolverState *st, int op, const double *s) {
  switch (op) {
    case FIN_STORE:
      for (int k = 0; k < RED_MAXV; k++) st->sums[k] = s[k];
      break;
    case FIN_ALPHA: {
      Cpx<double> den(s[0], s[1]);
      if (den.norm2() == 0.0 || bad_number(s[0]) || bad_number(s[1])) {
        st->status = ST_BREAKDOWN;
        st->done = 1;
        break;
      }
      Cpx<double> a = cdiv(Cpx<double>(st->rho[0], st->rho[1]), den);
      st->alpha[0] = a.re;
      st->alpha[1] = a.im;
      break;
    }
    case FIN_OMEGA: {
      if (s[2] == 0.0 || bad_number(s[2])) {
        st->status = bad_number(s[2]) ? ST_NAN : ST_BREAKDOWN;
        st->done = 1;
        break;
      }
      st->omega[0] = s[0] / s[2];
      st->omega[1] = s[1] / s[2];
      break;
    }
    case FIN_XR: {
      st->rho_prev[0] = st->rho[0];
      st->rho_prev[1] = st->rho[1];
      st->rho[0] = s[0];
      st->rho[1] = s[1];
      st->rr = s[2];
      st->iter += 1;
      if (bad_number(s[2])) {
        st->status = ST_NAN;
        st->done = 1;
      } else if (s[2] <= st->tol2 || s[2] <= st->delta2 * st->rr_max) {
        if (st->inner_mode) {
          st->status = ST_CONVERGED;
          st->done = 1;
        } else {
          st->update = 1;  // fold x, recompute the FP64 true residual
        }
      } else if (s[0] == 0.0 && s[1] == 0.0) {
        st->status = ST_BREAKDOWN;
        st->done = 1;
      }
      if (!st->done && st->iter >= st->maxiter) {
        st->status = ST_MAXITER;
        st->done = 1;
      }
      break;
    }
    case FIN_RTRUE:
      st->rr_true = s[0];
      break;
    case FIN_RCONV:
      st->rho[0] = s[0];
      st->rho[1] = s[1];
      st->rr = st->rr_true;
      st->rr_max = st->rr_true;
      st->update = 0;
      st->nupdates += 1;
      if (bad_number(st->rr_true)) {
        st->status = ST_NAN;
        st->done = 1;
      } else if (st->rr_true <= st->tol2) {
        st->status = ST_CONVERGED;
        st->done = 1;
      }
      break;
    case FIN_INIT:
      st->rho[0] = s[0];
      st->rho[1] = s[1];
      st->rho_prev[0] = 1.0;
      st->rho_prev[1] = 0.0;
      st->alpha[0] = 1.0;
      st->alpha[1] = 0.0;
      st->omega[0] = 1.0;
      st->omega[1] = 0.0;
      st->beta[0] = 0.0;
      st->beta[1] = 0.0;
      st->rr = s[2];
      st->rr_max = s[2];
      st->rr_true = s[2];
      st->update = 0;
      st->iter = 0;
      st->nupdates = 0;
      st->loop_guard = 0;
      if (st->inner_mode) st->tol2 = st->inner_rel2 * s[2];
      if (bad_number(s[2])) {
        st->status = ST_NAN;
        st->done = 1;
      } else if (s[2] <= st->tol2) {
        st->status = ST_CONVERGED;
        st->done = 1;
      } else {
        st->status = ST_RUNNING;
        st->done = 0;
      }
      break;
  }
}

// Inner products of one site's 12 complex components.  The site's partial is
// formed in the arithmetic type T of the storage (FP32 for FP32 and 16-bit
// fields: 12 terms) and added to the FP64 accumulator once; sums across sites
// (thread, block, grid) are FP64.  Converting every term to FP64 instead costs
// ~100 FP64-pipe instructions per site, a third of an issue-bound kernel.
template <typename T>
__device__ __forceinline__ void site_dot(const Cpx<T> a[12], const Cpx<T> b[12], double &re, double &im) {
  if constexpr (sizeof(T) == 8) {  // FP64 fields: every term straight into the accumulator
#pragma unroll
    for (int c = 0; c < 12; c++) {
      re += a[c].re * b[c].re + a[c].im * b[c].im;
      im += a[c].re * b[c].im - a[c].im * b[c].re;
    }
  } else {
    T sr = 0, si = 0;
#pragma unroll
    for (int c = 0; c < 12; c++) {
      sr += a[c].re * b[c].re + a[c].im * b[c].im;
      si += a[c].re * b[c].im - a[c].im * b[c].re;
    }
    re += (double)sr;
    im += (double)si;
  }
}
template <typename T>
__device__ __forceinline__ void site_norm2(const Cpx<T> a[12], double &n2) {
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int c = 0; c < 12; c++) n2 += a[c].re * a[c].re + a[c].im * a[c].im;
  } else {
    T s = 0;
#pragma unroll
    for (int c = 0; c < 12; c++) s += a[c].re * a[c].re + a[c].im * a[c].im;
    n2 += (double)s;
  }
}

struct RedCtx {
  SolverState *st;
  double *partials;  // value-major: value k of block b at [k * gridDim.x + b] (room for RED_MAXV values)
  int op;
};


__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum NV values over the block into `out` (valid in thread 0).  BS = blockDim.x.
template <int NV, int BS>
__device__ __forceinline__ void block_sum(double v[NV], double out[NV]) {
  __shared__ double sh[BS / 32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) sh[w][k] = v[k];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double q = lane < BS / 32 ? sh[lane][k] : 0.0;
      q = warp_sum(q);
      out[k] = q;
    }
  }
  __syncthreads();
}

// Sum of n partials (value-major, n per value) by the whole block, into
// tot (valid in thread 0).  Plain L2 loads (the partials were written by
// other blocks of this grid before their ticket), issued independently so
// the block keeps many in flight; the order of the sum is fixed.
template <int NV, int BS>
__device__ __forceinline__ void sum_partials(const double *P, int n, double tot[NV]) {
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) acc[k] = 0.0;
#pragma unroll 4
  for (int b = threadIdx.x; b < n; b += BS) {
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] += __ldcg(P + (size_t)k * n + b);
  }
  block_sum<NV, BS>(acc, tot);
}

// Block partial -> global partials; the last block to arrive reduces all
// partials in block order and runs the finalize op.
template <int NV, int BS>
__device__ __forceinline__ void grid_reduce(double v[NV], const RedCtx &rc) {
  __shared__ bool last;
  double part[NV];
  block_sum<NV, BS>(v, part);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) rc.partials[(size_t)k * gridDim.x + blockIdx.x] = part[k];
    __threadfence();
    unsigned t = atomicAdd(&rc.st->ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double tot[NV];
  sum_partials<NV, BS>(rc.partials, (int)gridDim.x, tot);
  if (threadIdx.x == 0) {
    double s[RED_MAXV];
#pragma unroll
    for (int k = 0; k < RED_MAXV; k++) s[k] = k < NV ? tot[k] : 0.0;
    finalize(rc.st, rc.op, s);
    rc.st->ticket = 0;
    __threadfence();
  }
}

}  // namespace qcu
