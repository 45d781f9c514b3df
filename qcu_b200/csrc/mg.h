// Two-level adaptive aggregation multigrid for the full Wilson or clover
// operator M = A - kappa D.  Parameter names and defaults follow PyQuda's
// multigrid set-up (python/PyQuda/pyquda/dslash/general.py:121-230, defaults
// from dslash/wilson.py:24: coarse_tol 0.1, coarse_maxiter 12, nu_pre 0,
// nu_post 8; two levels with geo_block_size 4 x 4 x 4 x 4).
#pragma once
#include "solver.h"

namespace qcu {

struct MGParams {
  int geo_block_size[4] = {4, 4, 4, 4};  // aggregate extent in x (full), y, z, t
  int n_vec = 12;                        // near-null vectors (coarse degrees of freedom per aggregate: 2 n_vec)
  int setup_maxiter = 48;                // iterations of the solve that makes each near-null vector
  double coarse_tol = 0.1;               // coarse BiCGSTAB: relative residual target
  int coarse_maxiter = 12;               // coarse BiCGSTAB: iteration cap
  int nu_pre = 0;                        // MR smoothing steps before the coarse correction
  int nu_post = 8;                       // MR smoothing steps after it
  int gcr_k = 8;                         // outer flexible GCR: directions kept before a restart
};

struct MGInfo {
  int outer = 0;         // outer GCR steps (one two-level cycle each)
  int coarse_iters = 0;  // coarse BiCGSTAB iterations, summed over the cycles
  int status = 0;        // ST_CONVERGED, ST_MAXITER, ST_BREAKDOWN or ST_NAN
  double true_residual = 0;  // ||b - M x|| / ||b||, FP64
  double seconds = 0;
};

struct MG;
// builds the near-null vectors, the prolongator and the coarse operator on
// the current device (with the handle's clover term when it has one)
MG *mg_create(GaugeHandle &G, double kappa, const MGParams &p);
void mg_free(MG *mg);
// x, b: full PyQuda-layout spinors (complex128, device); x starts from zero
MGInfo mg_solve(MG &mg, void *x, const void *b, double tol, int maxiter);
// |P^dag P c - c| / |c| and |A_c c - P^dag M P c| / |P^dag M P c| for a seeded coarse c
void mg_check(MG &mg, double *orth_err, double *galerkin_err);
double mg_setup_seconds(const MG &mg);

// The coarse-grid correction as a preconditioner of the even-odd system
// M_pc x_o = b_o (solve()'s precond 3): z_o = the odd part of P A_c^-1 P^dag
// applied to (0, A_o r_o), i.e. A_c's approximation of M_pc^-1 r_o (S^-1 of
// the Schur complement S = A_o - kappa^2 D_oe A_e^-1 D_eo, M_pc = A_o^-1 S).
// r_odd, z_odd: FP64 site-blocked half spinors (SOA64); queued on ctx's
// stream, the caller holds ctx.mu.
void mg_coarse_odd(MG &mg, Context &ctx, const void *r_odd, void *z_odd);
// with q = M_pc z on entry: alpha = <q, r> / |q|^2 (the minimal-residual
// multiple of the correction), z *= alpha, q = r - alpha q; returns alpha
double2 mg_minres_scale(MG &mg, Context &ctx, void *z, void *q, const void *r);
// throws unless mg was built on G for this kappa, with the clover term iff G has one
void mg_require_compatible(const MG &mg, const GaugeHandle &G, double kappa, int use_clover);
// kernels the coarse solves launched since the last call (read from the device)
long long mg_take_launches(MG &mg, Context &ctx);

}  // namespace qcu
