// Domain decomposition over a grid of ranks (ncclDslashQcu with grid != 1^4).
#pragma once
#include <vector>

#include "internal.h"

namespace qcu {

constexpr int DD_FACE_COMPLEX = 6;  // a face site carries a half spinor: 2 spins x 3 colours

// One rank's place in the grid (qcu's mapping, include/lattice_set.h:89-128):
// rank = ((gx * Gy + gy) * Gz + gz) * Gt + gt, periodic neighbours.
struct DDPlan {
  int nranks = 1, rank = 0;
  int latt[4];    // local lattice {Lx, Ly, Lz, Lt}
  int grid[4];
  int coord[4];
  int fwd[4], bwd[4];  // neighbour ranks in each direction
  int face[4];         // face sites of one parity per partitioned direction (0: not partitioned)
};
DDPlan dd_plan(const int latt[4], const int grid[4], int rank);

// One step of the face exchange.  Slot 0 of direction d: the low face
// (x_d = 0), projected for the backward rank's forward hops; slot 1: the high
// face, multiplied by this rank's links for the forward rank's backward hops.
// A rank sends its slots and receives the matching ones into its halo: halo
// slot 0 comes from the forward rank, slot 1 from the backward rank.
enum DDOpKind { DD_SEND = 0, DD_RECV = 1 };
struct DDOp {
  int kind;
  int dir;
  int slot;
  int peer;
  int count;  // complex numbers
};
// every rank's operations, in the order every rank issues them
std::vector<DDOp> dd_schedule(const DDPlan &p);

// all ranks of `grid` in this process on one device, faces exchanged by
// device copies; *_all hold the ranks' local fields back to back (rank order)
void dd_dslash_emulate(void *out_all, const void *in_all, const void *gauge_all, const int latt[4], int parity,
                       const int grid[4]);
// this rank's part, faces exchanged with NCCL over the device's communicator
void dd_dslash_nccl(void *out, const void *in, const void *gauge, const int latt[4], int parity, const int grid[4]);
// qcu's solver (ncclBistabCgQcu) on the grid: x, b full spinors of every
// domain of this process (all ranks when emulating, back to back), stop on
// the grid-wide iterated ||r_o||^2 < tol (absolute) or maxiter
struct DDSolveResult {
  int iterations = 0;
  double r2 = 0;
};
DDSolveResult dd_solve(void *x, const void *b, const void *gauge, const int latt[4], const int grid[4], bool emulate,
                       double kappa, double tol, int maxiter, uint64_t seed);
void dd_unique_id(void *id);  // 128 bytes
void dd_comm_init(const void *id, int nranks, int rank);
void dd_comm_free();

}  // namespace qcu
