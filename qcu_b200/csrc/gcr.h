// Flexible GCR outer-solver kernels.
#pragma once
#include "internal.h"

namespace qcu {

constexpr int GCR_MAXK = 16;  // longest GCR cycle (Krylov vectors kept before a restart)

struct GcrArgs {
  const void *w = nullptr;  // new direction image (M_pc z), FP64 component-major
  const void *z = nullptr;  // new direction
  void *W[GCR_MAXK] = {};   // stored images, W[k] receives the orthogonalised w
  void *Z[GCR_MAXK] = {};   // stored directions
  void *x = nullptr, *r = nullptr;
  double beta[2 * GCR_MAXK] = {};
  double alpha[2] = {0, 0};
  int k = 0;
};

void launch_gcr_multidot(int Vh, const GcrArgs &a, Context &ctx, cudaStream_t s);
void launch_gcr_orth(int Vh, const GcrArgs &a, Context &ctx, cudaStream_t s);
void launch_gcr_update(int Vh, const GcrArgs &a, Context &ctx, cudaStream_t s);

}  // namespace qcu
