// Device-side helpers shared by the batched kernels (batch.cu, batch_mma.cu).
#pragma once
#include "batch.h"

namespace qcu {

template <int K>
using Real = typename SpinorReal<K>::T;

__device__ __forceinline__ bool bgate(const BatchArgs &a, int rhs, int gate) {
  if (gate == BG_ALWAYS) return true;
  if (gate == BG_ACTIVE) return a.active[rhs] != 0;
  return ((volatile const SolverState *)(a.st + rhs))->done == 0;
}

// Once the last tile of a rhs has written its partial: the whole block sums
// that rhs's partials in tile order and applies the finalize op to its state.
template <int NV, int BS>
__device__ __forceinline__ void batch_finish(const BatchArgs &a, int rhs, int op) {
  const RhsDesc &d = a.d[rhs];
  const double *P = a.partials + (size_t)d.poff[a.table] * RED_MAXV;
  const int n = d.ntile[a.table];
  SolverState *st = a.st + rhs;
  __threadfence();
  double tot[NV];
  sum_partials<NV, BS>(P, n, tot);
  if (threadIdx.x == 0) {
    double s[RED_MAXV];
#pragma unroll
    for (int k = 0; k < RED_MAXV; k++) s[k] = k < NV ? tot[k] : 0.0;
    finalize(st, op, s);
    st->ticket = 0;
    __threadfence();
  }
}

// partial of tile b of one rhs -> its partials (value k of tile b at
// [k * ntile + b] in the rhs's region); returns (to every thread of
// the block) whether this was the rhs's last tile.  `part` valid in thread 0.
__device__ __forceinline__ bool batch_post(const BatchArgs &a, int rhs, int b, const double *part, int nv,
                                           bool *flag) {
  if (threadIdx.x == 0) {
    const RhsDesc &d = a.d[rhs];
    double *P = a.partials + (size_t)d.poff[a.table] * RED_MAXV;  // this rhs's region, value-major
    for (int k = 0; k < nv; k++) P[(size_t)k * d.ntile[a.table] + b] = part[k];
    __threadfence();
    const unsigned t = atomicAdd(&a.st[rhs].ticket, 1u);
    *flag = (t == (unsigned)d.ntile[a.table] - 1u);
  }
  __syncthreads();
  return *flag;
}

// block partial of one rhs -> its partials; the last of its tiles finishes it
template <int NV, int BS>
__device__ __forceinline__ void batch_reduce(double v[NV], const BatchArgs &a, int rhs, int b, int op) {
  __shared__ bool last;
  double part[NV];
  block_sum<NV, BS>(v, part);
  if (batch_post(a, rhs, b, part, NV, &last)) batch_finish<NV, BS>(a, rhs, op);
}

template <int K>
__device__ __forceinline__ SpinorView<K> bview(const RhsDesc &d, int role) {
  return SpinorView<K>{d.v[role], d.vn[role], d.g.Vh};
}

}  // namespace qcu
