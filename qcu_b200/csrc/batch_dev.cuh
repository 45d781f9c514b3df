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

// ---- persistent tile loop.  The gate of a rhs changes only in the finalize
// at the end of a launch, so each block evaluates every rhs's gate once, and
// copies the rhs groups, into shared memory; it then reads its tiles
// TILE_CHUNK at a time with one load per thread.  A tile of a closed rhs
// costs a few shared-memory reads instead of dependent global loads.
constexpr int TILE_CHUNK = 128;
struct BlockBatch {
  bool open[BATCH_MAX_RHS];
  RhsGroup grp[BATCH_MAX_RHS];
  int2 tiles[TILE_CHUNK];
};

__device__ __forceinline__ void block_batch_init(const BatchArgs &a, BlockBatch &bb, int gate) {
  for (int r = threadIdx.x; r < a.nrhs; r += blockDim.x) bb.open[r] = bgate(a, r, gate);
  if (a.groups)
    for (int g = threadIdx.x; g < a.ngroups; g += blockDim.x) bb.grp[g] = a.groups[g];
  __syncthreads();
}

// body(tile) for the tiles blockIdx.x, blockIdx.x + gridDim.x, ... in order
template <typename F>
__device__ __forceinline__ void for_tiles(const BatchArgs &a, BlockBatch &bb, F &&body) {
  const long G = gridDim.x;
  for (long k0 = blockIdx.x; k0 < a.ntiles; k0 += G * TILE_CHUNK) {
    __syncthreads();  // the previous chunk is done with bb.tiles
    for (int t = threadIdx.x; t < TILE_CHUNK; t += blockDim.x) {
      const long k = k0 + t * G;
      bb.tiles[t] = k < a.ntiles ? a.tiles[k] : make_int2(-1, 0);
    }
    __syncthreads();
    for (int t = 0; t < TILE_CHUNK; t++) {
      const int2 tile = bb.tiles[t];
      if (tile.x < 0) break;  // uniform: shared memory
      body(tile);
    }
  }
}

// The whole block sums n partials of one rhs (value-major at P) in a fixed
// order and applies the finalize op to its state.
template <int NV, int BS>
__device__ __forceinline__ void batch_finish_at(const BatchArgs &a, int rhs, int op, const double *P, int n) {
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

// Once the last tile of a rhs has written its partial: finish from the
// per-tile partials of that rhs.
template <int NV, int BS>
__device__ __forceinline__ void batch_finish(const BatchArgs &a, int rhs, int op) {
  const RhsDesc &d = a.d[rhs];
  batch_finish_at<NV, BS>(a, rhs, op, a.partials + (size_t)d.poff[a.table] * RED_MAXV, d.ntile[a.table]);
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

// ---- reductions of the per-iteration kernels: per block, not per tile.
// While a persistent block walks its tiles, each warp adds its warp-summed
// share to its own shared-memory slot of the tile's rhs (no barrier, no
// atomic, fixed order).  At the end the block posts one partial for every
// open rhs (zero for a rhs it never touched) and takes that rhs's ticket; the
// block that draws a rhs's last ticket sums the gridDim.x partials and
// finalises it.  Partials: rhs r owns RED_MAXV * BATCH_POST_GRID doubles at
// r * RED_MAXV * BATCH_POST_GRID, value-major with stride gridDim.x.
template <int NV, int NW>
struct WarpRed {
  double v[NW][BATCH_MAX_RHS][NV];
};

template <int NV, int NW>
__device__ __forceinline__ void warp_red_zero(WarpRed<NV, NW> &w) {
  double *p = &w.v[0][0][0];
  for (int i = threadIdx.x; i < NW * BATCH_MAX_RHS * NV; i += blockDim.x) p[i] = 0.0;
  __syncthreads();
}

// add this warp's share of a tile of `rhs` (every lane calls, with its values)
template <int NV, int NW>
__device__ __forceinline__ void warp_red_add(WarpRed<NV, NW> &w, int rhs, double (&v)[NV]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    const double t = warp_sum(v[k]);
    if (lane == 0) w.v[warp][rhs][k] += t;
  }
}

template <int NV, int NW>
__device__ __forceinline__ void warp_red_post(const BatchArgs &a, WarpRed<NV, NW> &w, int op, int gate) {
  __shared__ bool last[BATCH_MAX_RHS];
  __syncthreads();  // every warp's shares are in
  for (int r = threadIdx.x; r < a.nrhs; r += blockDim.x) {
    bool l = false;
    if (bgate(a, r, gate)) {
      double *P = a.partials + (size_t)r * RED_MAXV * BATCH_POST_GRID;
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < NW; q++) t += w.v[q][r][k];
        P[(size_t)k * gridDim.x + blockIdx.x] = t;
      }
      __threadfence();
      l = atomicAdd(&a.st[r].ticket, 1u) == gridDim.x - 1u;
    }
    last[r] = l;
  }
  __syncthreads();
  for (int r = 0; r < a.nrhs; r++)
    if (last[r]) batch_finish_at<NV, NW * 32>(a, r, op, a.partials + (size_t)r * RED_MAXV * BATCH_POST_GRID, gridDim.x);
}

template <int K>
__device__ __forceinline__ SpinorView<K> bview(const RhsDesc &d, int role) {
  return SpinorView<K>{d.v[role], d.vn[role], d.g.Vh};
}

}  // namespace qcu
