// Kernels of the flexible GCR outer solver (FP64, component-major spinors).
//
// One GCR step with preconditioned direction z and w = M_pc z:
//   beta_j = <W_j, w> / |W_j|^2            (k_gcr_multidot, all j in one pass)
//   w' = w - sum beta_j W_j ; z' = z - sum beta_j Z_j   -> stored as W_k, Z_k
//   alpha = <w', r> / |w'|^2               (reduced by k_gcr_orth)
//   x += alpha z' ; r -= alpha w'          (k_gcr_update, reduces |r|^2)
// All reductions are FP64 and deterministic (reduce.cuh).
#include "gcr.h"

namespace qcu {

using C = Cpx<double>;

// site-blocked FP64 spinor access (fields.cuh)
__device__ __forceinline__ void ld12(const double2 *p, int s, int, C v[12]) {
  p += blk_base<12>(s);
#pragma unroll
  for (int c = 0; c < 12; c++) {
    const double2 d = __ldg(p + c * SB);
    v[c] = C(d.x, d.y);
  }
}
__device__ __forceinline__ void st12(double2 *p, int s, int, const C v[12]) {
  p += blk_base<12>(s);
#pragma unroll
  for (int c = 0; c < 12; c++) p[c * SB] = make_double2(v[c].re, v[c].im);
}

// sums[2j], sums[2j+1] = <W_j, w>, j < k
__global__ void __launch_bounds__(BLAS_BLOCK) k_gcr_multidot(int Vh, GcrArgs a, SolverState *st, double *partials) {
  double red[2 * GCR_MAXK];
#pragma unroll
  for (int j = 0; j < 2 * GCR_MAXK; j++) red[j] = 0.0;
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    C w[12];
    ld12(static_cast<const double2 *>(a.w), s, Vh, w);
#pragma unroll
    for (int j = 0; j < GCR_MAXK; j++) {
      if (j < a.k) {
        const double2 *Wj = static_cast<const double2 *>(a.W[j]) + blk_base<12>(s);
#pragma unroll
        for (int c = 0; c < 12; c++) {
          const double2 q = __ldg(Wj + c * SB);
          red[2 * j] += q.x * w[c].re + q.y * w[c].im;
          red[2 * j + 1] += q.x * w[c].im - q.y * w[c].re;
        }
      }
    }
  }
  grid_reduce<2 * GCR_MAXK, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_STORE});
}

// W_k = w - sum beta_j W_j, Z_k = z - sum beta_j Z_j; sums = |W_k|^2, <W_k, r>
__global__ void __launch_bounds__(BLAS_BLOCK) k_gcr_orth(int Vh, GcrArgs a, SolverState *st, double *partials) {
  double red[3] = {0, 0, 0};
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    C w[12], z[12];
    ld12(static_cast<const double2 *>(a.w), s, Vh, w);
    ld12(static_cast<const double2 *>(a.z), s, Vh, z);
    for (int j = 0; j < a.k; j++) {
      const C b(a.beta[2 * j], a.beta[2 * j + 1]);
      C q[12];
      ld12(static_cast<const double2 *>(a.W[j]), s, Vh, q);
#pragma unroll
      for (int c = 0; c < 12; c++) w[c] -= b * q[c];
      ld12(static_cast<const double2 *>(a.Z[j]), s, Vh, q);
#pragma unroll
      for (int c = 0; c < 12; c++) z[c] -= b * q[c];
    }
    st12(static_cast<double2 *>(a.W[a.k]), s, Vh, w);
    st12(static_cast<double2 *>(a.Z[a.k]), s, Vh, z);
    C r[12];
    ld12(static_cast<const double2 *>(a.r), s, Vh, r);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      red[0] += w[c].norm2();
      const C d = cdotmul(w[c], r[c]);
      red[1] += d.re;
      red[2] += d.im;
    }
  }
  grid_reduce<3, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_STORE});
}

// x += alpha Z_k ; r -= alpha W_k ; sums[0] = |r|^2
__global__ void __launch_bounds__(BLAS_BLOCK) k_gcr_update(int Vh, GcrArgs a, SolverState *st, double *partials) {
  double red[1] = {0};
  const C al(a.alpha[0], a.alpha[1]);
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    C x[12], q[12];
    ld12(static_cast<const double2 *>(a.x), s, Vh, x);
    ld12(static_cast<const double2 *>(a.Z[a.k]), s, Vh, q);
#pragma unroll
    for (int c = 0; c < 12; c++) x[c] += al * q[c];
    st12(static_cast<double2 *>(a.x), s, Vh, x);
    ld12(static_cast<const double2 *>(a.r), s, Vh, x);
    ld12(static_cast<const double2 *>(a.W[a.k]), s, Vh, q);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      x[c] -= al * q[c];
      red[0] += x[c].norm2();
    }
    st12(static_cast<double2 *>(a.r), s, Vh, x);
  }
  grid_reduce<1, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_STORE});
}

void launch_gcr_multidot(int Vh, const GcrArgs &a, Context &ctx, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  k_gcr_multidot<<<g, BLAS_BLOCK, 0, s>>>(Vh, a, ctx.st, ctx.partials);
  QCU_CHECK_LAUNCH();
}
void launch_gcr_orth(int Vh, const GcrArgs &a, Context &ctx, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  k_gcr_orth<<<g, BLAS_BLOCK, 0, s>>>(Vh, a, ctx.st, ctx.partials);
  QCU_CHECK_LAUNCH();
}
void launch_gcr_update(int Vh, const GcrArgs &a, Context &ctx, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  k_gcr_update<<<g, BLAS_BLOCK, 0, s>>>(Vh, a, ctx.st, ctx.partials);
  QCU_CHECK_LAUNCH();
}

}  // namespace qcu
