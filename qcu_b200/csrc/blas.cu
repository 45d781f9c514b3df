// Fused level-1 kernels of the BiCGSTAB iteration, layout/precision
// conversion, and generic reductions.
//
// qcu runs one kernel per vector update plus a cuBLAS dot and an NCCL
// all-reduce per inner product, with the scalar recurrences in <<<1,1>>>
// kernels (src/bistabcg.cu:4-169, include/lattice_bistabcg.h:149-163,221-340).
// Here every update kernel also produces the inner products the next scalar
// needs, and the last block of the grid applies the recurrence in place
// (reduce.cuh), so one BiCGSTAB iteration is 7 launches and no host round trip.
#include "internal.h"

namespace qcu {

template <int K>
using Real = typename SpinorReal<K>::T;

template <int K>
__device__ __forceinline__ SpinorView<K> sv(void *p, float *n, int Vh) {
  return SpinorView<K>{p, n, Vh};
}

__device__ __forceinline__ Cpx<double> ld2(const double *a) { return Cpx<double>(a[0], a[1]); }

// ---------------------------------------------------------------- iteration kernels
// p = r + beta (p - omega v),  beta = (rho/rho_prev)(alpha/omega)
template <int K>
__global__ void __launch_bounds__(BLAS_BLOCK) k_pupdate(int Vh, VecSet vs, SolverState *st, int gate) {
  using T = Real<K>;
  if (!gate_open(st, gate)) return;
  const Cpx<double> rho = ld2(st->rho), rho_prev = ld2(st->rho_prev), alpha = ld2(st->alpha),
                    omega = ld2(st->omega);
  const Cpx<double> beta = cdiv(rho, rho_prev) * cdiv(alpha, omega);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->beta[0] = beta.re;
    st->beta[1] = beta.im;
  }
  const Cpx<T> b((T)beta.re, (T)beta.im), w((T)omega.re, (T)omega.im);
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<T> r[12], p[12], v[12];
    spinor_load<K, T>(sv<K>(vs.r, vs.rn, Vh), s, r);
    spinor_load<K, T>(sv<K>(vs.p, vs.pn, Vh), s, p);
    spinor_load<K, T>(sv<K>(vs.v, vs.vn, Vh), s, v);
#pragma unroll
    for (int c = 0; c < 12; c++) p[c] = r[c] + (p[c] - v[c] * w) * b;
    spinor_store<K, T>(sv<K>(vs.p, vs.pn, Vh), s, p);
  }
}

// s = r - alpha v
template <int K>
__global__ void __launch_bounds__(BLAS_BLOCK) k_supdate(int Vh, VecSet vs, SolverState *st, int gate) {
  using T = Real<K>;
  if (!gate_open(st, gate)) return;
  const Cpx<T> a((T)st->alpha[0], (T)st->alpha[1]);
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<T> r[12], v[12];
    spinor_load<K, T>(sv<K>(vs.r, vs.rn, Vh), s, r);
    spinor_load<K, T>(sv<K>(vs.v, vs.vn, Vh), s, v);
#pragma unroll
    for (int c = 0; c < 12; c++) r[c] = r[c] - v[c] * a;
    spinor_store<K, T>(sv<K>(vs.s, vs.sn, Vh), s, r);
  }
}

// x += alpha p + omega s ; r = s - omega t ; reduce <rt, r>, |r|^2  -> FIN_XR
template <int K, int XK>
__global__ void __launch_bounds__(BLAS_BLOCK) k_xrupdate(int Vh, VecSet vs, SolverState *st, double *partials,
                                                          int gate) {
  using T = Real<K>;
  using TX = Real<XK>;
  if (!gate_open(st, gate)) return;
  const Cpx<T> a((T)st->alpha[0], (T)st->alpha[1]), w((T)st->omega[0], (T)st->omega[1]);
  const Cpx<TX> ax((TX)st->alpha[0], (TX)st->alpha[1]), wx((TX)st->omega[0], (TX)st->omega[1]);
  double red[3] = {0, 0, 0};
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    // every input first: the vectors are distinct buffers, so no store below
    // feeds a load (0.6 % faster per solve than loading t and rt after the stores)
    Cpx<T> p[12], q[12], t[12], rt[12];
    Cpx<TX> x[12];
    spinor_load<K, T>(sv<K>(vs.p, vs.pn, Vh), s, p);
    spinor_load<K, T>(sv<K>(vs.s, vs.sn, Vh), s, q);
    spinor_load<XK, TX>(sv<XK>(vs.x, vs.xn, Vh), s, x);
    spinor_load<K, T>(sv<K>(vs.t, vs.tn, Vh), s, t);
    spinor_load<K, T>(sv<K>(vs.rt, vs.rtn, Vh), s, rt);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      x[c] += Cpx<TX>((TX)p[c].re, (TX)p[c].im) * ax;
      x[c] += Cpx<TX>((TX)q[c].re, (TX)q[c].im) * wx;
    }
    spinor_store<XK, TX>(sv<XK>(vs.x, vs.xn, Vh), s, x);
#pragma unroll
    for (int c = 0; c < 12; c++) q[c] = q[c] - t[c] * w;
    spinor_store<K, T>(sv<K>(vs.r, vs.rn, Vh), s, q);
    site_dot<T>(rt, q, red[0], red[1]);
    site_norm2<T>(q, red[2]);
  }
  grid_reduce<3, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_XR});
}

// x64 += x ; x = 0
template <int XK>
__global__ void __launch_bounds__(BLAS_BLOCK) k_xfold(int Vh, VecSet vs, SolverState *st, int gate) {
  using TX = Real<XK>;
  if (!gate_open(st, gate)) return;
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<TX> x[12];
    Cpx<double> y[12];
    spinor_load<XK, TX>(sv<XK>(vs.x, vs.xn, Vh), s, x);
    spinor_load<SOA64, double>(sv<SOA64>(vs.x64, nullptr, Vh), s, y);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      y[c] += Cpx<double>((double)x[c].re, (double)x[c].im);
      x[c] = Cpx<TX>(0, 0);
    }
    spinor_store<SOA64, double>(sv<SOA64>(vs.x64, nullptr, Vh), s, y);
    spinor_store<XK, TX>(sv<XK>(vs.x, vs.xn, Vh), s, x);
  }
}

// r = convert(r64) ; reduce <rt, r>  -> FIN_RCONV
template <int K>
__global__ void __launch_bounds__(BLAS_BLOCK) k_rconv(int Vh, VecSet vs, SolverState *st, double *partials,
                                                       int gate) {
  using T = Real<K>;
  if (!gate_open(st, gate)) return;
  double red[2] = {0, 0};
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<T> r[12], rt[12];
    spinor_load<SOA64, T>(sv<SOA64>(vs.r64, nullptr, Vh), s, r);
    if (K != SOA64 || vs.r != vs.r64) spinor_store<K, T>(sv<K>(vs.r, vs.rn, Vh), s, r);
    spinor_load<K, T>(sv<K>(vs.rt, vs.rtn, Vh), s, rt);
    site_dot<T>(rt, r, red[0], red[1]);
  }
  grid_reduce<2, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_RCONV});
}

// r = rt = convert(r64); p = v = x = 0; reduce <rt, r>, |r64|^2  -> FIN_INIT
template <int K, int XK>
__global__ void __launch_bounds__(BLAS_BLOCK) k_init(int Vh, VecSet vs, SolverState *st, double *partials) {
  using T = Real<K>;
  using TX = Real<XK>;
  double red[3] = {0, 0, 0};
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<double> r64[12];
    Cpx<T> r[12], z[12];
    Cpx<TX> zx[12];
    spinor_load<SOA64, double>(sv<SOA64>(vs.r64, nullptr, Vh), s, r64);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      r[c] = Cpx<T>((T)r64[c].re, (T)r64[c].im);
      z[c] = Cpx<T>(0, 0);
      zx[c] = Cpx<TX>(0, 0);
      red[0] += (double)r[c].re * r[c].re + (double)r[c].im * r[c].im;
      red[2] += r64[c].re * r64[c].re + r64[c].im * r64[c].im;
    }
    if (K != SOA64 || vs.r != vs.r64) spinor_store<K, T>(sv<K>(vs.r, vs.rn, Vh), s, r);
    spinor_store<K, T>(sv<K>(vs.rt, vs.rtn, Vh), s, r);
    spinor_store<K, T>(sv<K>(vs.p, vs.pn, Vh), s, z);
    spinor_store<K, T>(sv<K>(vs.v, vs.vn, Vh), s, z);
    spinor_store<XK, TX>(sv<XK>(vs.x, vs.xn, Vh), s, zx);
  }
  grid_reduce<3, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_INIT});
}

// ---------------------------------------------------------------- generic kernels
template <int KI, int KO>
__global__ void __launch_bounds__(BLAS_BLOCK) k_convert(int Vh, void *in, float *in_n, void *out, float *out_n) {
  using T = typename SpinorReal<(KI == AOS64 || KI == SOA64) && (KO == AOS64 || KO == SOA64) ? SOA64 : SOA32>::T;
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<T> v[12];
    spinor_load<KI, T>(sv<KI>(in, in_n, Vh), s, v);
    spinor_store<KO, T>(sv<KO>(out, out_n, Vh), s, v);
  }
}

// y = a x + b y
template <int K>
__global__ void __launch_bounds__(BLAS_BLOCK) k_axpby(int Vh, double a, void *x, float *xn, double b, void *y,
                                                       float *yn) {
  using T = Real<K>;
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<T> u[12], w[12];
    spinor_load<K, T>(sv<K>(x, xn, Vh), s, u);
    spinor_load<K, T>(sv<K>(y, yn, Vh), s, w);
#pragma unroll
    for (int c = 0; c < 12; c++) w[c] = u[c] * (T)a + w[c] * (T)b;
    spinor_store<K, T>(sv<K>(y, yn, Vh), s, w);
  }
}

// sums[0..1] = <a, b>, sums[2] = |a|^2, sums[3] = |b|^2
template <int K>
__global__ void __launch_bounds__(BLAS_BLOCK) k_dots(int Vh, void *a, float *an, void *b, float *bn, SolverState *st,
                                                      double *partials) {
  using T = Real<K>;
  double red[4] = {0, 0, 0, 0};
  for (int s = blockIdx.x * BLAS_BLOCK + threadIdx.x; s < Vh; s += gridDim.x * BLAS_BLOCK) {
    Cpx<T> u[12], w[12];
    spinor_load<K, T>(sv<K>(a, an, Vh), s, u);
    spinor_load<K, T>(sv<K>(b, bn, Vh), s, w);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      red[0] += (double)u[c].re * w[c].re + (double)u[c].im * w[c].im;
      red[1] += (double)u[c].re * w[c].im - (double)u[c].im * w[c].re;
      red[2] += (double)u[c].re * u[c].re + (double)u[c].im * u[c].im;
      red[3] += (double)w[c].re * w[c].re + (double)w[c].im * w[c].im;
    }
  }
  grid_reduce<4, BLAS_BLOCK>(red, RedCtx{st, partials, FIN_STORE});
}

// Condition of a device-side WHILE loop over solver iterations (a CUDA graph
// conditional node): continue while the solver is not done.  The guard
// bounds the loop whatever happens to `done`: after `cap` passes it stops
// and reports the solve as having hit its iteration limit.
__global__ void k_loop_cond(SolverState *st, cudaGraphConditionalHandle h, unsigned cap) {
  const unsigned n = ++st->loop_guard;
  bool go = st->done == 0;
  if (go && n >= cap) {
    st->status = ST_MAXITER;
    st->done = 1;
    go = false;
  }
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ---------------------------------------------------------------- launchers
void launch_loop_cond(SolverState *st, cudaGraphConditionalHandle h, unsigned cap, cudaStream_t s) {
  k_loop_cond<<<1, 1, 0, s>>>(st, h, cap);
  QCU_CHECK_LAUNCH();
}

#define QCU_DISPATCH_K(kind, F, ...)                   \
  switch (kind) {                                      \
    case SOA64: F<SOA64> __VA_ARGS__; break;           \
    case SOA32: F<SOA32> __VA_ARGS__; break;           \
    case SOA16: F<SOA16> __VA_ARGS__; break;           \
    default: throw Error(1, "unsupported spinor kind"); \
  }

void launch_pupdate(int kind, int Vh, const VecSet &vs, SolverState *st, int gate, cudaStream_t s) {
  QCU_DISPATCH_K(kind, k_pupdate, <<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, vs, st, gate));
  QCU_CHECK_LAUNCH();
}
void launch_supdate(int kind, int Vh, const VecSet &vs, SolverState *st, int gate, cudaStream_t s) {
  QCU_DISPATCH_K(kind, k_supdate, <<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, vs, st, gate));
  QCU_CHECK_LAUNCH();
}
void launch_xrupdate(int kind, int Vh, const VecSet &vs, Context &ctx, int gate, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  switch (kind) {
    case SOA64: k_xrupdate<SOA64, SOA64><<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials, gate); break;
    case SOA32: k_xrupdate<SOA32, SOA32><<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials, gate); break;
    case SOA16: k_xrupdate<SOA16, SOA32><<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials, gate); break;
    default: throw Error(1, "unsupported spinor kind");
  }
  QCU_CHECK_LAUNCH();
}
void launch_xfold(int kind, int Vh, const VecSet &vs, SolverState *st, int gate, cudaStream_t s) {
  if (kind == SOA64) k_xfold<SOA64><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, vs, st, gate);
  else k_xfold<SOA32><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, vs, st, gate);
  QCU_CHECK_LAUNCH();
}
void launch_rconv(int kind, int Vh, const VecSet &vs, Context &ctx, int gate, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  QCU_DISPATCH_K(kind, k_rconv, <<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials, gate));
  QCU_CHECK_LAUNCH();
}
void launch_init(int kind, int Vh, const VecSet &vs, Context &ctx, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  switch (kind) {
    case SOA64: k_init<SOA64, SOA64><<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials); break;
    case SOA32: k_init<SOA32, SOA32><<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials); break;
    case SOA16: k_init<SOA16, SOA32><<<g, BLAS_BLOCK, 0, s>>>(Vh, vs, ctx.st, ctx.partials); break;
    default: throw Error(1, "unsupported spinor kind");
  }
  QCU_CHECK_LAUNCH();
}

void launch_convert(int kin, int kout, int Vh, const void *in, const float *in_n, void *out, float *out_n,
                    cudaStream_t s) {
  const int g = blas_grid(Vh);
  void *i = const_cast<void *>(in);
  float *in2 = const_cast<float *>(in_n);
#define QCU_CONV(A, B)                                                    \
  if (kin == A && kout == B) {                                            \
    k_convert<A, B><<<g, BLAS_BLOCK, 0, s>>>(Vh, i, in2, out, out_n);     \
    QCU_CHECK_LAUNCH();                                                   \
    return;                                                               \
  }
  QCU_CONV(AOS64, SOA64)
  QCU_CONV(SOA64, AOS64)
  QCU_CONV(AOS64, SOA32)
  QCU_CONV(SOA32, AOS64)
  QCU_CONV(AOS64, SOA16)
  QCU_CONV(SOA16, AOS64)
  QCU_CONV(SOA64, SOA32)
  QCU_CONV(SOA32, SOA64)
  QCU_CONV(SOA64, SOA16)
  QCU_CONV(SOA16, SOA64)
  QCU_CONV(SOA32, SOA16)
  QCU_CONV(SOA16, SOA32)
  QCU_CONV(SOA64, SOA64)
  QCU_CONV(AOS64, AOS64)
#undef QCU_CONV
  throw Error(1, "unsupported conversion");
}

void launch_axpby(int kind, int Vh, double a, void *x, float *xn, double b, void *y, float *yn, cudaStream_t s) {
  switch (kind) {
    case AOS64: k_axpby<AOS64><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, a, x, xn, b, y, yn); break;
    case SOA64: k_axpby<SOA64><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, a, x, xn, b, y, yn); break;
    case SOA32: k_axpby<SOA32><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, a, x, xn, b, y, yn); break;
    case SOA16: k_axpby<SOA16><<<blas_grid(Vh), BLAS_BLOCK, 0, s>>>(Vh, a, x, xn, b, y, yn); break;
    default: throw Error(1, "unsupported spinor kind");
  }
  QCU_CHECK_LAUNCH();
}

void launch_dots(int kind, int Vh, void *a, float *an, void *b, float *bn, Context &ctx, cudaStream_t s) {
  const int g = blas_grid(Vh);
  ctx.ensure_partials(g);
  switch (kind) {
    case AOS64: k_dots<AOS64><<<g, BLAS_BLOCK, 0, s>>>(Vh, a, an, b, bn, ctx.st, ctx.partials); break;
    case SOA64: k_dots<SOA64><<<g, BLAS_BLOCK, 0, s>>>(Vh, a, an, b, bn, ctx.st, ctx.partials); break;
    case SOA32: k_dots<SOA32><<<g, BLAS_BLOCK, 0, s>>>(Vh, a, an, b, bn, ctx.st, ctx.partials); break;
    case SOA16: k_dots<SOA16><<<g, BLAS_BLOCK, 0, s>>>(Vh, a, an, b, bn, ctx.st, ctx.partials); break;
    default: throw Error(1, "unsupported spinor kind");
  }
  QCU_CHECK_LAUNCH();
}

}  // namespace qcu
