// Wilson / clover hopping-term kernels for sm_100a.
//
// One thread per output site of one parity; the eight neighbour spinors and
// eight reconstruct-12 links are read with 16-byte (8-byte for FP16 links)
// read-only loads in component-major layouts, so every warp instruction moves
// contiguous 256-512 byte segments and neighbour re-reads hit L1/L2.  The
// epilogue fuses, in registers, what the solver would otherwise do in extra
// passes over HBM:
//     w   = D_{p<-1-p} in                      (qcu's wilson_dslash, src/wilson_dslash.cu:9-245)
//     w   = A_p^{-1} w          (clover)       (qcu's give_clover, src/clover_dslash.cu:857-882)
//     out = a*w + b1*x1 + b2*x2                (qcu's bistabcg_give_dest_o/_b__0, src/bistabcg.cu:73-96)
//     and one of  <rt, out>,  <out, x1> & |out|^2,  |out|^2  reduced to the solver state.
#include <algorithm>

#include "hop32.cuh"
#include "internal.h"

namespace qcu {

// Resident blocks per SM requested from the register allocator.  The FP64
// kernels would otherwise take ~176 registers (2 blocks of 128 threads per
// SM); 3 blocks fit in 170 registers without spills.  The FP32- and
// 16-bit-spinor kernels (paired FP32 instructions, hop32.cuh) issue few
// enough instructions to be bound by memory latency instead: they take more
// resident blocks (72 registers, 7 blocks) for more loads in flight.  The
// variants with a reduction stride over the sites with one resident wave of 3
// blocks per SM, except the 16-bit ones (below).
#ifndef QCU_DSLASH32_BLOCKS
#define QCU_DSLASH32_BLOCKS 7  // FP32 / 16-bit spinors without a reduction
#endif
#ifndef QCU_DSLASH16_RED_BLOCKS
#define QCU_DSLASH16_RED_BLOCKS 7  // 16-bit spinors with a reduction
#endif
#ifndef QCU_DSLASH16_CLOV_RED_BLOCKS
#define QCU_DSLASH16_CLOV_RED_BLOCKS 6  // the same with the clover term
#endif
// 16-bit spinors reduce in two kernels: every block of the dslash writes its
// partial, and a one-block kernel sums them.  The strided one-wave form
// (every other kind) takes ~165 registers there and 3 resident blocks.  The
// split form measured faster for the 16-bit kernels and slower for the FP32
// ones.  It fits 72 registers and 7 blocks (4-8 bytes spilled), which made a
// solve 0.5 % faster than 80 registers and 6 blocks; with the clover term 7
// blocks would spill 52-68 bytes, so those keep 80 registers and 6 blocks.
#define DSLASH_SPLIT_RED(K) ((K) == SOA16)
#define DSLASH_RED_BLOCKS(K) ((K) == SOA16 ? QCU_DSLASH16_RED_BLOCKS : 3)
#define DSLASH_MIN_BLOCKS(K, RED, CLOV)                                                   \
  (((K) == AOS64 || (K) == AOS64W || (K) == SOA64) ? 3                                   \
   : (RED) == RED_NONE                            ? QCU_DSLASH32_BLOCKS                  \
   : ((K) == SOA16 && (CLOV))                     ? QCU_DSLASH16_CLOV_RED_BLOCKS         \
                                                  : DSLASH_RED_BLOCKS(K))

// FP32 and 16-bit spinors: the hop and the epilogue on spin-paired registers
// in FP32 arithmetic (hop32.cuh)
template <int K, int G, int C, bool CLOV, int NX, int RED, int NV>
__device__ __forceinline__ void dslash_site32(const Geom &g, const DslashArgs &a, int s, double (&red)[NV]) {
  const SpinorView<K> in{const_cast<void *>(a.in), const_cast<float *>(a.in_norm), g.Vh};
  const GaugeView<G> U{a.gauge, pad_sites(g.Vh)};
  Site2 w;
  const float unit = wilson_hop_site2<K, G>(w, in, U, g, s, a.parity, (float)a.t_bc);
  if constexpr (CLOV) {
    Cpx<float> v[12];
    site2_to_cpx(w, v);
    clover_apply_site<C, float>(CloverView<C>{a.clover, g.Vh}, s, v);
    cpx_to_site2(v, w);
  }
  site2_scale(w, bc2((float)a.a * unit));
  Site2 x1;
  if constexpr (NX >= 1) {
    site_load2<K>(SpinorView<K>{const_cast<void *>(a.x1), const_cast<float *>(a.x1_norm), g.Vh}, s, x1);
    site2_axpy(w, bc2((float)a.b1), x1);
  }
  if constexpr (NX >= 2) {
    Site2 x2;
    site_load2<K>(SpinorView<K>{const_cast<void *>(a.x2), const_cast<float *>(a.x2_norm), g.Vh}, s, x2);
    site2_axpy(w, bc2((float)a.b2), x2);
  }
  site_store2<K>(SpinorView<K>{a.out, a.out_norm, g.Vh}, s, w);
  if constexpr (RED != RED_NONE) {
    Cpx<float> wv[12];
    site2_to_cpx(w, wv);
    if constexpr (RED == RED_DOT_RT) {  // <rt, out>
      Cpx<float> rt[12];
      spinor_load<K, float>(SpinorView<K>{const_cast<void *>(a.rt), const_cast<float *>(a.rt_norm), g.Vh}, s, rt);
      site_dot<float>(rt, wv, red[0], red[1]);
    } else if constexpr (RED == RED_TS_TT) {  // <out, x1>, |out|^2
      Cpx<float> xv[12];
      site2_to_cpx(x1, xv);
      site_dot<float>(wv, xv, red[0], red[1]);
      site_norm2<float>(wv, red[2]);
    } else if constexpr (RED == RED_NORM) {
      site_norm2<float>(wv, red[0]);
    }
  }
}

template <int K, int G, int C, bool CLOV, int NX, int RED, int NV>
__device__ __forceinline__ void dslash_site_scalar(const Geom &g, const DslashArgs &a, int s, double (&red)[NV]);

// one output site: hop term, clover, epilogue, the site's share of the reduction
template <int K, int G, int C, bool CLOV, int NX, int RED, int NV>
__device__ __forceinline__ void dslash_site(const Geom &g, const DslashArgs &a, int s, double (&red)[NV]) {
  if constexpr (K == SOA32 || K == SOA16) {
    dslash_site32<K, G, C, CLOV, NX, RED, NV>(g, a, s, red);
  } else {
    dslash_site_scalar<K, G, C, CLOV, NX, RED, NV>(g, a, s, red);
  }
}

// FP64 spinors: scalar complex arithmetic
template <int K, int G, int C, bool CLOV, int NX, int RED, int NV>
__device__ __forceinline__ void dslash_site_scalar(const Geom &g, const DslashArgs &a, int s, double (&red)[NV]) {
  using T = typename SpinorReal<K>::T;
  Cpx<T> w[12];
  const SpinorView<K> in{const_cast<void *>(a.in), const_cast<float *>(a.in_norm), g.Vh};
  const GaugeView<G> U{a.gauge, G == GAOS64 ? g.Vh : pad_sites(g.Vh)};
  wilson_hop_site<K, G, T>(w, in, U, g, s, a.parity, (T)a.t_bc);
  if constexpr (CLOV) clover_apply_site<C, T>(CloverView<C>{a.clover, g.Vh}, s, w);
  const T aa = (T)a.a;
#pragma unroll
  for (int c = 0; c < 12; c++) w[c] = w[c] * aa;
  Cpx<T> x1[12];
  if constexpr (NX >= 1) {
    spinor_load<K, T>(SpinorView<K>{const_cast<void *>(a.x1), const_cast<float *>(a.x1_norm), g.Vh}, s, x1);
    const T b1 = (T)a.b1;
#pragma unroll
    for (int c = 0; c < 12; c++) w[c] += x1[c] * b1;
  }
  if constexpr (NX >= 2) {
    Cpx<T> x2[12];
    spinor_load<K, T>(SpinorView<K>{const_cast<void *>(a.x2), const_cast<float *>(a.x2_norm), g.Vh}, s, x2);
    const T b2 = (T)a.b2;
#pragma unroll
    for (int c = 0; c < 12; c++) w[c] += x2[c] * b2;
  }
  spinor_store<K, T>(SpinorView<K>{a.out, a.out_norm, g.Vh}, s, w);
  if constexpr (RED == RED_DOT_RT) {  // <rt, out>
    Cpx<T> rt[12];
    spinor_load<K, T>(SpinorView<K>{const_cast<void *>(a.rt), const_cast<float *>(a.rt_norm), g.Vh}, s, rt);
    site_dot<T>(rt, w, red[0], red[1]);
  } else if constexpr (RED == RED_TS_TT) {  // <out, x1>, |out|^2
    site_dot<T>(w, x1, red[0], red[1]);
    site_norm2<T>(w, red[2]);
  } else if constexpr (RED == RED_NORM) {
    site_norm2<T>(w, red[0]);
  }
}

template <int K, int G, int C, bool CLOV, int NX, int RED>
__global__ void __launch_bounds__(DSLASH_BLOCK, DSLASH_MIN_BLOCKS(K, RED, CLOV)) k_dslash(Geom g, DslashArgs a, RedCtx rc) {
  if (!gate_open(rc.st, a.gate)) return;
  constexpr int NV = RED == RED_NONE ? 1 : (RED == RED_TS_TT ? 3 : (RED == RED_DOT_RT ? 2 : 1));
  double red[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) red[k] = 0.0;
  if constexpr (RED == RED_NONE) {
    const int s = blockIdx.x * DSLASH_BLOCK + threadIdx.x;  // one site per thread
    if (s < g.Vh) dslash_site<K, G, C, CLOV, NX, RED, NV>(g, a, s, red);
  } else if constexpr (DSLASH_SPLIT_RED(K)) {
    // one site per thread; the block's partial goes to partials[k * grid + b]
    // and k_red_finish, launched next, reduces them
    const int s = blockIdx.x * DSLASH_BLOCK + threadIdx.x;
    if (s < g.Vh) dslash_site<K, G, C, CLOV, NX, RED, NV>(g, a, s, red);
    double part[NV];
    block_sum<NV, DSLASH_BLOCK>(red, part);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; k++) rc.partials[(size_t)k * gridDim.x + blockIdx.x] = part[k];
    }
  } else {
    // a grid of resident blocks strides over the sites, so the block
    // reduction and the ticket (barriers, a fence, an atomic) are paid once
    // per block rather than once per 128 sites
    for (int s = blockIdx.x * DSLASH_BLOCK + threadIdx.x; s < g.Vh; s += gridDim.x * DSLASH_BLOCK)
      dslash_site<K, G, C, CLOV, NX, RED, NV>(g, a, s, red);
    grid_reduce<NV, DSLASH_BLOCK>(red, rc);
  }
}

// Sum of the n block partials of a split reduction, in block order, and the
// finalize op; skipped with the dslash it belongs to when its gate is closed.
constexpr int FINISH_BLOCK = 512;
template <int NV>
__global__ void __launch_bounds__(FINISH_BLOCK) k_red_finish(const double *partials, int n, SolverState *st, int op,
                                                           int gate) {
  if (!gate_open(st, gate)) return;
  double tot[NV];
  sum_partials<NV, FINISH_BLOCK>(partials, n, tot);
  if (threadIdx.x == 0) {
    double v[RED_MAXV];
#pragma unroll
    for (int k = 0; k < RED_MAXV; k++) v[k] = k < NV ? tot[k] : 0.0;
    finalize(st, op, v);
  }
}

template <int K, int G, int C, bool CLOV, int NX, int RED>
static void launch_t(const Geom &g, const DslashArgs &a, Context &ctx, cudaStream_t s) {
  int blocks = (g.Vh + DSLASH_BLOCK - 1) / DSLASH_BLOCK;
  // reductions: one resident wave (the 16/32-bit reducing variants take ~167 registers, FP64 170)
  if (RED != RED_NONE && !DSLASH_SPLIT_RED(K)) blocks = std::min(blocks, DSLASH_RED_BLOCKS(K) * ctx.sms);
  RedCtx rc{ctx.st, ctx.partials, a.fin};
  if (RED != RED_NONE) {
    require(a.gate == GATE_ALWAYS || ctx.st != nullptr, "reduction without solver state");
    ctx.ensure_partials(blocks);
    rc.partials = ctx.partials;
  }
  k_dslash<K, G, C, CLOV, NX, RED><<<blocks, DSLASH_BLOCK, 0, s>>>(g, a, rc);
  QCU_CHECK_LAUNCH();
  if (RED != RED_NONE && DSLASH_SPLIT_RED(K)) {
    constexpr int NV = RED == RED_TS_TT ? 3 : (RED == RED_DOT_RT ? 2 : 1);
    k_red_finish<NV><<<1, FINISH_BLOCK, 0, s>>>(rc.partials, blocks, rc.st, rc.op, a.gate);
    QCU_CHECK_LAUNCH();
  }
}

template <int K, int G, int C, bool CLOV>
static void launch_nx(const Geom &g, const DslashArgs &a, Context &ctx, cudaStream_t s) {
  const int nx = a.x2 ? 2 : (a.x1 ? 1 : 0);
  if (nx == 0) {
    require(a.red == RED_NONE, "dslash: reduction needs an epilogue source");
    launch_t<K, G, C, CLOV, 0, RED_NONE>(g, a, ctx, s);
  } else if (nx == 1) {
    switch (a.red) {
      case RED_NONE: launch_t<K, G, C, CLOV, 1, RED_NONE>(g, a, ctx, s); break;
      case RED_DOT_RT: launch_t<K, G, C, CLOV, 1, RED_DOT_RT>(g, a, ctx, s); break;
      case RED_TS_TT: launch_t<K, G, C, CLOV, 1, RED_TS_TT>(g, a, ctx, s); break;
      default: throw Error(1, "dslash: unsupported reduction with one source");
    }
  } else {
    switch (a.red) {
      case RED_NONE: launch_t<K, G, C, CLOV, 2, RED_NONE>(g, a, ctx, s); break;
      case RED_NORM: launch_t<K, G, C, CLOV, 2, RED_NORM>(g, a, ctx, s); break;
      default: throw Error(1, "dslash: unsupported reduction with two sources");
    }
  }
}

template <int K, int G, int C>
static void launch_clov(const Geom &g, const DslashArgs &a, Context &ctx, cudaStream_t s) {
  if (a.clover) launch_nx<K, G, C, true>(g, a, ctx, s);
  else launch_nx<K, G, C, false>(g, a, ctx, s);
}

void launch_dslash(int kind, int gkind, int ckind, const Geom &g, const DslashArgs &a, Context &ctx,
                   cudaStream_t s) {
  // PyQuda-layout spinors whose buffers are all 32-byte aligned take the 32-byte accesses
  auto al32 = [](const void *p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 31) == 0; };
  if (kind == AOS64 && gkind == GAOS64 && ckind == CSOA64 && al32(a.in) && al32(a.out) && al32(a.x1) &&
      al32(a.x2) && al32(a.rt))
    launch_clov<AOS64W, GAOS64, CSOA64>(g, a, ctx, s);
  else if (kind == AOS64 && gkind == GAOS64 && ckind == CSOA64) launch_clov<AOS64, GAOS64, CSOA64>(g, a, ctx, s);
  else if (kind == SOA64 && gkind == GSOA64 && ckind == CSOA64) launch_clov<SOA64, GSOA64, CSOA64>(g, a, ctx, s);
  else if (kind == SOA32 && gkind == GSOA32 && ckind == CSOA32) launch_clov<SOA32, GSOA32, CSOA32>(g, a, ctx, s);
  else if (kind == SOA16 && gkind == GSOA16 && ckind == CSOA32) launch_clov<SOA16, GSOA16, CSOA32>(g, a, ctx, s);
  else if (kind == SOA32 && gkind == GSOA16 && ckind == CSOA32) launch_clov<SOA32, GSOA16, CSOA32>(g, a, ctx, s);
  else throw Error(1, "dslash: unsupported storage combination");
}

}  // namespace qcu
