// Batched kernels: every launch covers all right-hand sides of all lattices
// of a batch (tile table: tile k = (rhs, block of that rhs's sites)).
//
// The arithmetic per site is the single right-hand-side kernels' (dslash.cu,
// blas.cu, gcr.cu: qcu's wilson_dslash and BiCGSTAB updates,
// src/wilson_dslash.cu:9-245, src/bistabcg.cu:4-169, with the flexible GCR
// outer step on top); what changes is where each block finds its vectors,
// scalars and lattice: in the descriptor of its rhs.  Reductions end in the
// last block of the rhs's own tiles (per-rhs ticket, fixed summation order,
// so results are deterministic and independent of the other rhs).
#include <algorithm>
#include <type_traits>

#include "batch_dev.cuh"
#include "hop32.cuh"

namespace qcu {

// ---------------------------------------------------------------- hopping term
// One FP64 hop for the NR right-hand sides of a group: the link is loaded
// (row 2 rebuilt) once, scaled once, and applied to each right-hand side's
// neighbour spinor.  (FP32 and 16-bit spinors: wilson_hop_group2 below.)
template <int MU, bool FWD, int K, int G, typename T, int NR>
__device__ __forceinline__ void hop_group(Cpx<T> (&acc)[NR][12], const SpinorView<K> (&in)[NR], const bool (&on)[NR],
                                          const GaugeView<G> &U, int n, int lpar, int ls, T ph) {
  static_assert(K == SOA64, "the scalar group hop is the FP64 one");
  Cpx<T> u[9];
  link_load<G, T>(U, MU, lpar, ls, u);
  if constexpr (MU == 3) {
#pragma unroll
    for (int k = 0; k < 9; k++) u[k] = u[k] * ph;
  }
  // every slot is computed (a closed or empty slot reads a valid buffer and
  // is discarded in the epilogue): no branch between the loads of the slots
#pragma unroll
  for (int j = 0; j < NR; j++) {
    Cpx<T> psi[12];
    spinor_load<K, T>(in[j], n, psi);
    hop<MU, FWD, false, T>(acc[j], psi, u, T(1));
  }
  (void)on;
}

template <int K, int G, typename T, int NR>
__device__ __forceinline__ void wilson_hop_group(Cpx<T> (&acc)[NR][12], const SpinorView<K> (&in)[NR],
                                                 const bool (&on)[NR], const GaugeView<G> &U, const Geom &g, int s,
                                                 int par, T t_bc) {
#pragma unroll
  for (int j = 0; j < NR; j++)
#pragma unroll
    for (int c = 0; c < 12; c++) acc[j][c] = Cpx<T>(0, 0);
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  const int y = r % g.Ly;
  r /= g.Ly;
  const int z = r % g.Lz;
  const int t = r / g.Lz;
  const int xodd = (y + z + t + par) & 1;
  int n;
  n = xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s;
  hop_group<0, true>(acc, in, on, U, n, par, s, T(1));
  n = xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1);
  hop_group<0, false>(acc, in, on, U, n, 1 - par, n, T(1));
  n = (y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  hop_group<1, true>(acc, in, on, U, n, par, s, T(1));
  n = (y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  hop_group<1, false>(acc, in, on, U, n, 1 - par, n, T(1));
  n = (z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  hop_group<2, true>(acc, in, on, U, n, par, s, T(1));
  n = (z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  hop_group<2, false>(acc, in, on, U, n, 1 - par, n, T(1));
  n = (t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st;
  hop_group<3, true>(acc, in, on, U, n, par, s, (t == g.Lt - 1) ? t_bc : T(1));
  n = (t == 0) ? s + (g.Lt - 1) * g.st : s - g.st;
  hop_group<3, false>(acc, in, on, U, n, 1 - par, n, (t == 0) ? t_bc : T(1));
}

// FP32 and 16-bit spinors: the same hops on spin-paired registers
// (hop32.cuh), each link decoded and broadcast once for the NR right-hand
// sides.  acc holds the hop sums in units of the returned value (1/32767 for
// 16-bit links).
template <int K, int G, int NR>
__device__ __forceinline__ float wilson_hop_group2(Site2 (&acc)[NR], const SpinorView<K> (&in)[NR],
                                                   const GaugeView<G> &U, const Geom &g, int s, int par, float t_bc) {
#pragma unroll
  for (int j = 0; j < NR; j++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      acc[j].up.re[c] = acc[j].up.im[c] = acc[j].lo.re[c] = acc[j].lo.im[c] = make_float2(0.f, 0.f);
  int xh, y, z, t;
  site_coords(g, s, xh, y, z, t);
  const int xodd = (y + z + t + par) & 1;
  float unit = 1.0f;
  auto hop = [&](auto mu_c, auto fwd_c, int n, int lpar, int ls, float ph) {
    constexpr int MU = decltype(mu_c)::value;
    constexpr bool FWD = decltype(fwd_c)::value;
    Link2 u;
    unit = link2_load<G>(U, MU, lpar, ls, u);
#pragma unroll
    for (int j = 0; j < NR; j++) {  // every slot is computed; closed slots read a valid buffer
      Site2 psi;
      if constexpr (K == SOA16) {
        const float f = ph * site16_load_biased<(MU < 2)>(in[j], n, psi) * (1.0f / FIX16_SCALE);
        hop2<MU, FWD, true, true, link2_row2_raw<G>()>(acc[j], psi, u, f, LINK16_ROW2_F);
      } else {
        site2_load(in[j], n, psi);
        hop2<MU, FWD, false, false, link2_row2_raw<G>()>(acc[j], psi, u, ph, LINK16_ROW2_F);
      }
    }
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using I3 = std::integral_constant<int, 3>;
  using BT = std::true_type;
  using BF = std::false_type;
  int n;
  n = xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s;
  hop(I0{}, BT{}, n, par, s, 1.f);
  n = xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1);
  hop(I0{}, BF{}, n, 1 - par, n, 1.f);
  n = (y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  hop(I1{}, BT{}, n, par, s, 1.f);
  n = (y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  hop(I1{}, BF{}, n, 1 - par, n, 1.f);
  n = (z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  hop(I2{}, BT{}, n, par, s, 1.f);
  n = (z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  hop(I2{}, BF{}, n, 1 - par, n, 1.f);
  n = (t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st;
  hop(I3{}, BT{}, n, par, s, (t == g.Lt - 1) ? t_bc : 1.f);
  n = (t == 0) ? s + (g.Lt - 1) * g.st : s - g.st;
  hop(I3{}, BF{}, n, 1 - par, n, (t == 0) ? t_bc : 1.f);
  return unit;
}

// resident blocks asked of the register allocator: QCU_BDSL32_BLOCKS x 128
// threads for one FP32 rhs per thread, 3 x 128 for FP64; the
// register-blocked groups keep their registers
#ifndef QCU_BDSL32_BLOCKS
#define QCU_BDSL32_BLOCKS 4
#endif
#define BDSL_MIN_BLOCKS(K, NT, NR) ((K) == SOA64 ? 384 / (NT) : ((NR) == 1 ? QCU_BDSL32_BLOCKS * 128 / (NT) : 1))

// Tile = (group of NR rhs of one system, block of NT sites); every thread
// computes its site for all open rhs of the group, then the epilogue and the
// per-rhs reductions rhs by rhs.
template <int K, int G, bool CLOV, int NX, int RED, int NT, int NR, typename WR>
__device__ __forceinline__ void kb_dslash_tile(const BatchArgs &a, const int2 tile, const BDslOp &op, WR &wr,
                                               const BlockBatch &bb) {
  using T = Real<K>;
  constexpr int C = K == SOA64 ? CSOA64 : CSOA32;
  const RhsGroup &grp = bb.grp[tile.x];
  bool on[NR];
  bool any = false;
#pragma unroll
  for (int j = 0; j < NR; j++) {
    on[j] = j < grp.n && bb.open[grp.rhs[j]];
    any = any || on[j];
  }
  if (!any) return;
  const RhsDesc &d0 = a.d[grp.rhs[0]];  // lattice, links, clover and kappa are the group's system's
  constexpr int NV = RED == RED_NONE ? 1 : (RED == RED_TS_TT ? 3 : (RED == RED_DOT_RT ? 2 : 1));
  double red[NR][NV];
#pragma unroll
  for (int j = 0; j < NR; j++)
#pragma unroll
    for (int k = 0; k < NV; k++) red[j][k] = 0.0;
  const Geom g = d0.g;
  const int s = tile.y * NT + threadIdx.x;
  if (s < g.Vh) {
    Cpx<T> w[NR][12];
    SpinorView<K> in[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) in[j] = bview<K>(a.d[grp.rhs[j]], op.in);  // empty slots repeat the first rhs
    const GaugeView<G> U{K == SOA64 ? d0.g64 : d0.gin, pad_sites(g.Vh)};
    T unit = T(1);
    if constexpr (K == SOA32 || K == SOA16) {
      Site2 w2[NR];
      unit = wilson_hop_group2<K, G, NR>(w2, in, U, g, s, op.parity, (float)d0.t_bc);
#pragma unroll
      for (int j = 0; j < NR; j++) site2_to_cpx(w2[j], w[j]);
    } else {
      wilson_hop_group<K, G, T, NR>(w, in, on, U, g, s, op.parity, (T)d0.t_bc);
    }
    const void *cl = CLOV ? (K == SOA64 ? d0.c64[op.parity] : d0.cin[op.parity]) : nullptr;
    const T aa = (T)(op.a0 + op.ak * d0.kappa + op.ak2 * d0.k2) * unit;
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (!on[j]) continue;
      const RhsDesc &d = a.d[grp.rhs[j]];
      if constexpr (CLOV) {
        if (cl) clover_apply_site<C, T>(CloverView<C>{cl, g.Vh}, s, w[j]);
      }
#pragma unroll
      for (int c = 0; c < 12; c++) w[j][c] = w[j][c] * aa;
      Cpx<T> x1[12];
      if constexpr (NX >= 1) {
        spinor_load<K, T>(bview<K>(d, op.x1), s, x1);
#pragma unroll
        for (int c = 0; c < 12; c++) w[j][c] += x1[c] * (T)op.b1;
      }
      if constexpr (NX >= 2) {
        Cpx<T> x2[12];
        spinor_load<K, T>(bview<K>(d, op.x2), s, x2);
#pragma unroll
        for (int c = 0; c < 12; c++) w[j][c] += x2[c] * (T)op.b2;
      }
      spinor_store<K, T>(bview<K>(d, op.out), s, w[j]);
      if constexpr (RED == RED_DOT_RT) {  // <rt, out>
        Cpx<T> rt[12];
        spinor_load<K, T>(bview<K>(d, op.rt), s, rt);
        site_dot<T>(rt, w[j], red[j][0], red[j][1]);
      } else if constexpr (RED == RED_TS_TT) {  // <out, x1>, |out|^2
        site_dot<T>(w[j], x1, red[j][0], red[j][1]);
        site_norm2<T>(w[j], red[j][2]);
      } else if constexpr (RED == RED_NORM) {
        site_norm2<T>(w[j], red[j][0]);
      }
    }
  }
  if constexpr (RED != RED_NONE) {
#pragma unroll
    for (int j = 0; j < NR; j++)
      if (on[j]) warp_red_add(wr, grp.rhs[j], red[j]);  // on[j] is uniform per block
  }
}

// ---------------------------------------------------------------- inner BiCGSTAB iteration
constexpr int BB = 128;  // threads per BLAS tile

#define BTILE_SITES(a, tile, d)                                                    \
  const int s_begin = (tile).y * (a).tile_sites;                                   \
  const int s_end = min(s_begin + (a).tile_sites, (d).g.Vh);

// p = r + beta (p - omega v),  beta = (rho/rho_prev)(alpha/omega)
template <int K>
__device__ __forceinline__ void kb_pupdate_tile(const BatchArgs &a, const int2 tile, const BlockBatch &bb) {
  using T = Real<K>;
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  SolverState *st = a.st + tile.x;
  const Cpx<double> rho(st->rho[0], st->rho[1]), rho_prev(st->rho_prev[0], st->rho_prev[1]),
      alpha(st->alpha[0], st->alpha[1]), omega(st->omega[0], st->omega[1]);
  const Cpx<double> beta = cdiv(rho, rho_prev) * cdiv(alpha, omega);
  if (tile.y == 0 && threadIdx.x == 0) {
    st->beta[0] = beta.re;
    st->beta[1] = beta.im;
  }
  const Cpx<T> b((T)beta.re, (T)beta.im), w((T)omega.re, (T)omega.im);
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    Cpx<T> r[12], p[12], v[12];
    spinor_load<K, T>(bview<K>(d, BV_R), s, r);
    spinor_load<K, T>(bview<K>(d, BV_P), s, p);
    spinor_load<K, T>(bview<K>(d, BV_V), s, v);
#pragma unroll
    for (int c = 0; c < 12; c++) p[c] = r[c] + (p[c] - v[c] * w) * b;
    spinor_store<K, T>(bview<K>(d, BV_P), s, p);
  }
}

// s = r - alpha v
template <int K>
__device__ __forceinline__ void kb_supdate_tile(const BatchArgs &a, const int2 tile, const BlockBatch &bb) {
  using T = Real<K>;
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  const SolverState *st = a.st + tile.x;
  const Cpx<T> al((T)st->alpha[0], (T)st->alpha[1]);
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    Cpx<T> r[12], v[12];
    spinor_load<K, T>(bview<K>(d, BV_R), s, r);
    spinor_load<K, T>(bview<K>(d, BV_V), s, v);
#pragma unroll
    for (int c = 0; c < 12; c++) r[c] = r[c] - v[c] * al;
    spinor_store<K, T>(bview<K>(d, BV_S), s, r);
  }
}

// x += alpha p + omega s ; r = s - omega t ; <rt, r>, |r|^2 -> FIN_XR
template <int K, int XK, typename WR>
__device__ __forceinline__ void kb_xrupdate_tile(const BatchArgs &a, const int2 tile, WR &wr, const BlockBatch &bb) {
  using T = Real<K>;
  using TX = Real<XK>;
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  const SolverState *st = a.st + tile.x;
  const Cpx<T> w((T)st->omega[0], (T)st->omega[1]);
  const Cpx<TX> ax((TX)st->alpha[0], (TX)st->alpha[1]), wx((TX)st->omega[0], (TX)st->omega[1]);
  double red[3] = {0, 0, 0};
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    Cpx<T> p[12], q[12], t[12];
    Cpx<TX> x[12];
    spinor_load<K, T>(bview<K>(d, BV_P), s, p);
    spinor_load<K, T>(bview<K>(d, BV_S), s, q);
    spinor_load<XK, TX>(bview<XK>(d, BV_X), s, x);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      x[c] += Cpx<TX>((TX)p[c].re, (TX)p[c].im) * ax;
      x[c] += Cpx<TX>((TX)q[c].re, (TX)q[c].im) * wx;
    }
    spinor_store<XK, TX>(bview<XK>(d, BV_X), s, x);
    spinor_load<K, T>(bview<K>(d, BV_T), s, t);
#pragma unroll
    for (int c = 0; c < 12; c++) q[c] = q[c] - t[c] * w;
    spinor_store<K, T>(bview<K>(d, BV_R), s, q);
    spinor_load<K, T>(bview<K>(d, BV_RT), s, p);
    site_dot<T>(p, q, red[0], red[1]);
    site_norm2<T>(q, red[2]);
  }
  warp_red_add(wr, tile.x, red);
}

// r = rt = r64, p = v = x = 0 ; <rt, r>, |r64|^2 -> FIN_INIT.  An inactive
// rhs reduces zeros, which FIN_INIT (inner mode) turns into "done".
template <int K, int XK, typename WR>
__device__ __forceinline__ void kb_init_tile(const BatchArgs &a, const int2 tile, WR &wr, const BlockBatch &bb) {
  using T = Real<K>;
  using TX = Real<XK>;
  const RhsDesc &d = a.d[tile.x];
  double red[3] = {0, 0, 0};
  if (bb.open[tile.x]) {
    BTILE_SITES(a, tile, d)
    for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
      Cpx<double> r64[12];
      Cpx<T> r[12], z[12];
      Cpx<TX> zx[12];
      spinor_load<SOA64, double>(bview<SOA64>(d, BV_R64), s, r64);
#pragma unroll
      for (int c = 0; c < 12; c++) {
        r[c] = Cpx<T>((T)r64[c].re, (T)r64[c].im);
        z[c] = Cpx<T>(0, 0);
        zx[c] = Cpx<TX>(0, 0);
        red[0] += (double)r[c].re * r[c].re + (double)r[c].im * r[c].im;
        red[2] += r64[c].re * r64[c].re + r64[c].im * r64[c].im;
      }
      spinor_store<K, T>(bview<K>(d, BV_R), s, r);
      spinor_store<K, T>(bview<K>(d, BV_RT), s, r);
      spinor_store<K, T>(bview<K>(d, BV_P), s, z);
      spinor_store<K, T>(bview<K>(d, BV_V), s, z);
      spinor_store<XK, TX>(bview<XK>(d, BV_X), s, zx);
    }
  }
  warp_red_add(wr, tile.x, red);
}

// z = x in FP64 (active rhs)
template <int XK>
__device__ __forceinline__ void kb_xout_tile(const BatchArgs &a, const int2 tile, const BlockBatch &bb) {
  using TX = Real<XK>;
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    Cpx<double> z[12];
    spinor_load<XK, double>(bview<XK>(d, BV_X), s, z);
    spinor_store<SOA64, double>(bview<SOA64>(d, BV_Z), s, z);
  }
}

// continue while any rhs is not done; after `cap` passes stop everything
__global__ void kb_loop_cond(BatchArgs a, cudaGraphConditionalHandle h, unsigned cap) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int r = threadIdx.x;
  if (r < a.nrhs && ((volatile SolverState *)(a.st + r))->done == 0) atomicOr(&any, 1);
  __syncthreads();
  __shared__ int go;
  if (threadIdx.x == 0) {
    const unsigned n = ++a.st[0].loop_guard;
    go = any;
    if (go && n >= cap) go = 0;
  }
  __syncthreads();
  if (!go && r < a.nrhs && a.st[r].done == 0) {
    a.st[r].status = ST_MAXITER;
    a.st[r].done = 1;
  }
  if (threadIdx.x == 0) cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ---------------------------------------------------------------- outer GCR step (FP64)
using C = Cpx<double>;

__device__ __forceinline__ void ld64(const void *p, int s, C v[12]) {
  const double2 *q = static_cast<const double2 *>(p) + blk_base<12>(s);
#pragma unroll
  for (int c = 0; c < 12; c++) {
    const double2 t = __ldg(q + c * SB);
    v[c] = C(t.x, t.y);
  }
}
__device__ __forceinline__ void st64(void *p, int s, const C v[12]) {
  double2 *q = static_cast<double2 *>(p) + blk_base<12>(s);
#pragma unroll
  for (int c = 0; c < 12; c++) q[c * SB] = make_double2(v[c].re, v[c].im);
}

// sums[2j], sums[2j+1] = <W_j, w>, j < k
__device__ __forceinline__ void kb_gcr_multidot_tile(const BatchArgs &a, const int2 tile, int k, const BlockBatch &bb) {
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  double red[2 * GCR_MAXK];
#pragma unroll
  for (int j = 0; j < 2 * GCR_MAXK; j++) red[j] = 0.0;
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    C w[12];
    ld64(d.v[BV_W], s, w);
#pragma unroll
    for (int j = 0; j < GCR_MAXK; j++) {
      if (j < k) {
        const double2 *Wj = static_cast<const double2 *>(d.W[j]) + blk_base<12>(s);
#pragma unroll
        for (int c = 0; c < 12; c++) {
          const double2 q = __ldg(Wj + c * SB);
          red[2 * j] += q.x * w[c].re + q.y * w[c].im;
          red[2 * j + 1] += q.x * w[c].im - q.y * w[c].re;
        }
      }
    }
  }
  batch_reduce<2 * GCR_MAXK, BB>(red, a, tile.x, tile.y, FIN_STORE);
}

// W_k = w - sum beta_j W_j, Z_k = z - sum beta_j Z_j ; sums = |W_k|^2, <W_k, r>
__device__ __forceinline__ void kb_gcr_orth_tile(const BatchArgs &a, const int2 tile, int k, const BlockBatch &bb) {
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  const BatchCoef &cf = a.coef[tile.x];
  double red[3] = {0, 0, 0};
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    C w[12], z[12], q[12];
    ld64(d.v[BV_W], s, w);
    ld64(d.v[BV_Z], s, z);
    for (int j = 0; j < k; j++) {
      const C b(cf.beta[2 * j], cf.beta[2 * j + 1]);
      ld64(d.W[j], s, q);
#pragma unroll
      for (int c = 0; c < 12; c++) w[c] -= b * q[c];
      ld64(d.Z[j], s, q);
#pragma unroll
      for (int c = 0; c < 12; c++) z[c] -= b * q[c];
    }
    st64(d.W[k], s, w);
    st64(d.Z[k], s, z);
    ld64(d.v[BV_R64], s, q);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      red[0] += w[c].norm2();
      const C t = cdotmul(w[c], q[c]);
      red[1] += t.re;
      red[2] += t.im;
    }
  }
  batch_reduce<3, BB>(red, a, tile.x, tile.y, FIN_STORE);
}

// x64 += alpha Z_k ; r64 -= alpha W_k ; sums[0] = |r64|^2
__device__ __forceinline__ void kb_gcr_update_tile(const BatchArgs &a, const int2 tile, int k, const BlockBatch &bb) {
  if (!bb.open[tile.x]) return;
  const RhsDesc &d = a.d[tile.x];
  const C al(a.coef[tile.x].alpha[0], a.coef[tile.x].alpha[1]);
  double red[1] = {0};
  BTILE_SITES(a, tile, d)
  for (int s = s_begin + threadIdx.x; s < s_end; s += BB) {
    C x[12], q[12];
    ld64(d.v[BV_X64], s, x);
    ld64(d.Z[k], s, q);
#pragma unroll
    for (int c = 0; c < 12; c++) x[c] += al * q[c];
    st64(d.v[BV_X64], s, x);
    ld64(d.v[BV_R64], s, x);
    ld64(d.W[k], s, q);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      x[c] -= al * q[c];
      red[0] += x[c].norm2();
    }
    st64(d.v[BV_R64], s, x);
  }
  batch_reduce<1, BB>(red, a, tile.x, tile.y, FIN_STORE);
}

// ---------------------------------------------------------------- persistent wrappers
// Each kernel loops over the tile table with a grid of resident blocks: a tile
// of a converged rhs costs a few instructions instead of a block launch.
template <int K, int G, bool CLOV, int NX, int RED, int NT, int NR>
__global__ void __launch_bounds__(NT, BDSL_MIN_BLOCKS(K, NT, NR)) kb_dslash(BatchArgs a, BDslOp op) {
  constexpr int NV = RED == RED_NONE ? 1 : (RED == RED_TS_TT ? 3 : (RED == RED_DOT_RT ? 2 : 1));
  __shared__ WarpRed<NV, NT / 32> wr;
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, op.gate);
  if constexpr (RED != RED_NONE) warp_red_zero(wr);
  for_tiles(a, bb, [&](int2 tile) { kb_dslash_tile<K, G, CLOV, NX, RED, NT, NR>(a, tile, op, wr, bb); });
  if constexpr (RED != RED_NONE) warp_red_post(a, wr, op.fin, op.gate);
}

template <int K>
__global__ void __launch_bounds__(BB) kb_pupdate(BatchArgs a) {
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_NOT_DONE);
  for_tiles(a, bb, [&](int2 tile) { kb_pupdate_tile<K>(a, tile, bb); });
}

template <int K>
__global__ void __launch_bounds__(BB) kb_supdate(BatchArgs a) {
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_NOT_DONE);
  for_tiles(a, bb, [&](int2 tile) { kb_supdate_tile<K>(a, tile, bb); });
}

template <int K, int XK>
__global__ void __launch_bounds__(BB) kb_xrupdate(BatchArgs a) {
  __shared__ WarpRed<3, BB / 32> wr;
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_NOT_DONE);
  warp_red_zero(wr);
  for_tiles(a, bb, [&](int2 tile) { kb_xrupdate_tile<K, XK>(a, tile, wr, bb); });
  warp_red_post(a, wr, FIN_XR, BG_NOT_DONE);
}

template <int K, int XK>
__global__ void __launch_bounds__(BB) kb_init(BatchArgs a) {
  __shared__ WarpRed<3, BB / 32> wr;
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_ACTIVE);
  warp_red_zero(wr);
  for_tiles(a, bb, [&](int2 tile) { kb_init_tile<K, XK>(a, tile, wr, bb); });
  warp_red_post(a, wr, FIN_INIT, BG_ALWAYS);  // inactive rhs reduce zeros: FIN_INIT marks them done
}

template <int XK>
__global__ void __launch_bounds__(BB) kb_xout(BatchArgs a) {
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_ACTIVE);
  for_tiles(a, bb, [&](int2 tile) { kb_xout_tile<XK>(a, tile, bb); });
}

__global__ void __launch_bounds__(BB) kb_gcr_multidot(BatchArgs a, int k) {
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_ACTIVE);
  for_tiles(a, bb, [&](int2 tile) { kb_gcr_multidot_tile(a, tile, k, bb); });
}

__global__ void __launch_bounds__(BB) kb_gcr_orth(BatchArgs a, int k) {
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_ACTIVE);
  for_tiles(a, bb, [&](int2 tile) { kb_gcr_orth_tile(a, tile, k, bb); });
}

__global__ void __launch_bounds__(BB) kb_gcr_update(BatchArgs a, int k) {
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, BG_ACTIVE);
  for_tiles(a, bb, [&](int2 tile) { kb_gcr_update_tile(a, tile, k, bb); });
}

// ---------------------------------------------------------------- launchers
// Grid of a persistent batched kernel: as many blocks as the SMs can hold by
// thread count (or fewer when the table has fewer tiles); each block then
// walks the tile table with a stride of the grid.
static int persistent_grid(const BatchArgs &a, int threads) {
  const int cap = std::min(BATCH_POST_GRID, std::max(1, a.sms) * std::max(1, 1024 / threads));
  return std::max(1, std::min(a.ntiles, cap));
}
// the hopping kernels: the blocks their registers let reside per SM
static int dslash_grid(const BatchArgs &a, int per_sm) {
  const int cap = std::min(BATCH_POST_GRID, std::max(1, a.sms) * std::max(1, per_sm));
  return std::max(1, std::min(a.ntiles, cap));
}
template <int K, int G, bool CLOV, int NT, int NR>
static void bdsl_nx(const BatchArgs &a, const BDslOp &op, cudaStream_t s) {
  const int nx = op.x2 >= 0 ? 2 : (op.x1 >= 0 ? 1 : 0);
  constexpr int per_sm = (K != SOA64 && NR == 1) ? 512 / NT : 384 / NT;
#define QCU_BD(NX, RED) kb_dslash<K, G, CLOV, NX, RED, NT, NR><<<dslash_grid(a, per_sm), NT, 0, s>>>(a, op)
  // the combinations the batched solver uses: inner (0,-), (1,<rt,v>), (1,<t,s>|t|^2);
  // FP64 outer (0,-), (1,-), (2,|r|^2)
  if (nx == 0 && op.red == RED_NONE) {
    QCU_BD(0, RED_NONE);
  } else if constexpr (K == SOA64) {  // outer operator, and the inner one at precision 64
    if (nx == 1 && op.red == RED_NONE) QCU_BD(1, RED_NONE);
    else if (nx == 2 && op.red == RED_NORM) QCU_BD(2, RED_NORM);
    else if (nx == 1 && op.red == RED_DOT_RT) QCU_BD(1, RED_DOT_RT);
    else if (nx == 1 && op.red == RED_TS_TT) QCU_BD(1, RED_TS_TT);
    else throw Error(1, "batched FP64 dslash: unsupported epilogue/reduction combination");
  } else {
    if (nx == 1 && op.red == RED_DOT_RT) QCU_BD(1, RED_DOT_RT);
    else if (nx == 1 && op.red == RED_TS_TT) QCU_BD(1, RED_TS_TT);
    else throw Error(1, "batched dslash: unsupported epilogue/reduction combination");
  }
#undef QCU_BD
  QCU_CHECK_LAUNCH();
}

template <int K, int G, int NT, int NR>
static void bdsl_clov(const BatchArgs &a, const BDslOp &op, cudaStream_t s) {
  if (op.clover) bdsl_nx<K, G, true, NT, NR>(a, op, s);
  else bdsl_nx<K, G, false, NT, NR>(a, op, s);
}

template <int K, int G>
static void bdsl_shape(const BatchArgs &a, const BDslOp &op, const BatchTune &t, cudaStream_t s) {
  require(a.tile_sites == t.dslash_threads && a.groups != nullptr, "batched dslash: tile table does not match");
  if constexpr (K == SOA64) {
    require(t.dslash_threads == 128 && t.dslash_rhs == 1, "batched FP64 dslash: 128 threads, 1 rhs per thread");
    bdsl_clov<K, G, 128, 1>(a, op, s);
  } else {
    const int key = t.dslash_threads * 10 + t.dslash_rhs;
    switch (key) {
      case 641: bdsl_clov<K, G, 64, 1>(a, op, s); break;
      case 1281: bdsl_clov<K, G, 128, 1>(a, op, s); break;
      case 2561: bdsl_clov<K, G, 256, 1>(a, op, s); break;
      case 642: bdsl_clov<K, G, 64, 2>(a, op, s); break;
      case 1282: bdsl_clov<K, G, 128, 2>(a, op, s); break;
      case 644: bdsl_clov<K, G, 64, 4>(a, op, s); break;
      case 1284: bdsl_clov<K, G, 128, 4>(a, op, s); break;
      default: throw Error(1, "batched dslash: unsupported block shape");
    }
  }
}

void launch_bdslash_mma(int gkind, int mode, const BatchArgs &a, const BDslOp &op, cudaStream_t s);

void launch_bdslash(int kind, int gkind, const BatchArgs &a, const BDslOp &op, const BatchTune &t, cudaStream_t s) {
  if (a.ntiles == 0) return;
  if (t.mma) {
    require(kind == SOA32, "tensor-core dslash: FP32 spinors only");
    launch_bdslash_mma(gkind, t.mma, a, op, s);
    return;
  }
  if (kind == SOA64 && gkind == GSOA64) bdsl_shape<SOA64, GSOA64>(a, op, t, s);
  else if (kind == SOA32 && gkind == GSOA32) bdsl_shape<SOA32, GSOA32>(a, op, t, s);
  else if (kind == SOA32 && gkind == GSOA16) bdsl_shape<SOA32, GSOA16>(a, op, t, s);
  else if (kind == SOA16 && gkind == GSOA16) bdsl_shape<SOA16, GSOA16>(a, op, t, s);
  else throw Error(1, "batched dslash: unsupported storage combination");
}

void launch_bpupdate(int kind, const BatchArgs &a, cudaStream_t s) {
  if (kind == SOA64) kb_pupdate<SOA64><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else if (kind == SOA16) kb_pupdate<SOA16><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else kb_pupdate<SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  QCU_CHECK_LAUNCH();
}
void launch_bsupdate(int kind, const BatchArgs &a, cudaStream_t s) {
  if (kind == SOA64) kb_supdate<SOA64><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else if (kind == SOA16) kb_supdate<SOA16><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else kb_supdate<SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  QCU_CHECK_LAUNCH();
}
void launch_bxrupdate(int kind, const BatchArgs &a, cudaStream_t s) {
  if (kind == SOA64) kb_xrupdate<SOA64, SOA64><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else if (kind == SOA16) kb_xrupdate<SOA16, SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);  // x in FP32
  else kb_xrupdate<SOA32, SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  QCU_CHECK_LAUNCH();
}
void launch_binit(int kind, const BatchArgs &a, cudaStream_t s) {
  if (kind == SOA64) kb_init<SOA64, SOA64><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else if (kind == SOA16) kb_init<SOA16, SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else kb_init<SOA32, SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  QCU_CHECK_LAUNCH();
}
void launch_bxout(int kind, const BatchArgs &a, cudaStream_t s) {
  if (kind == SOA64) kb_xout<SOA64><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  else kb_xout<SOA32><<<persistent_grid(a, BB), BB, 0, s>>>(a);
  QCU_CHECK_LAUNCH();
}
void launch_bloop_cond(const BatchArgs &a, cudaGraphConditionalHandle h, unsigned cap, cudaStream_t s) {
  require(a.nrhs <= BATCH_MAX_RHS, "too many right-hand sides");
  kb_loop_cond<<<1, BATCH_MAX_RHS, 0, s>>>(a, h, cap);
  QCU_CHECK_LAUNCH();
}
void launch_bgcr_multidot(const BatchArgs &a, int k, cudaStream_t s) {
  kb_gcr_multidot<<<persistent_grid(a, BB), BB, 0, s>>>(a, k);
  QCU_CHECK_LAUNCH();
}
void launch_bgcr_orth(const BatchArgs &a, int k, cudaStream_t s) {
  kb_gcr_orth<<<persistent_grid(a, BB), BB, 0, s>>>(a, k);
  QCU_CHECK_LAUNCH();
}
void launch_bgcr_update(const BatchArgs &a, int k, cudaStream_t s) {
  kb_gcr_update<<<persistent_grid(a, BB), BB, 0, s>>>(a, k);
  QCU_CHECK_LAUNCH();
}

}  // namespace qcu
