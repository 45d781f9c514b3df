// Tensor-core path of the batched inner dslash: the link x half-spinor
// products of 8 right-hand sides at one site are one warp-level contraction
// per hop on the tensor pipe (mma.sync m16n8k8, TF32 operands, FP32
// accumulation).
//
// Real form of one hop at one site, for the 8 rhs g of a group:
//   D[row][n] += sum_k A[row][k] B[k][n]
//   k = 2c + part      (input colour c, real/imaginary part; k = 6, 7 zero)
//   n = 2r + part      (output colour r; n = 6, 7 zero)
//   B[2c+i][2r+o] = Re u_rc (i == o), Im u_rc (i = 0, o = 1), -Im u_rc (i = 1, o = 0)
// with u = U_mu(x) (forward hop) or U_mu(x-mu)^dag (backward hop), the
// boundary phase folded in.  Two accumulator tiles per site: rows (g, spin 0),
// (g, spin 1) take the projected half spinor h_k = psi_k + s g_k psi_gcol(k)
// (src/wilson_dslash.cu:56-243), rows (g, spin 2), (g, spin 3) take the
// lower-spin reconstruction s g_m h_gcol(m) -- the link is linear, so
// u (s g h) = s g (u h) and all 8 hops accumulate in the same two tiles.
//
// Mode 1 splits each operand into a TF32 head and a TF32 tail (x = hi + lo)
// and takes the product as lo*hi + hi*lo + hi*hi, which keeps the result to
// within a few units of FP32 rounding (the hi/lo split of 3xTF32 GEMMs); the
// autotuner may choose it in place of the FP32 kernel.  Mode 2 takes single
// TF32 products (11-bit operands): a lower-precision inner operator, used
// only when asked for.
//
// Block: 8 warps, tile = 32 sites x one group of <= 8 rhs.  Phase 1: warp h
// loads, decodes and stores the link of hop h for the 32 sites.  Phase 2, per
// hop: warp j loads rhs j's neighbour spinors (one lane per site, the
// coalesced pattern of the scalar kernel) and stores their projections in
// shared memory; then each warp contracts 4 sites for all 8 rhs.  Phase 3:
// warp j runs the epilogue (clover, axpy, store, fused reduction) of rhs j
// with one lane per site.
#include <algorithm>

#include "batch_dev.cuh"

namespace qcu {

constexpr int MMA_SITES = 32;
constexpr int MMA_THREADS = 256;

__device__ __forceinline__ uint32_t tf32_rn(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
  hi = tf32_rn(x);
  lo = tf32_rn(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// d += a b with both operands split (3 tensor-core products)
__device__ __forceinline__ void mma3(float (&d)[4], const float (&a)[4], const uint32_t (&bh)[2],
                                     const uint32_t (&bl)[2]) {
  uint32_t ah[4], al[4];
#pragma unroll
  for (int i = 0; i < 4; i++) tf32_split(a[i], ah[i], al[i]);
  mma_tf32(d, al, bh);
  mma_tf32(d, ah, bl);
  mma_tf32(d, ah, bh);
}

__device__ __forceinline__ float part(const Cpx<float> &z, int p) { return p ? z.im : z.re; }

// neighbour site and link of hop h (mu = h/2, forward for even h) of site s
__device__ __forceinline__ void hop_geometry(const Geom &g, int s, int par, int h, int &n, int &lpar, int &ls,
                                             bool &boundary) {
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  const int y = r % g.Ly;
  r /= g.Ly;
  const int z = r % g.Lz;
  const int t = r / g.Lz;
  const int xodd = (y + z + t + par) & 1;
  const int mu = h >> 1;
  const bool fwd = (h & 1) == 0;
  boundary = false;
  switch (mu) {
    case 0:
      n = fwd ? (xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s) : (xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1));
      break;
    case 1:
      n = fwd ? ((y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy) : ((y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy);
      break;
    case 2:
      n = fwd ? ((z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz) : ((z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz);
      break;
    default:
      n = fwd ? ((t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st) : ((t == 0) ? s + (g.Lt - 1) * g.st : s - g.st);
      boundary = fwd ? (t == g.Lt - 1) : (t == 0);
      break;
  }
  lpar = fwd ? par : 1 - par;
  ls = fwd ? s : n;
}

// Projected half spinors of hop H for one site and one rhs: h_k = psi_k + s g_k psi_gcol(k)
template <int H>
__device__ __forceinline__ void project(const Cpx<float> (&psi)[12], Cpx<float> (&h)[6]) {
  constexpr int MU = H >> 1;
  constexpr int S = (H & 1) == 0 ? -1 : 1;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    h[c] = psi[c] + unit_mul<S * gre(MU, 0), S * gim(MU, 0)>(psi[gcol(MU, 0) * 3 + c]);
    h[3 + c] = psi[3 + c] + unit_mul<S * gre(MU, 1), S * gim(MU, 1)>(psi[gcol(MU, 1) * 3 + c]);
  }
}

// Contraction of hop H for one site: A tiles from the staged half spinors of
// the 8 rhs (lane g = rhs slot, lane t = k column), B from the staged link.
// SPLIT 3: 3xTF32 (FP32-accurate); 1: one TF32 product.
template <int H, int SPLIT>
__device__ __forceinline__ void mma_hop(float (&d1)[4], float (&d2)[4], const float2 (*hs)[6][MMA_SITES + 1], int sl,
                                        const float2 *u, int g, int t) {
  constexpr int MU = H >> 1;
  constexpr int S = (H & 1) == 0 ? -1 : 1;
  const int c1 = t >> 1, pt = t & 1;
  const bool has2 = t < 2;  // column t + 4 is colour 2 for t < 2, padding otherwise
  const float2 (*h)[MMA_SITES + 1] = hs[g];  // [component][site] of rhs slot g
  auto cx = [](float2 v) { return Cpx<float>(v.x, v.y); };
  Cpx<float> h1[2], h2[2];  // half spins k = 0, 1 at colours c1 and 2
  h1[0] = cx(h[c1][sl]);
  h1[1] = cx(h[3 + c1][sl]);
  h2[0] = has2 ? cx(h[2][sl]) : Cpx<float>(0, 0);
  h2[1] = has2 ? cx(h[5][sl]) : Cpx<float>(0, 0);
  // lower spins: s g_m h_gcol(m)
  const Cpx<float> l1_2 = unit_mul<S * gre(MU, 2), S * gim(MU, 2)>(h1[gcol(MU, 2)]);
  const Cpx<float> l1_3 = unit_mul<S * gre(MU, 3), S * gim(MU, 3)>(h1[gcol(MU, 3)]);
  const Cpx<float> l2_2 = unit_mul<S * gre(MU, 2), S * gim(MU, 2)>(h2[gcol(MU, 2)]);
  const Cpx<float> l2_3 = unit_mul<S * gre(MU, 3), S * gim(MU, 3)>(h2[gcol(MU, 3)]);
  const float a_up[4] = {part(h1[0], pt), part(h1[1], pt), part(h2[0], pt), part(h2[1], pt)};
  const float a_lo[4] = {part(l1_2, pt), part(l1_3, pt), part(l2_2, pt), part(l2_3, pt)};
  // B fragment: rows k = t and t + 4, column n = g
  float b[2] = {0.f, 0.f};
  if (g < 6) {
    const int r = g >> 1, o = g & 1;
    const Cpx<float> ua = cx(u[r * 3 + c1]);
    b[0] = pt == o ? ua.re : (pt == 0 ? ua.im : -ua.im);
    if (has2) {
      const Cpx<float> ub = cx(u[r * 3 + 2]);
      b[1] = pt == o ? ub.re : (pt == 0 ? ub.im : -ub.im);
    }
  }
  if constexpr (SPLIT == 3) {
    uint32_t bh[2], bl[2];
    tf32_split(b[0], bh[0], bl[0]);
    tf32_split(b[1], bh[1], bl[1]);
    mma3(d1, a_up, bh, bl);
    mma3(d2, a_lo, bh, bl);
  } else {
    const uint32_t bb[2] = {tf32_rn(b[0]), tf32_rn(b[1])};
    const uint32_t au[4] = {tf32_rn(a_up[0]), tf32_rn(a_up[1]), tf32_rn(a_up[2]), tf32_rn(a_up[3])};
    const uint32_t al[4] = {tf32_rn(a_lo[0]), tf32_rn(a_lo[1]), tf32_rn(a_lo[2]), tf32_rn(a_lo[3])};
    mma_tf32(d1, au, bb);
    mma_tf32(d2, al, bb);
  }
}

// shared memory of one block: links and neighbours of the 8 hops, the
// projected half spinors of the current hop, then (aliasing both) the
// results of the 8 rhs for the epilogue
struct MmaSmem {
  union {
    struct {
      float2 u[8][MMA_SITES][9];
      float2 h[8][6][MMA_SITES + 1];  // [rhs slot][component][site]: padded against bank conflicts
    } in;
    float2 out[8][MMA_SITES][12];
  };
  int n[8][MMA_SITES];
};

// stage hop H: warp w = rhs slot w, lane = site; projected half spinors to smem
template <int H>
__device__ __forceinline__ void stage_hop(MmaSmem &sm, const float4 *in, bool live, int lane, int slot) {
  Cpx<float> h[6];
  if (live) {
    Cpx<float> psi[12];
    spinor_load<SOA32, float>(SpinorView<SOA32>{const_cast<float4 *>(in), nullptr, 0}, sm.n[H][lane], psi);
    project<H>(psi, h);
  } else {
#pragma unroll
    for (int k = 0; k < 6; k++) h[k] = Cpx<float>(0, 0);
  }
#pragma unroll
  for (int k = 0; k < 6; k++) sm.in.h[slot][k][lane] = make_float2(h[k].re, h[k].im);
}

template <int H, int SPLIT>
__device__ __forceinline__ void hop_step(MmaSmem &sm, float (&d1)[4][4], float (&d2)[4][4], const float4 *in,
                                         bool live_slot, int s0, int Vh, int warp, int lane) {
  stage_hop<H>(sm, in, live_slot && s0 + lane < Vh, lane, warp);
  __syncthreads();
  const int gq = lane >> 2, t = lane & 3;
#pragma unroll
  for (int q = 0; q < MMA_SITES / 8; q++) {
    const int sl = warp * (MMA_SITES / 8) + q;
    if (s0 + sl < Vh) mma_hop<H, SPLIT>(d1[q], d2[q], sm.in.h, sl, sm.in.u[H][sl], gq, t);  // warp-uniform
  }
  __syncthreads();
}

template <int G, bool CLOV, int NX, int RED, int SPLIT, typename WR>
__device__ __forceinline__ void kb_dslash_mma_tile(const BatchArgs &a, const int2 tile, const BDslOp &op,
                                                   MmaSmem &sm, WR &wr, const BlockBatch &bb) {
  const RhsGroup &grp = bb.grp[tile.x];
  bool on[8];
  bool any = false;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    on[j] = j < grp.n && bb.open[grp.rhs[j]];
    any = any || on[j];
  }
  if (!any) return;
  const RhsDesc &d0 = a.d[grp.rhs[0]];
  const Geom g = d0.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s0 = tile.y * MMA_SITES;

  // phase 1: warp h stages hop h's link (u = U or U^dag, phase folded) and neighbour
  {
    const int h = warp, s = s0 + lane;
    Cpx<float> u[9];
    int n = 0;
    if (s < g.Vh) {
      int lpar, ls;
      bool bnd;
      hop_geometry(g, s, op.parity, h, n, lpar, ls, bnd);
      const GaugeView<G> U{d0.gin, pad_sites(g.Vh)};
      Cpx<float> m[9];
      link_load<G, float>(U, h >> 1, lpar, ls, m);
      const float ph = bnd ? (float)d0.t_bc : 1.0f;
      if ((h & 1) == 0) {
#pragma unroll
        for (int k = 0; k < 9; k++) u[k] = m[k] * ph;
      } else {
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) u[r * 3 + c] = m[c * 3 + r].conj() * ph;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) u[k] = Cpx<float>(0, 0);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) sm.in.u[h][lane][k] = make_float2(u[k].re, u[k].im);
    sm.n[h][lane] = n;
  }
  __syncthreads();

  // phase 2: per hop, stage the 8 rhs' half spinors (warp = rhs slot), then
  // each warp contracts its 4 sites; accumulators stay in registers
  float d1[4][4], d2[4][4];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int k = 0; k < 4; k++) d1[q][k] = d2[q][k] = 0.f;
  {
    const bool live = warp < grp.n && on[warp];
    const float4 *in = static_cast<const float4 *>(a.d[grp.rhs[warp < grp.n ? warp : 0]].v[op.in]);
    hop_step<0, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<1, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<2, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<3, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<4, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<5, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<6, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
    hop_step<7, SPLIT>(sm, d1, d2, in, live, s0, g.Vh, warp, lane);
  }
  {
    const int gq = lane >> 2, t = lane & 3;
    if (t < 3) {  // column pair t = output colour t
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int sl = warp * 4 + q;
        sm.out[gq][sl][0 * 3 + t] = make_float2(d1[q][0], d1[q][1]);
        sm.out[gq][sl][1 * 3 + t] = make_float2(d1[q][2], d1[q][3]);
        sm.out[gq][sl][2 * 3 + t] = make_float2(d2[q][0], d2[q][1]);
        sm.out[gq][sl][3 * 3 + t] = make_float2(d2[q][2], d2[q][3]);
      }
    }
  }
  __syncthreads();

  // phase 3: warp j finishes rhs slot j, one lane per site
  constexpr int NV = RED == RED_NONE ? 1 : (RED == RED_TS_TT ? 3 : (RED == RED_DOT_RT ? 2 : 1));
  double red[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) red[k] = 0.0;
  const int j = warp;
  const bool on_j = j < grp.n && on[j];
  const int s = s0 + lane;
  if (on_j && s < g.Vh) {
    const RhsDesc &d = a.d[grp.rhs[j]];
    Cpx<float> w[12];
#pragma unroll
    for (int c = 0; c < 12; c++) w[c] = Cpx<float>(sm.out[j][lane][c].x, sm.out[j][lane][c].y);
    if constexpr (CLOV) {
      const void *cl = d0.cin[op.parity];
      if (cl) clover_apply_site<CSOA32, float>(CloverView<CSOA32>{cl, g.Vh}, s, w);
    }
    const float aa = (float)(op.a0 + op.ak * d0.kappa + op.ak2 * d0.k2);
#pragma unroll
    for (int c = 0; c < 12; c++) w[c] = w[c] * aa;
    Cpx<float> x1[12];
    if constexpr (NX >= 1) {
      spinor_load<SOA32, float>(bview<SOA32>(d, op.x1), s, x1);
#pragma unroll
      for (int c = 0; c < 12; c++) w[c] += x1[c] * (float)op.b1;
    }
    spinor_store<SOA32, float>(bview<SOA32>(d, op.out), s, w);
    if constexpr (RED == RED_DOT_RT) {  // <rt, out>
      Cpx<float> rt[12];
      spinor_load<SOA32, float>(bview<SOA32>(d, op.rt), s, rt);
      site_dot<float>(rt, w, red[0], red[1]);
    } else if constexpr (RED == RED_TS_TT) {  // <out, x1>, |out|^2
      site_dot<float>(w, x1, red[0], red[1]);
      site_norm2<float>(w, red[2]);
    }
  }
  if constexpr (RED != RED_NONE) {
    if (on_j) warp_red_add(wr, grp.rhs[j], red);  // warp j's share of rhs slot j
  }
  __syncthreads();  // the next tile overwrites the shared memory the epilogue read
}

template <int G, bool CLOV, int NX, int RED, int SPLIT>
__global__ void __launch_bounds__(MMA_THREADS) kb_dslash_mma(BatchArgs a, BDslOp op) {
  constexpr int NV = RED == RED_NONE ? 1 : (RED == RED_TS_TT ? 3 : (RED == RED_DOT_RT ? 2 : 1));
  __shared__ MmaSmem sm;
  __shared__ WarpRed<NV, MMA_THREADS / 32> wr;
  __shared__ BlockBatch bb;
  block_batch_init(a, bb, op.gate);
  if constexpr (RED != RED_NONE) warp_red_zero(wr);
  for_tiles(a, bb, [&](int2 tile) { kb_dslash_mma_tile<G, CLOV, NX, RED, SPLIT>(a, tile, op, sm, wr, bb); });
  if constexpr (RED != RED_NONE) warp_red_post(a, wr, op.fin, op.gate);
}

template <int G, bool CLOV, int SPLIT>
static void mma_nx(const BatchArgs &a, const BDslOp &op, cudaStream_t s) {
  const int nx = op.x2 >= 0 ? 2 : (op.x1 >= 0 ? 1 : 0);
  const dim3 grid(std::max(1, std::min(a.ntiles, std::min(BATCH_POST_GRID, std::max(1, a.sms) * 2)))),
      block(MMA_THREADS);  // 2 resident per SM
  if (nx == 0 && op.red == RED_NONE) kb_dslash_mma<G, CLOV, 0, RED_NONE, SPLIT><<<grid, block, 0, s>>>(a, op);
  else if (nx == 1 && op.red == RED_DOT_RT) kb_dslash_mma<G, CLOV, 1, RED_DOT_RT, SPLIT><<<grid, block, 0, s>>>(a, op);
  else if (nx == 1 && op.red == RED_TS_TT) kb_dslash_mma<G, CLOV, 1, RED_TS_TT, SPLIT><<<grid, block, 0, s>>>(a, op);
  else throw Error(1, "tensor-core dslash: unsupported epilogue/reduction combination");
  QCU_CHECK_LAUNCH();
}

template <int G>
static void mma_clov(const BatchArgs &a, const BDslOp &op, int mode, cudaStream_t s) {
  if (mode == 1) {
    if (op.clover) mma_nx<G, true, 3>(a, op, s);
    else mma_nx<G, false, 3>(a, op, s);
  } else {
    if (op.clover) mma_nx<G, true, 1>(a, op, s);
    else mma_nx<G, false, 1>(a, op, s);
  }
}

// mode 1: 3xTF32 products (FP32-accurate); mode 2: single TF32 products
void launch_bdslash_mma(int gkind, int mode, const BatchArgs &a, const BDslOp &op, cudaStream_t s) {
  require(a.tile_sites == MMA_SITES && a.groups != nullptr, "tensor-core dslash: tile table must have 32 sites");
  require(mode == 1 || mode == 2, "tensor-core dslash: mode must be 1 (3xTF32) or 2 (TF32)");
  if (gkind == GSOA16) mma_clov<GSOA16>(a, op, mode, s);
  else if (gkind == GSOA32) mma_clov<GSOA32>(a, op, mode, s);
  else throw Error(1, "tensor-core dslash: links must be 16 or 32 bit");
}

}  // namespace qcu
