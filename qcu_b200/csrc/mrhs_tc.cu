// Multi-right-hand-side Wilson hopping term on the 5th-generation tensor
// cores (tcgen05).
//
// For R right-hand sides of one system the hop sum at an output site x,
//     out_r(x) = sum_h V_h (1 + S_h gamma_mu) psi_r(x + h)        (8 hops h)
// (qcu's wilson_dslash, src/wilson_dslash.cu:9-245, for each r) is, per hop,
// one real matrix product that every right-hand side shares:
//     [out_r components] += [psi_r(x + h) components] x B_h^T,
//     B_h = real form of (1 + S gamma_mu) (x) V_h    (24 x 24: spin, colour, re/im)
// with V_h = U_mu(x) (forward, S = -1) or U_mu(x - mu)^dag (backward, S = +1),
// times the time-boundary phase.  A site is therefore one GEMM with M = R
// (right-hand sides), N = 24 output components and K = 8 hops x 24 input
// components: projection, colour product and reconstruction all run on the
// tensor core, and the only per-rhs work left to the threads is the epilogue.
//
// Layout of a multi-rhs field (one parity, FP16): site-major; within a site,
// 3 K-chunks of 8 components (16 B) for each of the RP rows (right-hand sides
// padded to RP = 64 or 128, padding rows zero):
//     element (site s, rhs r, component k) at  s * 24 RP + (k / 8) * 8 RP + r * 8 + k % 8
// (halves), components k = (spin * 3 + colour) * 2 + (re, im) as in PyQuda.
// That is the K-major, no-swizzle operand layout of tcgen05 (core matrices
// of 8 rows x 16 B, LBO = 16 RP B between K-chunks, SBO = 128 B between
// 8-row groups), so one bulk copy brings a neighbour's whole A tile.
//
// Persistent CTAs (two per SM for 64 rows, one for 128: shared memory), with
// warp roles joined only by mbarriers, so that loads, B builds, MMAs and
// read-back of different sites overlap (3 site slots, four accumulator slots):
//   * warps 0-3 load, running ahead of the others: per site the 8
//     neighbours' A tiles as 16-byte cp.async pieces (a warp moves 512
//     contiguous bytes per step; one bulk-copy engine per SM issued them
//     ~8x slower) and the 8 links' 16-bit words, one cp.async group per
//     site, released one site later (wait, proxy fence, arrive);
//   * warps 4-7 decode the links (a thread per link element, row 2 rebuilt
//     where taken), write for every element its signed and swapped FP16
//     pairs, and assemble the B operand from those pairs (a 16-byte segment
//     of a B row per thread; all-zero segments are never written);
//   * one thread of warp 8 issues the site's 12 MMAs (kind::f16, M = 128,
//     N = 32, K = 16; FP32 accumulators in tensor memory) and commits them
//     to the slot (freeing it) and to the accumulator slot;
//   * warps 9-12 read the accumulators back (tcgen05.ld, one warp per 32
//     right-hand sides), round them to FP16 and store them.
// The 8 neighbour tiles of a site lie back to back with one K-chunk stride
// (chunk c of hop h at (3 h + c) LBO), so the site is a single GEMM with
// K = 192: 12 MMAs of K = 16, B stored as one 32 x 192 operand (rows 24-31
// zero).
// With RP = 64 the MMA's rows 64-127 read neighbouring data; those rows of
// D are never stored.  Sites are visited in z-slabs (every t of zb z-planes,
// then the next slab), so the 8 reads of an input tile fall within a window
// that L2 holds.  Every wait is bounded and ends early once any role has
// set the CTA's abort flag; a time-out sets the error flag, and the warps
// that issued copies or MMAs wait (bounded) for them before the CTA frees
// its tensor memory and exits.
#include <cuda_fp16.h>

#include <algorithm>

#include "internal.h"
#include "mrhs.h"
#include "solver.h"
#include "tc.cuh"

namespace qcu {

namespace {

// roles: warps 0-3 load (the A tiles and the link words, by cp.async),
// warps 4-7 build the B matrices, one thread of warp 8 issues the MMAs,
// warps 9-12 read the accumulators back (tensor-memory lane quarters 1, 2,
// 3, 0: warp w may access lanes 32 (w % 4) to 32 (w % 4) + 31)
constexpr int MT_WARPS = 13;
constexpr int MT_THREADS = MT_WARPS * 32;
constexpr int MT_LOADERS = 128;  // warps 0-3
constexpr int MT_BUILDERS = 128;  // warps 4-7
constexpr int MT_BUILD_WARP0 = 4;
constexpr int MT_MMA_WARP = 8;
constexpr int MT_HOPS = 8;
constexpr int MT_K = MT_HOPS * 24;       // K of a site's GEMM: 8 hops x 24 input components
constexpr int MT_B_BYTES = 32 * MT_K * 2; // B: 32 rows (24 used) x K 192, FP16
constexpr int MT_NVAR = MT_HOPS * 9 * 4;  // signed / swapped pairs of the link elements
constexpr int MT_ZERO_WORD = MT_NVAR;     // index of a zero pair
constexpr int MT_SEGS = MT_HOPS * 24 * 3;  // 16-byte B segments that can be non-zero
constexpr int MT_SEG_SLOTS = (MT_SEGS + MT_BUILDERS - 1) / MT_BUILDERS;
constexpr int MT_ND = 4;                  // accumulator slots (32 tensor-memory columns each)

template <int RP>
struct MtShape {
  static constexpr int A_HOP = 48 * RP;  // bytes of one neighbour tile
  static constexpr int A_BYTES = MT_HOPS * A_HOP;
  static constexpr int B_BYTES = MT_B_BYTES;
  // per site slot: [A tiles + pad][B matrices][link words 8 x 16 B][8 x 8 B][phases 8 x 4 B]
  static constexpr int OFF_L16 = A_BYTES + B_BYTES;
  static constexpr int OFF_L8 = OFF_L16 + MT_HOPS * 16;
  static constexpr int OFF_PH = OFF_L8 + MT_HOPS * 8;
  static constexpr int SLOT = (OFF_PH + MT_HOPS * 4 + 1023) / 1024 * 1024;
  static constexpr int NS = 3;  // site slots (shared memory: 3 x 37 KB or 3 x 61 KB)
  static constexpr int CTAS_PER_SM = RP == 64 ? 2 : 1;  // 64 rows: two pipelines per SM
  static constexpr int OFF_VAR = NS * SLOT;    // builders' scratch: the pairs of the 8 links' elements
  static constexpr int OFF_BAR = OFF_VAR + (MT_NVAR + 4) * 4;
  // mbarriers: full[NS] (A tiles + link words landed), bready[NS] (B built),
  // mdone[NS] (the site's MMAs done: slot free), dfull[ND], dempty[ND]
  static constexpr int NBAR = 3 * NS + 2 * MT_ND;
  static constexpr int SMEM = OFF_BAR + NBAR * 8 + 16;  // + tensor-memory address, abort flag
  static constexpr int EPI_WARPS = RP / 32;
};

struct MtArgs {
  Geom g;
  const void *gauge;  // GSOA16 links of both parities
  float t_bc;
  const __half *in;   // multi-rhs field of parity 1 - par
  __half *out;        // multi-rhs field of parity par
  int par;
  int zb;             // z-planes per slab of the visiting order
  int *err;
  // reciprocal multipliers (geom_div) of Ly * Lxh, zb, Lt and Lxh, or 0: plain division
  unsigned m_plane, m_zb, m_lt, m_lxh;
};

// coordinates of the q-th site of the visiting order: z-slabs of zb planes,
// then t, then the planes of the slab, then (y, xh)
struct MtSite {
  int s, xh, y, z, t;
};
__device__ __forceinline__ MtSite mt_site(const MtArgs &a, int q) {
  const Geom &g = a.g;
  const int plane = g.Ly * g.Lxh;
  const int r1 = geom_div(q, plane, a.m_plane);
  const int yx = q - r1 * plane;
  const int r2 = geom_div(r1, a.zb, a.m_zb);
  const int zz = r1 - r2 * a.zb;
  const int zs = geom_div(r2, g.Lt, a.m_lt);
  MtSite c;
  c.t = r2 - zs * g.Lt;
  c.z = zs * a.zb + zz;
  c.s = (c.t * g.Lz + c.z) * plane + yx;
  c.y = geom_div(yx, g.Lxh, a.m_lxh);
  c.xh = yx - c.y * g.Lxh;
  return c;
}
// neighbour of hop h (x+, x-, y+, y-, z+, z-, t+, t-) of output site c on parity par
__device__ __forceinline__ int mt_nbr(const Geom &g, const MtSite &c, int par, int h) {
  const int s = c.s, mu = h >> 1;
  const bool fwd = (h & 1) == 0;
  if (mu == 0) {  // even-odd x: the neighbour is s itself or s -+ 1 (wrapping within the row)
    const int xodd = (c.y + c.z + c.t + par) & 1;
    return fwd ? (xodd ? (c.xh == g.Lxh - 1 ? s - c.xh : s + 1) : s) : (xodd ? s : (c.xh == 0 ? s + g.Lxh - 1 : s - 1));
  }
  const int x = mu == 1 ? c.y : (mu == 2 ? c.z : c.t);
  const int L = mu == 1 ? g.Ly : (mu == 2 ? g.Lz : g.Lt);
  const int st = mu == 1 ? g.sy : (mu == 2 ? g.sz : g.st);
  return fwd ? (x == L - 1 ? s - (L - 1) * st : s + st) : (x == 0 ? s + (L - 1) * st : s - st);
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// mbarrier wait bounded in iterations and ended early by the CTA's abort flag
__device__ __forceinline__ bool mt_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag) {
  for (unsigned i = 0; i < TC_WAIT_LIMIT; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 63) == 63) {
      if (*abort_flag) return false;
      __nanosleep(32);
    }
  }
  return false;
}
// AND of a predicate over the 128 builder threads (named barrier 1)
__device__ __forceinline__ bool builders_and(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void builders_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__device__ __forceinline__ uint32_t half2_bits(float lo, float hi) {
  const __half2 v = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// word of the pair table for B row n = (spin s, colour c, re/im ri), input pair k2 = (spin s', colour c')
// of hop h (mu = h / 2, forward for even h): the real form of P[s][s'] V[c][c'],
// P = 1 + S gamma_mu.  Pairs of element e of hop h: 4 (9 h + e) + {F0, -F0, F1, -F1},
// F0 = (Re V, -Im V) (row re), F1 = (Im V, Re V) (row im).
__device__ __forceinline__ int mt_pair_word(int h, int n, int k2) {
  const int s = n / 6, c = (n >> 1) % 3, ri = n & 1;
  const int sp = k2 / 3, cp = k2 % 3;
  const int mu = h >> 1, S = (h & 1) ? 1 : -1;
  const int base = (h * 9 + c * 3 + cp) * 4;
  if (sp == s) return base + (ri ? 2 : 0);
  if (sp == gcol(mu, s)) {
    const int gr = S * gre(mu, s), gi = S * gim(mu, s);
    if (gr != 0) return base + (ri ? 2 : 0) + (gr < 0 ? 1 : 0);
    // P = i gi:  row re takes -gi F1, row im takes gi F0
    return ri ? base + (gi > 0 ? 0 : 1) : base + 2 + (gi > 0 ? 1 : 0);
  }
  return MT_ZERO_WORD;
}

template <int RP>
__global__ void __launch_bounds__(MT_THREADS, MtShape<RP>::CTAS_PER_SM) k_mrhs_tc(MtArgs a) {
  using S = MtShape<RP>;
  constexpr int NS = S::NS;
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Geom &g = a.g;
  const uint32_t s0 = smem_u32(smem);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::OFF_BAR);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + S::NBAR);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  auto bar_full = [&](int k) { return smem_u32(&bars[k]); };
  auto bar_bready = [&](int k) { return smem_u32(&bars[NS + k]); };
  auto bar_mdone = [&](int k) { return smem_u32(&bars[2 * NS + k]); };
  auto bar_dfull = [&](int d) { return smem_u32(&bars[3 * NS + d]); };
  auto bar_dempty = [&](int d) { return smem_u32(&bars[3 * NS + MT_ND + d]); };
  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(a.err, 1);
  };

  // zero the slots (pads, the zero columns and rows of B) and the scratch
  for (int i = tid * 16; i < S::OFF_BAR; i += MT_THREADS * 16)
    *reinterpret_cast<uint4 *>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    *abort_flag = 0;
    for (int k = 0; k < NS; k++) {
      // every loader thread arrives once its copies for the site have landed
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_full(k)), "r"(MT_LOADERS) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_bready(k)), "r"(MT_BUILDERS / 32) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_mdone(k)) : "memory");
    }
    for (int d = 0; d < MT_ND; d++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_dfull(d)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_dempty(d)), "r"(S::EPI_WARPS) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(32u * MT_ND)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the zeros, before any async write or read
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int nloc = blockIdx.x < g.Vh ? (g.Vh - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto q_of = [&](int i) { return (int)blockIdx.x + i * (int)gridDim.x; };

  if (warp < MT_BUILD_WARP0) {
    // ---------------------------------------------------------- loaders
    // a site's 8 tiles are 8 x 3 RP pieces of 16 B; loader thread lt copies
    // pieces lt, lt + 128, ...: a warp moves 512 contiguous bytes per step.
    // Each site's copies are one cp.async group, released LAG sites later:
    // wait for the group, fence (the tensor core reads what cp.async wrote),
    // arrive on the slot's full barrier.
    const int lt = tid;
    constexpr int PIECES = MT_HOPS * 3 * RP, PER_TILE = 3 * RP;
    // a site's group is released once the next site's copies are issued
    // (a lag of 2 sites with 5 slots measured slower at 64 rows)
    constexpr int LAG = 1;
    auto release = [&](int k) {
      asm volatile("cp.async.wait_group %0;" ::"n"(LAG) : "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(bar_full(k));
    };
    int i = 0;
    for (; i < nloc; i++) {
      const int k = i % NS, u = i / NS;
      // the slot's previous site (i - NS) has finished its MMAs
      if (u >= 1 && !__all_sync(0xffffffffu, mt_wait(bar_mdone(k), (u - 1) & 1, abort_flag))) {
        if (lane == 0) fail();
        break;
      }
      const MtSite c = mt_site(a, q_of(i));
      uint8_t *slot = smem + k * S::SLOT;
      const uint32_t sbase = s0 + k * S::SLOT;
      int nbr[MT_HOPS];
#pragma unroll
      for (int h = 0; h < MT_HOPS; h++) nbr[h] = mt_nbr(g, c, a.par, h);
#pragma unroll
      for (int j = 0; j < PIECES / MT_LOADERS; j++) {
        const int pc = lt + j * MT_LOADERS;
        const int h = pc / PER_TILE, off = (pc - h * PER_TILE) * 16;
        const char *src = reinterpret_cast<const char *>(a.in) + (size_t)nbr[h] * (48 * RP) + off;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sbase + h * S::A_HOP + off), "l"(src)
                     : "memory");
      }
      if (lt < MT_HOPS) {  // the link of hop h = lt: forward U_mu(x), backward U_mu(x - mu)
        const int h = lt, mu = h >> 1;
        const int lpar = (h & 1) ? 1 - a.par : a.par;
        const int ls = (h & 1) ? nbr[h] : c.s;
        const char *blk = static_cast<const char *>(a.gauge) + (size_t)(mu * 2 + lpar) * pad_sites(g.Vh) * 24 +
                          (size_t)(ls >> 5) * G16_BLOCK_BYTES;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(slot + S::OFF_L16 + 16 * h)),
                     "l"(blk + (ls & 31) * 16)
                     : "memory");
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(slot + S::OFF_L8 + 8 * h)),
                     "l"(blk + 512 + (ls & 31) * 8)
                     : "memory");
      }
      if (lt == 0) {
        float *ph = reinterpret_cast<float *>(slot + S::OFF_PH);
#pragma unroll
        for (int h = 0; h < MT_HOPS; h++) ph[h] = 1.f;
        if (c.t == g.Lt - 1) ph[6] = a.t_bc;
        if (c.t == 0) ph[7] = a.t_bc;
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
      if (i >= LAG) release((i - LAG) % NS);
    }
    // the last sites' copies (and, after an abort, whatever is in flight)
    // complete before the shared memory goes away
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (i == nloc)
      for (int j = nloc - LAG < 0 ? 0 : nloc - LAG; j < nloc; j++) mbar_arrive(bar_full(j % NS));
  } else if (warp < MT_MMA_WARP) {
    // ---------------------------------------------------------- B builders
    const int bt = tid - MT_BUILD_WARP0 * 32;
    uint32_t *sVar = reinterpret_cast<uint32_t *>(smem + S::OFF_VAR);
    int segw[MT_SEG_SLOTS][4];
    int segoff[MT_SEG_SLOTS];
    bool segon[MT_SEG_SLOTS];
#pragma unroll
    for (int m = 0; m < MT_SEG_SLOTS; m++) {
      const int sg = bt + m * MT_BUILDERS;
      segon[m] = false;
      segoff[m] = 0;
#pragma unroll
      for (int p = 0; p < 4; p++) segw[m][p] = MT_ZERO_WORD;
      if (sg < MT_SEGS) {
        const int h = sg / 72, n = (sg % 72) / 3, j = sg % 3;
#pragma unroll
        for (int p = 0; p < 4; p++) {
          segw[m][p] = mt_pair_word(h, n, 4 * j + p);
          segon[m] = segon[m] || segw[m][p] != MT_ZERO_WORD;
        }
        segoff[m] = S::A_BYTES + (int)kmajor_off(n, 24 * h + 8 * j, MT_K);
      }
    }
    for (int i = 0; i < nloc; i++) {
      const int k = i % NS, u = i / NS;
      bool ok = true;
      if (bt < MT_HOPS) ok = mt_wait(bar_full(k), u & 1, abort_flag);
      ok = builders_and(ok);
      if (!ok) {
        if (bt == 0) fail();
        break;
      }
      const uint8_t *slot = smem + k * S::SLOT;
      if (bt < MT_HOPS * 9) {  // element (r, cc) of V = phase x (U or U^dag) of hop h, as four FP16 pairs
        const int h = bt / 9, e = bt - 9 * h, r = e / 3, cc = e - 3 * r;
        const bool fwd = (h & 1) == 0;
        const int ur = fwd ? r : cc, uc = fwd ? cc : r;  // the element of U it takes
        auto word = [&](int w) {
          return w < 4 ? reinterpret_cast<const uint32_t *>(slot + S::OFF_L16 + 16 * h)[w]
                       : reinterpret_cast<const uint32_t *>(slot + S::OFF_L8 + 8 * h)[w - 4];
        };
        auto elem = [&](int w) {
          const float2 d = fix16_unpack(word(w));
          return Cpx<float>(d.x * (1.0f / FIX16_SCALE), d.y * (1.0f / FIX16_SCALE));
        };
        Cpx<float> v;
        if (ur < 2) {
          v = elem(ur * 3 + uc);
        } else {  // row 2 = conj(row0 x row1)
          const int b1 = uc == 2 ? 0 : uc + 1, b2 = uc == 0 ? 2 : uc - 1;
          v = (elem(b1) * elem(3 + b2) - elem(b2) * elem(3 + b1)).conj();
        }
        if (!fwd) v = v.conj();
        const float ph = reinterpret_cast<const float *>(slot + S::OFF_PH)[h];
        const uint32_t f0 = half2_bits(v.re * ph, -v.im * ph), f1 = half2_bits(v.im * ph, v.re * ph);
        *reinterpret_cast<uint4 *>(sVar + bt * 4) = make_uint4(f0, f0 ^ 0x80008000u, f1, f1 ^ 0x80008000u);
      }
      builders_sync();
      uint8_t *wslot = smem + k * S::SLOT;
#pragma unroll
      for (int m = 0; m < MT_SEG_SLOTS; m++)
        if (segon[m])
          *reinterpret_cast<uint4 *>(wslot + segoff[m]) =
              make_uint4(sVar[segw[m][0]], sVar[segw[m][1]], sVar[segw[m][2]], sVar[segw[m][3]]);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // B visible to the tensor core
      __syncwarp();
      if (lane == 0) mbar_arrive(bar_bready(k));  // one arrival per builder warp
    }
  } else if (warp == MT_MMA_WARP) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_f16<128, 32>(false);
      int last_bar = -1, last_par = 0;
      for (int i = 0; i < nloc; i++) {
        const int k = i % NS, u = i / NS, d = i % MT_ND, ud = i / MT_ND;
        if (!mt_wait(bar_bready(k), u & 1, abort_flag) || !mt_wait(bar_full(k), u & 1, abort_flag) ||
            (ud >= 1 && !mt_wait(bar_dempty(d), (ud - 1) & 1, abort_flag))) {
          fail();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = s0 + k * S::SLOT;
        // the 8 tiles are one run of 24 K-chunks (chunk c of hop h at (3 h + c) LBO): K = 192 in 12 steps
#pragma unroll
        for (int ks = 0; ks < MT_K / 16; ks++) {
          const uint64_t ad = umma_desc(base + ks * 2 * (16 * RP), 16 * RP, 128);
          const uint64_t bd = umma_desc(base + S::A_BYTES + ks * 256, 128, MT_K / 8 * 128);
          umma_f16(tmem + d * 32, ad, bd, idesc, ks > 0 ? 1u : 0u);
        }
        umma_commit(bar_mdone(k));
        umma_commit(bar_dfull(d));
        last_bar = k;
        last_par = u & 1;
      }
      // every MMA issued is complete before the tensor memory is freed
      if (last_bar >= 0 && !mbar_wait(bar_mdone(last_bar), last_par)) atomicExch(a.err, 1);
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int qd = warp & 3;  // tensor-memory lane quarter of this warp
    if (qd * 32 < RP) {
      for (int i = 0; i < nloc; i++) {
        const int d = i % MT_ND, ud = i / MT_ND;
        const bool ok = __all_sync(0xffffffffu, mt_wait(bar_dfull(d), ud & 1, abort_flag));
        if (!ok) {
          if (lane == 0) fail();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float d0[16], d1[16];
        const uint32_t taddr = tmem + ((uint32_t)(qd * 32) << 16) + d * 32;
        tmem_ld16(taddr, d0);
        tmem_ld16(taddr + 16, d1);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_dempty(d));  // the accumulators are read: the slot is free
        const int s = mt_site(a, q_of(i)).s;
        const int row = qd * 32 + lane;
        uint4 *o = reinterpret_cast<uint4 *>(a.out + (size_t)s * (24 * RP) + row * 8);
        o[0] = make_uint4(half2_bits(d0[0], d0[1]), half2_bits(d0[2], d0[3]), half2_bits(d0[4], d0[5]),
                          half2_bits(d0[6], d0[7]));
        o[RP] = make_uint4(half2_bits(d0[8], d0[9]), half2_bits(d0[10], d0[11]), half2_bits(d0[12], d0[13]),
                           half2_bits(d0[14], d0[15]));
        o[2 * RP] = make_uint4(half2_bits(d1[0], d1[1]), half2_bits(d1[2], d1[3]), half2_bits(d1[4], d1[5]),
                               half2_bits(d1[6], d1[7]));
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u * MT_ND) : "memory");
  }
}

// PyQuda half spinors [nrhs][Vh][12] complex128 <-> multi-rhs FP16 field;
// one thread per (site, K-chunk, row); padding rows are written as zeros
__global__ void k_mrhs_pack(const double2 *in, __half *out, int Vh, int nrhs, int RP) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Vh * 3 * RP) return;
  const int r = (int)(idx % RP);
  const int j = (int)((idx / RP) % 3);
  const int s = (int)(idx / (3LL * RP));
  uint32_t w[4] = {0u, 0u, 0u, 0u};
  if (r < nrhs) {
    const double2 *p = in + ((size_t)r * Vh + s) * 12 + 4 * j;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double2 z = p[q];
      w[q] = half2_bits((float)z.x, (float)z.y);
    }
  }
  *reinterpret_cast<uint4 *>(out + (size_t)s * 24 * RP + (size_t)j * 8 * RP + r * 8) = make_uint4(w[0], w[1], w[2], w[3]);
}

__global__ void k_mrhs_unpack(const __half *in, double2 *out, int Vh, int nrhs, int RP) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Vh * 3 * nrhs) return;
  const int r = (int)(idx % nrhs);
  const int j = (int)((idx / nrhs) % 3);
  const int s = (int)(idx / (3LL * nrhs));
  const uint4 v = *reinterpret_cast<const uint4 *>(in + (size_t)s * 24 * RP + (size_t)j * 8 * RP + r * 8);
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
  double2 *p = out + ((size_t)r * Vh + s) * 12 + 4 * j;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const __half2 h = *reinterpret_cast<const __half2 *>(&w[q]);
    const float2 f = __half22float2(h);
    p[q] = make_double2((double)f.x, (double)f.y);
  }
}

// seeded values in [-1, 1) on the right-hand-side rows, zero on the padding rows
__global__ void k_mrhs_random(__half *out, int Vh, int nrhs, int RP, unsigned long long seed) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Vh * 3 * RP) return;
  const int r = (int)(idx % RP);
  uint32_t w[4] = {0u, 0u, 0u, 0u};
  if (r < nrhs) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      unsigned long long x = (seed + (unsigned long long)idx * 4 + q + 1) * 0x9E3779B97F4A7C15ULL;
      x ^= x >> 31;
      x *= 0xBF58476D1CE4E5B9ULL;
      x ^= x >> 29;
      const float lo = (float)(x & 0xFFFF) / 32768.0f - 1.0f, hi = (float)((x >> 16) & 0xFFFF) / 32768.0f - 1.0f;
      w[q] = half2_bits(lo, hi);
    }
  }
  const int j = (int)((idx / RP) % 3);
  const int s = (int)(idx / (3LL * RP));
  *reinterpret_cast<uint4 *>(out + (size_t)s * 24 * RP + (size_t)j * 8 * RP + r * 8) = make_uint4(w[0], w[1], w[2], w[3]);
}

template <int RP>
void launch_mt(const MtArgs &a, int sms, cudaStream_t s) {
  using S = MtShape<RP>;
  auto k = k_mrhs_tc<RP>;
  QCU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM));
  QCU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  const int grid = std::min(a.g.Vh, sms * S::CTAS_PER_SM);  // as many CTAs as shared memory holds
  k<<<grid, MT_THREADS, S::SMEM, s>>>(a);
  QCU_CHECK_LAUNCH();
}

}  // namespace

int mrhs_rows(int nrhs) { return nrhs <= 64 ? 64 : 128; }
size_t mrhs_bytes(int Vh, int nrhs) { return (size_t)Vh * 48 * mrhs_rows(nrhs); }

void launch_mrhs_tc(const Geom &g, const void *gauge16, double t_bc, const void *in, void *out, int nrhs, int par,
                    int *err, int sms, cudaStream_t s) {
  require(nrhs >= 1 && nrhs <= 128, "multi-rhs tensor-core dslash: 1 to 128 right-hand sides");
  MtArgs a;
  a.g = g;
  a.gauge = gauge16;
  a.t_bc = (float)t_bc;
  a.in = static_cast<const __half *>(in);
  a.out = static_cast<__half *>(out);
  a.par = par;
  a.zb = g.Lz % 8 == 0 ? 8 : (g.Lz % 4 == 0 ? 4 : (g.Lz % 2 == 0 ? 2 : 1));
  auto magic = [&](int d) -> unsigned {  // exact for every q < Vh while (Vh + 64) d < 2^32 (geom_div)
    if (d < 2 || (uint64_t)(g.Vh + 64) * (uint64_t)d >= (1ULL << 32)) return 0u;
    return (unsigned)(((1ULL << 32) + (uint64_t)d - 1) / (uint64_t)d);
  };
  a.m_plane = magic(g.Ly * g.Lxh);
  a.m_zb = magic(a.zb);
  a.m_lt = magic(g.Lt);
  a.m_lxh = magic(g.Lxh);
  a.err = err;
  if (mrhs_rows(nrhs) == 64) launch_mt<64>(a, sms, s);
  else launch_mt<128>(a, sms, s);
}

void launch_mrhs_pack(const void *pyq, void *mrhs, int Vh, int nrhs, cudaStream_t s) {
  const int RP = mrhs_rows(nrhs);
  const long long n = (long long)Vh * 3 * RP;
  k_mrhs_pack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(static_cast<const double2 *>(pyq), static_cast<__half *>(mrhs),
                                                         Vh, nrhs, RP);
  QCU_CHECK_LAUNCH();
}
void launch_mrhs_unpack(const void *mrhs, void *pyq, int Vh, int nrhs, cudaStream_t s) {
  const int RP = mrhs_rows(nrhs);
  const long long n = (long long)Vh * 3 * nrhs;
  k_mrhs_unpack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(static_cast<const __half *>(mrhs), static_cast<double2 *>(pyq),
                                                           Vh, nrhs, RP);
  QCU_CHECK_LAUNCH();
}
void launch_mrhs_random(void *mrhs, int Vh, int nrhs, unsigned long long seed, cudaStream_t s) {
  const int RP = mrhs_rows(nrhs);
  const long long n = (long long)Vh * 3 * RP;
  k_mrhs_random<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(static_cast<__half *>(mrhs), Vh, nrhs, RP, seed);
  QCU_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- operators on a handle
namespace {
struct MrhsSpace {
  DevBuf in, out, err;
};
// the kernel's error flag: set on a timed-out wait
void mrhs_check_err(MrhsSpace &w, cudaStream_t st) {
  int bad = 0;
  QCU_CUDA(cudaMemcpyAsync(&bad, w.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  QCU_CUDA(cudaStreamSynchronize(st));
  if (bad) throw Error(2, "multi-rhs tensor-core dslash: a wait in the kernel timed out");
}
}  // namespace

void handle_dslash_mrhs(GaugeHandle &G, void *out, const void *in, int nrhs, int par) {
  require(out && in, "dslash: null spinor pointer");
  require(par == 0 || par == 1, "parity must be 0 or 1");
  require(nrhs >= 1 && nrhs <= 128, "multi-rhs tensor-core dslash: 1 to 128 right-hand sides");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  MrhsSpace &w = per_device<MrhsSpace>(ctx);
  const int Vh = G.g.Vh;
  w.in.ensure(mrhs_bytes(Vh, nrhs));
  w.out.ensure(mrhs_bytes(Vh, nrhs));
  w.err.ensure(sizeof(int));
  QCU_CUDA(cudaDeviceSynchronize());
  QCU_CUDA(cudaMemsetAsync(w.err.p, 0, sizeof(int), ctx.stream));
  launch_mrhs_pack(in, w.in.p, Vh, nrhs, ctx.stream);
  launch_mrhs_tc(G.g, G.g16.p, G.t_bc, w.in.p, w.out.p, nrhs, par, w.err.as<int>(), ctx.sms, ctx.stream);
  launch_mrhs_unpack(w.out.p, out, Vh, nrhs, ctx.stream);
  mrhs_check_err(w, ctx.stream);
}

double handle_dslash_mrhs_time(GaugeHandle &G, int nrhs, int par, int iters) {
  require(par == 0 || par == 1, "parity must be 0 or 1");
  require(nrhs >= 1 && nrhs <= 128, "multi-rhs tensor-core dslash: 1 to 128 right-hand sides");
  require(iters >= 1, "iters must be positive");
  Context &ctx = context();
  std::lock_guard<std::mutex> lk(ctx.mu);
  MrhsSpace &w = per_device<MrhsSpace>(ctx);
  const int Vh = G.g.Vh;
  w.in.ensure(mrhs_bytes(Vh, nrhs));
  w.out.ensure(mrhs_bytes(Vh, nrhs));
  w.err.ensure(sizeof(int));
  QCU_CUDA(cudaDeviceSynchronize());
  QCU_CUDA(cudaMemsetAsync(w.err.p, 0, sizeof(int), ctx.stream));
  launch_mrhs_random(w.in.p, Vh, nrhs, 20251204ULL, ctx.stream);
  auto run = [&]() {
    launch_mrhs_tc(G.g, G.g16.p, G.t_bc, w.in.p, w.out.p, nrhs, par, w.err.as<int>(), ctx.sms, ctx.stream);
  };
  for (int i = 0; i < 3; i++) run();
  cudaEvent_t e0, e1;
  QCU_CUDA(cudaEventCreate(&e0));
  QCU_CUDA(cudaEventCreate(&e1));
  QCU_CUDA(cudaEventRecord(e0, ctx.stream));
  for (int i = 0; i < iters; i++) run();
  QCU_CUDA(cudaEventRecord(e1, ctx.stream));
  QCU_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  QCU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  mrhs_check_err(w, ctx.stream);
  return (double)ms / iters;
}

}  // namespace qcu
