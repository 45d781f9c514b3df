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
// A CTA of 128 threads is persistent over sites, two in flight:
//   * thread 0 issues, one site ahead, the 8 bulk copies (cp.async.bulk, no
//     multicast) of the neighbours' A tiles, completing on the slot's mbarrier;
//   * eight threads decode the 8 links (16-bit reconstruct-12), 72 threads
//     write for every link element its signed and swapped FP16 pairs, and all
//     threads assemble the 8 B matrices from those pairs (a 16-byte segment
//     of a B row each; all-zero segments are never written);
//   * thread 0 issues the site's 16 MMAs (kind::f16, M = 128, N = 32,
//     K = 16; FP32 accumulators in tensor memory) and commits them;
//   * the previous site's accumulators are read back (tcgen05.ld, one warp
//     per 32 right-hand sides), rounded to FP16 and stored.
// K runs to 32 per hop (24 used): B's columns 24-31 are zero, so the fourth
// K-chunk of A (the next tile, or a zeroed pad after the last) adds nothing.
// With RP = 64 the MMA's rows 64-127 read neighbouring data; those rows of
// D are never stored.  Sites are visited in z-slabs (every t of zb z-planes,
// then the next slab), so the 8 reads of an input tile fall within a window
// that L2 holds.  Every wait is bounded: a time-out sets the error flag,
// stops the CTA and still frees its tensor memory.
#include <cuda_fp16.h>

#include <algorithm>

#include "internal.h"
#include "mrhs.h"
#include "solver.h"
#include "tc.cuh"

namespace qcu {

namespace {

constexpr int MT_THREADS = 128;
constexpr int MT_HOPS = 8;
constexpr int MT_B_HOP = 32 * 32 * 2;  // one B matrix: 32 rows x K 32, FP16
constexpr int MT_A_PAD = 2048;         // zeros read as the last hop's fourth K-chunk
constexpr int MT_NVAR = MT_HOPS * 9 * 4;  // signed / swapped pairs of the link elements
constexpr int MT_ZERO_WORD = MT_NVAR;     // index of a zero pair
constexpr int MT_SEGS = MT_HOPS * 24 * 3;  // 16-byte B segments that can be non-zero
constexpr int MT_SEG_SLOTS = (MT_SEGS + MT_THREADS - 1) / MT_THREADS;

template <int RP>
struct MtShape {
  static constexpr int A_HOP = 48 * RP;  // bytes of one neighbour tile
  static constexpr int A_BYTES = MT_HOPS * A_HOP + MT_A_PAD;
  static constexpr int B_BYTES = MT_HOPS * MT_B_HOP;
  static constexpr int SLOT = (A_BYTES + B_BYTES + 1023) / 1024 * 1024;
  // shared: [slot 0 | slot 1] [V 8x9 float2] [pairs 8x9x4 + 4 words] [info x2] [2 + 2 mbarriers, tmem slot]
  static constexpr int OFF_V = 2 * SLOT;
  static constexpr int OFF_VAR = OFF_V + MT_HOPS * 9 * 8;
  static constexpr int OFF_INFO = OFF_VAR + (MT_NVAR + 4) * 4;
  static constexpr int OFF_BAR = OFF_INFO + 2 * 128;
  static constexpr int SMEM = OFF_BAR + 64;
  static constexpr int CTAS_PER_SM = RP == 64 ? 2 : 1;
};

// per site: the output site, the neighbour of each hop, the site and phase of each hop's link
struct MtInfo {
  int s;
  int nbr[MT_HOPS];
  int lsite[MT_HOPS];
  float ph[MT_HOPS];
};
static_assert(sizeof(MtInfo) <= 128, "site info");

struct MtArgs {
  Geom g;
  const void *gauge;  // GSOA16 links of both parities
  float t_bc;
  const __half *in;   // multi-rhs field of parity 1 - par
  __half *out;        // multi-rhs field of parity par
  int par;
  int zb;             // z-planes per slab of the visiting order
  int *err;
};

// q-th site of the visiting order: z-slabs of zb planes, t, then the planes of the slab, then (y, xh)
__device__ __forceinline__ void mt_site_info(const MtArgs &a, int q, MtInfo &f) {
  const Geom &g = a.g;
  const int plane = g.Ly * g.Lxh;
  const int yx = q % plane;
  int r = q / plane;
  const int zz = r % a.zb;
  r /= a.zb;
  const int t = r % g.Lt;
  const int z = (r / g.Lt) * a.zb + zz;
  const int s = (t * g.Lz + z) * plane + yx;
  const int xh = yx % g.Lxh, y = yx / g.Lxh;
  const int xodd = (y + z + t + a.par) & 1;
  f.s = s;
  f.nbr[0] = xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s;
  f.nbr[1] = xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1);
  f.nbr[2] = (y == g.Ly - 1) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  f.nbr[3] = (y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  f.nbr[4] = (z == g.Lz - 1) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  f.nbr[5] = (z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  f.nbr[6] = (t == g.Lt - 1) ? s - (g.Lt - 1) * g.st : s + g.st;
  f.nbr[7] = (t == 0) ? s + (g.Lt - 1) * g.st : s - g.st;
#pragma unroll
  for (int h = 0; h < MT_HOPS; h++) {
    f.lsite[h] = (h & 1) ? f.nbr[h] : s;  // forward: U_mu(x); backward: U_mu(x - mu)
    f.ph[h] = 1.f;
  }
  if (t == g.Lt - 1) f.ph[6] = a.t_bc;
  if (t == 0) f.ph[7] = a.t_bc;
}

__device__ __forceinline__ void bulk_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

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
__global__ void __launch_bounds__(MT_THREADS) k_mrhs_tc(MtArgs a) {
  using S = MtShape<RP>;
  extern __shared__ __align__(1024) uint8_t smem[];
  float2 *sV = reinterpret_cast<float2 *>(smem + S::OFF_V);
  uint32_t *sVar = reinterpret_cast<uint32_t *>(smem + S::OFF_VAR);
  MtInfo *sInfo = reinterpret_cast<MtInfo *>(smem + S::OFF_INFO);  // stride 128 B
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::OFF_BAR);  // [0,1] A full, [2,3] MMAs done
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Geom &g = a.g;
  const uint32_t s0 = smem_u32(smem);
  auto info = [&](int slot) -> MtInfo & { return *reinterpret_cast<MtInfo *>(smem + S::OFF_INFO + slot * 128); };
  (void)sInfo;

  // zero everything the MMAs may read before it is written (pads, zero columns of B)
  for (int i = tid * 16; i < S::OFF_BAR; i += MT_THREADS * 16)
    *reinterpret_cast<uint4 *>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  // this thread's B segments: table words of their four pairs and their offsets
  int segw[MT_SEG_SLOTS][4];
  int segoff[MT_SEG_SLOTS];
  bool segon[MT_SEG_SLOTS];
#pragma unroll
  for (int m = 0; m < MT_SEG_SLOTS; m++) {
    const int sg = tid + m * MT_THREADS;
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
      segoff[m] = h * MT_B_HOP + (int)kmajor_off(n, 8 * j, 32);
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(64u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int k = 0; k < 4; k++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[k])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // zeros visible to the async proxy
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc_f16<128, 32>(false);
  const GaugeView<GSOA16> U{a.gauge, pad_sites(g.Vh)};
  const int nloc = blockIdx.x < g.Vh ? (g.Vh - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto a_addr = [&](int slot, int h) { return s0 + slot * S::SLOT + h * S::A_HOP; };
  auto b_addr = [&](int slot, int h) { return s0 + slot * S::SLOT + S::A_BYTES + h * MT_B_HOP; };
  // thread 0's count of what it issued and what it has seen complete, per
  // slot: bulk-copy batches (A full) and MMA batches; the drain on an error
  // waits for the difference
  int a_iss[2] = {0, 0}, a_done[2] = {0, 0}, m_iss[2] = {0, 0}, m_done[2] = {0, 0};
  // thread 0: site info of the i-th site and the bulk copies of its 8 A tiles
  auto issue_site = [&](int i) {
    const int slot = i & 1;
    a_iss[slot]++;
    MtInfo &f = info(slot);
    mt_site_info(a, (int)blockIdx.x + i * (int)gridDim.x, f);
    const uint32_t bar = smem_u32(&bars[slot]);
    bulk_expect(bar, MT_HOPS * S::A_HOP);
#pragma unroll
    for (int h = 0; h < MT_HOPS; h++)
      bulk_load(a_addr(slot, h), a.in + (size_t)f.nbr[h] * (24 * RP), S::A_HOP, bar);
  };
  if (tid == 0 && nloc > 0) issue_site(0);
  __syncthreads();

  bool ok = true;
  int s_prev = 0;
  for (int i = 0; i < nloc && ok; i++) {
    const int slot = i & 1;
    // (1) the previous site's MMAs are done: its buffers are free and its accumulators ready
    if (i >= 1) {
      ok = mbar_wait(smem_u32(&bars[2 + (slot ^ 1)]), ((i - 1) >> 1) & 1);
      if (ok) m_done[slot ^ 1]++;
    }
    // (2) one site ahead: info and A tiles of site i + 1 into the other slot
    if (tid == 0 && ok && i + 1 < nloc) issue_site(i + 1);
    // (3) B matrices of site i: links -> V, V -> signed / swapped pairs, pairs -> B segments
    const MtInfo &f = info(slot);
    const int s_cur = f.s;
    if (tid < MT_HOPS) {
      const int h = tid, mu = h >> 1;
      const bool fwd = (h & 1) == 0;
      const int lpar = fwd ? a.par : 1 - a.par;
      unsigned w[6];
      g16_load_words(U.p, (size_t)(mu * 2 + lpar) * U.stride, f.lsite[h], w);
      Cpx<float> m[9];
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const float2 d = fix16_unpack(w[k]);
        m[k] = Cpx<float>(d.x * (1.0f / FIX16_SCALE), d.y * (1.0f / FIX16_SCALE));
      }
      m[6] = (m[1] * m[5] - m[2] * m[4]).conj();
      m[7] = (m[2] * m[3] - m[0] * m[5]).conj();
      m[8] = (m[0] * m[4] - m[1] * m[3]).conj();
      const float ph = f.ph[h];
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const Cpx<float> v = fwd ? m[r * 3 + c] : m[c * 3 + r].conj();
          sV[h * 9 + r * 3 + c] = make_float2(v.re * ph, v.im * ph);
        }
    }
    __syncthreads();
    if (tid < MT_HOPS * 9) {
      const float2 v = sV[tid];
      const uint32_t f0 = half2_bits(v.x, -v.y), f1 = half2_bits(v.y, v.x);
      *reinterpret_cast<uint4 *>(sVar + tid * 4) = make_uint4(f0, f0 ^ 0x80008000u, f1, f1 ^ 0x80008000u);
    }
    __syncthreads();
    const uint32_t bslot = (uint32_t)(slot * S::SLOT + S::A_BYTES);
#pragma unroll
    for (int m = 0; m < MT_SEG_SLOTS; m++)
      if (segon[m])
        *reinterpret_cast<uint4 *>(smem + bslot + segoff[m]) =
            make_uint4(sVar[segw[m][0]], sVar[segw[m][1]], sVar[segw[m][2]], sVar[segw[m][3]]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // B visible to the tensor core
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) break;
    // (4) the site's 16 MMAs, once its A tiles have landed
    if (tid == 0) {
      const bool landed = mbar_wait(smem_u32(&bars[slot]), (i >> 1) & 1);
      if (landed) {
        a_done[slot]++;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int h = 0; h < MT_HOPS; h++)
#pragma unroll
          for (int ks = 0; ks < 2; ks++) {
            const uint64_t ad = umma_desc(a_addr(slot, h) + ks * 2 * (16 * RP), 16 * RP, 128);
            const uint64_t bd = umma_desc(b_addr(slot, h) + ks * 256, 128, 512);
            umma_f16(tmem + slot * 32, ad, bd, idesc, (h > 0 || ks > 0) ? 1u : 0u);
          }
        umma_commit(smem_u32(&bars[2 + slot]));
        m_iss[slot]++;
      }
      ok = landed;
    }
    // (5) epilogue of the previous site
    if (i >= 1 && warp * 32 < RP) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float d0[16], d1[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (slot ^ 1) * 32;
      tmem_ld16(taddr, d0);
      tmem_ld16(taddr + 16, d1);
      const int row = warp * 32 + lane;
      uint4 *o = reinterpret_cast<uint4 *>(a.out + (size_t)s_prev * (24 * RP) + row * 8);
      o[0] = make_uint4(half2_bits(d0[0], d0[1]), half2_bits(d0[2], d0[3]), half2_bits(d0[4], d0[5]),
                        half2_bits(d0[6], d0[7]));
      o[RP] = make_uint4(half2_bits(d0[8], d0[9]), half2_bits(d0[10], d0[11]), half2_bits(d0[12], d0[13]),
                         half2_bits(d0[14], d0[15]));
      o[2 * RP] = make_uint4(half2_bits(d1[0], d1[1]), half2_bits(d1[2], d1[3]), half2_bits(d1[4], d1[5]),
                             half2_bits(d1[6], d1[7]));
    }
    s_prev = s_cur;
    // the accumulators just read are overwritten by the MMAs of site i + 1 only after this barrier
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // the last site's epilogue
  if (ok && nloc > 0) {
    const int slot = (nloc - 1) & 1;
    ok = mbar_wait(smem_u32(&bars[2 + slot]), ((nloc - 1) >> 1) & 1);
    if (ok) m_done[slot]++;
    // tcgen05.ld is warp-collective: a warp reads only if all its threads saw the MMAs complete
    if (__all_sync(0xffffffffu, ok) && warp * 32 < RP) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float d0[16], d1[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + slot * 32;
      tmem_ld16(taddr, d0);
      tmem_ld16(taddr + 16, d1);
      const int row = warp * 32 + lane;
      uint4 *o = reinterpret_cast<uint4 *>(a.out + (size_t)s_prev * (24 * RP) + row * 8);
      o[0] = make_uint4(half2_bits(d0[0], d0[1]), half2_bits(d0[2], d0[3]), half2_bits(d0[4], d0[5]),
                        half2_bits(d0[6], d0[7]));
      o[RP] = make_uint4(half2_bits(d0[8], d0[9]), half2_bits(d0[10], d0[11]), half2_bits(d0[12], d0[13]),
                         half2_bits(d0[14], d0[15]));
      o[2 * RP] = make_uint4(half2_bits(d1[0], d1[1]), half2_bits(d1[2], d1[3]), half2_bits(d1[4], d1[5]),
                             half2_bits(d1[6], d1[7]));
    }
  }
  if (!ok) atomicExch(a.err, 1);
  // drain: every MMA batch thread 0 issued must be done before the tensor
  // memory is freed, and every bulk copy before the shared memory goes away
  // (bounded waits, completions in order)
  if (tid == 0) {
    for (int k = 0; k < 2; k++) {
      while (a_done[k] < a_iss[k]) {
        if (!mbar_wait(smem_u32(&bars[k]), a_done[k] & 1)) atomicExch(a.err, 1);
        a_done[k]++;
      }
      while (m_done[k] < m_iss[k]) {
        if (!mbar_wait(smem_u32(&bars[2 + k]), m_done[k] & 1)) atomicExch(a.err, 1);
        m_done[k]++;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64u) : "memory");
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
  const int grid = std::min(a.g.Vh, sms * S::CTAS_PER_SM);
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
