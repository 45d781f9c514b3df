// Inference layer of the learned preconditioner on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory).
//
// One parallel-transport layer (nn.h) is, per site x and colour c,
//     out_a(x, c) = sum_{h, b} W[h][a][b] (T_h in_b)(x, c)
// a shared-weight complex GEMM: rows = (site, colour), K = (hop, input
// channel), N = output channel.  In real form, with the row's transported
// inputs laid out as [Re v | Im v] per hop,
//     [Re out | Im out] = [Re v | Im v] x [[Re W^T, Im W^T], [-Im W^T, Re W^T]]
// so one BF16 MMA (FP32 accumulate) computes it.
//
// Fields are site-blocked like the solver's (32 sites per block, one
// component of 32 sites contiguous), so every warp access is coalesced:
// layer 1 reads the residual straight from the solver's FP64 layout (SOA64,
// odd sites) and writes the 16-channel hidden field as bf16 pairs
// ([parity][block][48 components][32 sites] of (re, im) bf16); layer 2 reads
// that and writes N(r) straight into the solver's FP64 layout.
//
// A CTA of 128 threads owns a tile of 128 output sites; each thread is one
// site, i.e. one row of three M = 128 GEMMs (one per colour, sharing B):
//   * the FMA pipes compute the parallel transports T_h in (FP32, from the
//     16-bit reconstruct-12 links), a chunk of hops at a time (K = 16 or 32
//     per chunk), round them to BF16 and store them as the A operand in
//     shared memory, K-major in 8 x 16-byte core matrices (no swizzle);
//   * one thread issues tcgen05.mma for the three colours, accumulating
//     D = A x B in tensor memory (three column blocks of N FP32 each) while
//     the others transport the next chunk into the second A buffer; a
//     tcgen05.commit per chunk arrives on that buffer's mbarrier, which
//     gates its reuse;
//   * after the last chunk every warp reads its 32 rows of D back with
//     tcgen05.ld (warp w owns tensor-memory lanes 32w..32w+31) and stores
//     the complex outputs.
// B (the weights, N x K) is staged once per CTA; the CTA is persistent over
// tiles.  Every wait on an mbarrier is bounded: on time-out the kernel sets
// an error flag, stops issuing work, and still frees its tensor memory.
#include <cuda_bf16.h>

#include <algorithm>

#include "nn.h"
#include "tc.cuh"

namespace qcu {

namespace {

template <int CIN, int COUT>
struct TcShape {
  static constexpr int HOPS_PER_CHUNK = CIN == 4 ? 2 : 1;
  static constexpr int KC = 2 * CIN * HOPS_PER_CHUNK;  // real K per chunk: 16 or 32
  static constexpr int KSTEPS = KC / 16;               // MMAs (K = 16 each) per chunk and colour
  static constexpr int NCHUNK = (NN_HOPS + HOPS_PER_CHUNK - 1) / HOPS_PER_CHUNK;
  static constexpr int KPAD = KC * NCHUNK;             // 80 or 288
  static constexpr int N = 2 * COUT < 16 ? 16 : 2 * COUT;  // 32 or 16 (padded)
  static constexpr int TMEM_COLS = 3 * N <= 64 ? 64 : 128;
  // B rows stored: with N padded from 8 to 16 only the 8 real rows are kept,
  // and the descriptor's row-group stride of 0 makes the MMA read them twice
  // (the duplicate output columns are never read)
  static constexpr int B_ROWS = 2 * COUT < 16 ? 8 : N;
  static constexpr int B_SBO = B_ROWS == N ? KPAD / 8 * 128 : 0;
  static constexpr int B_BYTES = B_ROWS * KPAD * 2;
  static constexpr int A_COLOUR_BYTES = 128 * KC * 2;
  static constexpr int A_BYTES = 3 * A_COLOUR_BYTES;   // one buffer: three colours
  static constexpr int SMEM = B_BYTES + 2 * A_BYTES + 64;
};

constexpr int TC_THREADS = 128;

// instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D, M = 128
template <int N>
__device__ __forceinline__ uint32_t umma_idesc() {
  return umma_idesc_f16<128, N>(true);
}

// layouts of the layer inputs and outputs
enum TcIo { TC_SOA64 = 0, TC_HID16 = 1 };
constexpr int HID_COMP = NN_C_HID * 3;  // 48 complex components per site of the hidden field

__device__ __forceinline__ size_t hid_index(int Vp, int par, int s, int comp) {
  return (size_t)par * Vp * HID_COMP + ((size_t)(s >> 5) * HID_COMP + comp) * 32 + (s & 31);
}

struct TcArgs {
  Geom g;
  const void *gauge;  // GSOA16 links
  float t_bc;
  const void *in;     // TC_SOA64: odd-parity FP64 spinor; TC_HID16: hidden field (both parities)
  void *out;          // TC_HID16: hidden field (both parities); TC_SOA64: odd-parity FP64 spinor
  const uint32_t *w16;  // [9][COUT][CIN] (re, im) bf16 pairs
  int *err;
};

// coordinates of this thread's output site, computed once per tile
struct TcSite {
  int s, par, xh, y, z, t, xodd;
};
__device__ __forceinline__ TcSite tc_site(const Geom &g, int s, int par) {
  TcSite c;
  c.s = s;
  c.par = par;
  c.xh = s % g.Lxh;
  int r = s / g.Lxh;
  c.y = r % g.Ly;
  r /= g.Ly;
  c.z = r % g.Lz;
  c.t = r / g.Lz;
  c.xodd = (c.y + c.z + c.t + par) & 1;
  return c;
}
// neighbour index of hop (mu, fwd) and whether it crosses the t boundary
__device__ __forceinline__ int tc_hop_nbr(const Geom &g, const TcSite &c, int mu, int fwd, bool &tcross) {
  const int s = c.s;
  tcross = false;
  switch (mu) {
    case 0:
      return fwd ? (c.xodd ? (c.xh == g.Lxh - 1 ? s - c.xh : s + 1) : s) : (c.xodd ? s : (c.xh == 0 ? s + g.Lxh - 1 : s - 1));
    case 1:
      return fwd ? (c.y == g.Ly - 1 ? s - (g.Ly - 1) * g.sy : s + g.sy) : (c.y == 0 ? s + (g.Ly - 1) * g.sy : s - g.sy);
    case 2:
      return fwd ? (c.z == g.Lz - 1 ? s - (g.Lz - 1) * g.sz : s + g.sz) : (c.z == 0 ? s + (g.Lz - 1) * g.sz : s - g.sz);
    default:
      tcross = fwd ? (c.t == g.Lt - 1) : (c.t == 0);
      return fwd ? (c.t == g.Lt - 1 ? s - (g.Lt - 1) * g.st : s + g.st) : (c.t == 0 ? s + (g.Lt - 1) * g.st : s - g.st);
  }
}

__device__ __forceinline__ uint32_t bf16x2_rn(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// One hop of this thread's row of A: T_h in at the output site, rounded to
// bf16 and stored at K = hh * 2 CIN ([Re of the CIN channels | Im of them])
// in each colour's A tile; zero where the input has no parity (layer 1's
// input lives on the odd sites only), past the ninth hop, or for rows past
// the last site.  Four channels at a time, to bound the registers a thread
// holds; the colour products run on paired FP32 instructions, (re, im) of an
// output element as one lane pair.
template <int CIN, int IN, int KC, int A_COLOUR_BYTES>
__device__ __forceinline__ void tc_stage_hop(const TcArgs &a, bool valid, const TcSite &cs, int h, int hh, uint8_t *A,
                                             int row) {
  const Geom &g = a.g;
  const int par = cs.par;
  const int src_par = h == 0 ? par : 1 - par;
  const bool zero = !valid || h >= NN_HOPS || (IN == TC_SOA64 && src_par != 1);
  int n = cs.s, mu = 0, fwd = 0;
  bool tc = false;
  float2 ur[9], ui[9];  // link elements of the colour product, each broadcast to a lane pair
  if (!zero && h > 0) {
    mu = (h - 1) >> 1;
    fwd = h & 1;
    n = tc_hop_nbr(g, cs, mu, fwd, tc);
    Cpx<float> u[9];
    const GaugeView<GSOA16> U{a.gauge, pad_sites(g.Vh)};
    link_load<GSOA16, float>(U, mu, fwd ? par : 1 - par, fwd ? cs.s : n, u);
    const float ph = tc ? a.t_bc : 1.f;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) {  // m = U_rc (forward) or conj(U_cr) (backward), times the t phase
        const Cpx<float> m = fwd ? u[r * 3 + c] : u[c * 3 + r].conj();
        ur[r * 3 + c] = make_float2(m.re * ph, m.re * ph);
        ui[r * 3 + c] = make_float2(m.im * ph, m.im * ph);
      }
  }
  const double2 *p64 = nullptr;
  const uint32_t *p16 = nullptr;
  if constexpr (IN == TC_SOA64) {
    p64 = static_cast<const double2 *>(a.in) + blk_base<12>(n);
  } else {
    p16 = static_cast<const uint32_t *>(a.in) + hid_index(pad_sites(g.Vh), src_par, n, 0);
  }
#pragma unroll
  for (int b4 = 0; b4 < CIN; b4 += 4) {
    float2 v[4][3];
    if (zero) {
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int c = 0; c < 3; c++) v[b][c] = make_float2(0.f, 0.f);
    } else {
      float2 q[4][3];
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const int comp = (b4 + b) * 3 + c;
          if constexpr (IN == TC_SOA64) {
            const double2 d = __ldg(p64 + comp * SB);
            q[b][c] = make_float2((float)d.x, (float)d.y);
          } else {
            const uint32_t w = __ldg(p16 + comp * 32);
            q[b][c] = make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
          }
        }
      if (h == 0) {
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int c = 0; c < 3; c++) v[b][c] = q[b][c];
      } else {
#pragma unroll
        for (int b = 0; b < 4; b++) {
          float2 qs[3];  // i q: (-Im, Re)
#pragma unroll
          for (int c = 0; c < 3; c++) qs[c] = make_float2(-q[b][c].y, q[b][c].x);
#pragma unroll
          for (int r = 0; r < 3; r++) {
            float2 acc = __fmul2_rn(ur[r * 3], q[b][0]);
            acc = __ffma2_rn(ui[r * 3], qs[0], acc);
#pragma unroll
            for (int c = 1; c < 3; c++) {
              acc = __ffma2_rn(ur[r * 3 + c], q[b][c], acc);
              acc = __ffma2_rn(ui[r * 3 + c], qs[c], acc);
            }
            v[b][r] = acc;
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      uint8_t *Ac = A + c * A_COLOUR_BYTES;
#pragma unroll
      for (int ri = 0; ri < 2; ri++) {
        const int k0 = hh * 2 * CIN + ri * CIN + b4;
        const float x0 = ri ? v[0][c].y : v[0][c].x, x1 = ri ? v[1][c].y : v[1][c].x;
        const float x2 = ri ? v[2][c].y : v[2][c].x, x3 = ri ? v[3][c].y : v[3][c].x;
        *reinterpret_cast<uint2 *>(Ac + kmajor_off(row, k0, KC)) = make_uint2(bf16x2_rn(x0, x1), bf16x2_rn(x2, x3));
      }
    }
  }
}

template <int CIN, int COUT, int IN, int OUT>
__global__ void __launch_bounds__(TC_THREADS) k_nn_tc(TcArgs a, long long nsites) {
  using S = TcShape<CIN, COUT>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint8_t *sA = smem + S::B_BYTES;  // two buffers of three colours
  uint64_t *bars = reinterpret_cast<uint64_t *>(sA + 2 * S::A_BYTES);  // [0], [1]: A buffers
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const Geom &g = a.g;

  // B: the real form of W (bf16), K ordered (chunk, hop in chunk, re/im, input channel)
  for (int e = tid; e < S::B_ROWS * S::KPAD; e += TC_THREADS) {
    const int n = e / S::KPAD, K = e % S::KPAD;
    const int ch = K / S::KC, kk = K % S::KC;
    const int h = ch * S::HOPS_PER_CHUNK + kk / (2 * CIN), ri = (kk / CIN) & 1, b = kk % CIN;
    float val = 0.f;
    if (h < NN_HOPS && n < 2 * COUT) {
      const int o = n % COUT;
      const uint32_t w = a.w16[(h * COUT + o) * CIN + b];
      const float wr = __uint_as_float(w << 16), wi = __uint_as_float(w & 0xffff0000u);
      if (n < COUT) val = ri == 0 ? wr : -wi;  // Re out = Wr vr - Wi vi
      else val = ri == 0 ? wi : wr;            // Im out = Wi vr + Wr vi
    }
    *reinterpret_cast<__nv_bfloat16 *>(sB + kmajor_off(n, K, S::KPAD)) = __float2bfloat16_rn(val);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)S::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int k = 0; k < 2; k++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[k])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // B visible to the tensor core
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc<S::N>();
  const uint32_t sA0 = smem_u32(sA), sB0 = smem_u32(sB);
  unsigned issued[2] = {0, 0}, waited[2] = {0, 0};
  unsigned q = 0;  // chunks issued so far by this CTA
  bool ok = true;
  const long long ntiles = (nsites + TC_THREADS - 1) / TC_THREADS;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long idx = tile * TC_THREADS + tid;
    const bool valid = idx < nsites;
    // layer 1 writes both parities (index = parity * Vh + site), layer 2 the odd one
    const int par = OUT == TC_HID16 ? (int)(idx / g.Vh) : 1;
    const int s = OUT == TC_HID16 ? (int)(idx % g.Vh) : (int)idx;
    const TcSite cs = tc_site(g, valid ? s : 0, par);
    for (int ch = 0; ch < S::NCHUNK && ok; ch++, q++) {
      const int buf = q & 1;
      if (issued[buf] > waited[buf]) {  // the MMAs that read this buffer two chunks ago are done
        ok = mbar_wait(smem_u32(&bars[buf]), waited[buf] & 1);
        waited[buf]++;
      }
      uint8_t *A = sA + buf * S::A_BYTES;
#pragma unroll
      for (int hh = 0; hh < S::HOPS_PER_CHUNK; hh++)
        tc_stage_hop<CIN, IN, S::KC, S::A_COLOUR_BYTES>(a, valid, cs, ch * S::HOPS_PER_CHUNK + hh, hh, A, tid);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A visible to the tensor core
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      ok = __syncthreads_and(ok);  // a timed-out wait stops every thread alike
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (!ok) break;
      if (tid == 0) {
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int ks = 0; ks < S::KSTEPS; ks++) {
            const uint64_t ad = umma_desc(sA0 + buf * S::A_BYTES + c * S::A_COLOUR_BYTES + ks * 256, 128,
                                          S::KC / 8 * 128);
            const uint64_t bd = umma_desc(sB0 + (ch * S::KC / 16 + ks) * 256, 128, S::B_SBO);
            umma_f16(tmem + c * S::N, ad, bd, idesc, (ch > 0 || ks > 0) ? 1u : 0u);
          }
        umma_commit(smem_u32(&bars[buf]));
      }
      issued[buf]++;
    }
    if (!ok) break;
    // all MMAs of this tile done: the later of the two buffers' commits covers them
    for (int k = 0; k < 2; k++)
      if (issued[k] > waited[k]) {
        ok = mbar_wait(smem_u32(&bars[k]), waited[k] & 1) && ok;
        waited[k]++;
      }
    ok = __syncthreads_and(ok);
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float2 o[COUT][3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int n0 = 0; n0 < S::N; n0 += 16) {
        float d[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c * S::N + n0, d);
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int n = n0 + j;
          if (n < COUT) o[n][c].x = d[j];
          else if (n < 2 * COUT) o[n - COUT][c].y = d[j];
        }
      }
    }
    if (valid) {
      if constexpr (OUT == TC_HID16) {
        uint32_t *p = static_cast<uint32_t *>(a.out);
        const int Vp = pad_sites(g.Vh);
#pragma unroll
        for (int oc = 0; oc < COUT; oc++)
#pragma unroll
          for (int c = 0; c < 3; c++) p[hid_index(Vp, par, s, oc * 3 + c)] = bf16x2_rn(o[oc][c].x, o[oc][c].y);
      } else {
        double2 *p = static_cast<double2 *>(a.out) + blk_base<12>(s);
#pragma unroll
        for (int oc = 0; oc < COUT; oc++)
#pragma unroll
          for (int c = 0; c < 3; c++) p[(oc * 3 + c) * SB] = make_double2(o[oc][c].x, o[oc][c].y);
      }
    }
    // the next tile's first MMAs overwrite D only after every warp has read it
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
  // drain: no MMA of this CTA may still be writing tensor memory when it is freed
  for (int k = 0; k < 2; k++)
    if (issued[k] > waited[k]) {
      if (!mbar_wait(smem_u32(&bars[k]), waited[k] & 1) && tid == 0) atomicExch(a.err, 1);
      waited[k]++;
    }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)S::TMEM_COLS)
                 : "memory");
  }
}

template <int CIN, int COUT, int IN, int OUT>
void launch_tc(const TcArgs &a, long long nsites, int sms, cudaStream_t s) {
  using S = TcShape<CIN, COUT>;
  // shared memory per CTA caps the CTAs per SM so that their tensor memory
  // (TMEM_COLS columns each) fits in the SM's 512 columns
  const int per_sm = 512 / S::TMEM_COLS;
  const int smem = std::max(S::SMEM, 232448 / per_sm - 1024);
  auto k = k_nn_tc<CIN, COUT, IN, OUT>;
  QCU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  QCU_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  const long long ntiles = (nsites + TC_THREADS - 1) / TC_THREADS;
  // as many CTAs as can be resident (shared memory allows at most per_sm per
  // SM; CTAs beyond that start, and allocate tensor memory, as others finish)
  const int resident = std::min(per_sm, 233472 / (smem + 1024));
  const int grid = (int)std::min<long long>(ntiles, (long long)sms * resident);
  k<<<grid, TC_THREADS, smem, s>>>(a, nsites);
  QCU_CHECK_LAUNCH();
}

}  // namespace

void launch_nn_tc(const Geom &g, const void *gauge16, float t_bc, const uint32_t *w16_1, const uint32_t *w16_2,
                  const void *r64, void *hid16, void *z64, int *err, int sms, cudaStream_t s) {
  TcArgs a;
  a.g = g;
  a.gauge = gauge16;
  a.t_bc = t_bc;
  a.err = err;
  // layer 1: odd residual (FP64) -> hidden field on both parities (bf16)
  a.in = r64;
  a.out = hid16;
  a.w16 = w16_1;
  launch_tc<NN_C_IN, NN_C_HID, TC_SOA64, TC_HID16>(a, 2LL * g.Vh, sms, s);
  // layer 2: hidden field -> N(r) on the odd sites (FP64)
  a.in = hid16;
  a.out = z64;
  a.w16 = w16_2;
  launch_tc<NN_C_HID, NN_C_OUT, TC_HID16, TC_SOA64>(a, g.Vh, sms, s);
}

size_t nn_hid16_bytes(int Vh) { return (size_t)2 * pad_sites(Vh) * HID_COMP * sizeof(uint32_t); }

}  // namespace qcu
