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
// A CTA of 128 threads owns a tile of 128 output sites; each thread is one
// site, i.e. one row of three M = 128 GEMMs (one per colour, sharing B):
//   * the FMA pipes compute the parallel transports T_h in (FP32, from the
//     FP32 reconstruct-12 links), a chunk of hops at a time (K = 16 or 32
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
  static constexpr int B_BYTES = N * KPAD * 2;
  static constexpr int A_COLOUR_BYTES = 128 * KC * 2;
  static constexpr int A_BYTES = 3 * A_COLOUR_BYTES;   // one buffer: three colours
  static constexpr int SMEM = B_BYTES + 2 * A_BYTES + 64;
};

constexpr int TC_THREADS = 128;
constexpr unsigned TC_WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row, k) in a K-major no-swizzle operand whose rows
// hold `kpad` elements: 8-row x 8-element core matrices of 128 contiguous
// bytes, adjacent along K (LBO = 128 B), then along rows (SBO = kpad / 8 * 128 B)
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int kpad) {
  return (uint32_t)((row >> 3) * (kpad / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor of tcgen05 (no swizzle)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, relative LBO, no swizzle
}

// instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D, M = 128
template <int N>
__device__ __forceinline__ uint32_t umma_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned i = 0; i < TC_WAIT_LIMIT; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > 64) __nanosleep(64);
  }
  return false;
}

// 16 consecutive FP32 columns of this warp's 32 tensor-memory lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
  const __nv_bfloat16 a = __float2bfloat16_rn(lo), b = __float2bfloat16_rn(hi);
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// the neighbour, link and t-phase of hop h (the transport of nn.cu, FP32)
__device__ __forceinline__ int tc_nbr(const Geom &g, int s, int par, int mu, int fwd, bool &tcross) {
  const int xh = s % g.Lxh;
  int r = s / g.Lxh;
  const int y = r % g.Ly;
  r /= g.Ly;
  const int z = r % g.Lz;
  const int t = r / g.Lz;
  const int xodd = (y + z + t + par) & 1;
  tcross = false;
  switch (mu) {
    case 0:
      return fwd ? (xodd ? (xh == g.Lxh - 1 ? s - xh : s + 1) : s) : (xodd ? s : (xh == 0 ? s + g.Lxh - 1 : s - 1));
    case 1:
      return fwd ? (y == g.Ly - 1 ? s - (g.Ly - 1) * g.sy : s + g.sy) : (y == 0 ? s + (g.Ly - 1) * g.sy : s - g.sy);
    case 2:
      return fwd ? (z == g.Lz - 1 ? s - (g.Lz - 1) * g.sz : s + g.sz) : (z == 0 ? s + (g.Lz - 1) * g.sz : s - g.sz);
    default:
      tcross = fwd ? (t == g.Lt - 1) : (t == 0);
      return fwd ? (t == g.Lt - 1 ? s - (g.Lt - 1) * g.st : s + g.st) : (t == 0 ? s + (g.Lt - 1) * g.st : s - g.st);
  }
}

// v = T_h in at (s, par): CIN colour vectors (zero if the hop's source parity holds no input)
template <int CIN>
__device__ __forceinline__ void tc_transport(const Geom &g, const PtcArgs &a, const float2 *in_sample, int s, int par,
                                             int h, float2 (&v)[CIN][3]) {
  const int src_par = h == 0 ? par : 1 - par;
  if (h >= NN_HOPS || !(a.in_mask >> src_par & 1)) {
#pragma unroll
    for (int b = 0; b < CIN; b++)
#pragma unroll
      for (int c = 0; c < 3; c++) v[b][c] = make_float2(0.f, 0.f);
    return;
  }
  const size_t slab = (size_t)src_par * g.Vh;
  if (h == 0) {
    const float2 *p = in_sample + (slab + s) * CIN * 3;
#pragma unroll
    for (int b = 0; b < CIN; b++)
#pragma unroll
      for (int c = 0; c < 3; c++) v[b][c] = p[b * 3 + c];
    return;
  }
  const int mu = (h - 1) >> 1, fwd = (h & 1);
  bool tc;
  const int n = tc_nbr(g, s, par, mu, fwd, tc);
  Cpx<float> u[9];
  const GaugeView<GSOA32> U{a.gauge, pad_sites(g.Vh)};
  link_load<GSOA32, float>(U, mu, fwd ? par : 1 - par, fwd ? s : n, u);
  const float ph = tc ? a.t_bc : 1.f;
  const float2 *p = in_sample + (slab + n) * CIN * 3;
#pragma unroll
  for (int b = 0; b < CIN; b++) {
    float2 q[3];
#pragma unroll
    for (int c = 0; c < 3; c++) q[c] = p[b * 3 + c];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const Cpx<float> m = fwd ? u[r * 3 + c] : u[c * 3 + r].conj();
        re += m.re * q[c].x - m.im * q[c].y;
        im += m.re * q[c].y + m.im * q[c].x;
      }
      v[b][r] = make_float2(re * ph, im * ph);
    }
  }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(TC_THREADS) k_ptc_tc(Geom g, PtcArgs a, long long nsites, int *err) {
  using S = TcShape<CIN, COUT>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint8_t *sA = smem + S::B_BYTES;  // two buffers of three colours
  uint64_t *bars = reinterpret_cast<uint64_t *>(sA + 2 * S::A_BYTES);  // [0], [1]: A buffers
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;

  // B: the real form of W (bf16), K ordered (chunk, hop in chunk, re/im, input channel)
  for (int e = tid; e < S::N * S::KPAD; e += TC_THREADS) {
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
  const int np = (a.out_mask & 1) + (a.out_mask >> 1 & 1);
  unsigned issued[2] = {0, 0}, waited[2] = {0, 0};
  unsigned q = 0;  // chunks issued so far by this CTA
  bool ok = true;
  const long long ntiles = (nsites + TC_THREADS - 1) / TC_THREADS;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long idx = tile * TC_THREADS + tid;
    const bool valid = idx < nsites;
    int b = 0, par = 0, s = 0;
    if (valid) {
      const long long per = (long long)np * g.Vh;
      b = (int)(idx / per);
      const long long r = idx % per;
      s = (int)(r % g.Vh);
      par = np == 2 ? (int)(r / g.Vh) : (a.out_mask == 1 ? 0 : 1);
    }
    const float2 *in_sample = a.in + (size_t)b * 2 * g.Vh * CIN * 3;
    for (int ch = 0; ch < S::NCHUNK && ok; ch++, q++) {
      const int buf = q & 1;
      if (issued[buf] > waited[buf]) {  // the MMAs that read this buffer two chunks ago are done
        ok = mbar_wait(smem_u32(&bars[buf]), waited[buf] & 1);
        waited[buf]++;
      }
      uint8_t *A = sA + buf * S::A_BYTES;
#pragma unroll
      for (int hh = 0; hh < S::HOPS_PER_CHUNK; hh++) {
        float2 v[CIN][3];
        const int h = ch * S::HOPS_PER_CHUNK + hh;
        if (valid) tc_transport<CIN>(g, a, in_sample, s, par, h, v);
        else
#pragma unroll
          for (int bb = 0; bb < CIN; bb++)
#pragma unroll
            for (int c = 0; c < 3; c++) v[bb][c] = make_float2(0.f, 0.f);
        // row tid of colour c: [Re v_0..CIN-1 | Im v_0..CIN-1] at K = hh * 2 CIN
#pragma unroll
        for (int c = 0; c < 3; c++) {
          uint8_t *Ac = A + c * S::A_COLOUR_BYTES;
#pragma unroll
          for (int ri = 0; ri < 2; ri++)
#pragma unroll
            for (int b8 = 0; b8 < CIN; b8 += 4) {  // 4 channels = 8 bytes
              const int k0 = hh * 2 * CIN + ri * CIN + b8;
              const float x0 = ri ? v[b8][c].y : v[b8][c].x, x1 = ri ? v[b8 + 1][c].y : v[b8 + 1][c].x;
              const float x2 = ri ? v[b8 + 2][c].y : v[b8 + 2][c].x, x3 = ri ? v[b8 + 3][c].y : v[b8 + 3][c].x;
              *reinterpret_cast<uint2 *>(Ac + kmajor_off(tid, k0, S::KC)) = make_uint2(bf16x2(x0, x1), bf16x2(x2, x3));
            }
        }
      }
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
            const uint64_t bd = umma_desc(sB0 + (ch * S::KC / 16 + ks) * 256, 128, S::KPAD / 8 * 128);
            umma_bf16(tmem + c * S::N, ad, bd, idesc, (ch > 0 || ks > 0) ? 1u : 0u);
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
      float2 *out = a.out + (((size_t)b * 2 + par) * g.Vh + s) * COUT * 3;
#pragma unroll
      for (int oc = 0; oc < COUT; oc++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          float2 r = o[oc][c];
          if (a.accumulate) {
            const float2 p = out[oc * 3 + c];
            r = make_float2(r.x + p.x, r.y + p.y);
          }
          out[oc * 3 + c] = r;
        }
    }
    // the next tile's first MMAs overwrite D only after every warp has read it
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  // drain: no MMA of this CTA may still be writing tensor memory when it is freed
  for (int k = 0; k < 2; k++)
    if (issued[k] > waited[k]) {
      if (!mbar_wait(smem_u32(&bars[k]), waited[k] & 1) && tid == 0) atomicExch(err, 1);
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

template <int CIN, int COUT>
void launch_tc(const Geom &g, const PtcArgs &a, int *err, int sms, cudaStream_t s) {
  using S = TcShape<CIN, COUT>;
  // shared memory per CTA caps the CTAs per SM so that their tensor memory
  // (TMEM_COLS columns each) fits in the SM's 512 columns
  const int per_sm = 512 / S::TMEM_COLS;
  const int smem = std::max(S::SMEM, 232448 / per_sm - 1024);
  QCU_CUDA(cudaFuncSetAttribute(k_ptc_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int np = (a.out_mask & 1) + (a.out_mask >> 1 & 1);
  const long long nsites = (long long)np * g.Vh * a.B;
  const long long ntiles = (nsites + TC_THREADS - 1) / TC_THREADS;
  int per_sm_occ = 0;
  QCU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_occ, k_ptc_tc<CIN, COUT>, TC_THREADS, smem));
  require(per_sm_occ >= 1 && per_sm_occ <= per_sm, "tensor-core layer: unexpected occupancy");
  const int grid = (int)std::min<long long>(ntiles, (long long)sms * per_sm_occ);
  k_ptc_tc<CIN, COUT><<<grid, TC_THREADS, smem, s>>>(g, a, nsites, err);
  QCU_CHECK_LAUNCH();
}

}  // namespace

void launch_ptc_tc(int cin, int cout, const Geom &g, const PtcArgs &a, int *err, int sms, cudaStream_t s) {
  require(a.w16 != nullptr && !a.adjoint, "tensor-core layer: bf16 forward weights only");
  if (cin == 4 && cout == 16) launch_tc<4, 16>(g, a, err, sms, s);
  else if (cin == 16 && cout == 4) launch_tc<16, 4>(g, a, err, sms, s);
  else throw Error(1, "ptc layer: channels must be 4->16 or 16->4");
}

}  // namespace qcu
