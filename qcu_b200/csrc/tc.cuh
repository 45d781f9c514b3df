// tcgen05 building blocks shared by the tensor-core kernels (nn_tc.cu,
// mrhs_tc.cu): shared-memory matrix descriptors (K-major, no swizzle), the
// kind::f16 MMA, its commit, bounded mbarrier waits and tensor-memory loads.
#pragma once
#include <cstdint>

namespace qcu {

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

// instruction descriptor of tcgen05.mma kind::f16 (K-major A and B, FP32
// accumulator): bits 4-5 D type (1 = F32), 7-9 A type and 10-12 B type
// (0 = F16, 1 = BF16), 17-22 N / 8, 24-28 M / 16
template <int M, int N>
__device__ __forceinline__ uint32_t umma_idesc_f16(bool bf16) {
  static_assert(M == 64 || M == 128, "M");
  static_assert(N % 8 == 0 && N >= 8 && N <= 256 && (M == 64 || N % 16 == 0), "N");
  const uint32_t ab = bf16 ? 1u : 0u;
  return (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (tensor memory) [+]= A (shared) x B (shared)^T, issued by one thread
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
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



}  // namespace qcu
