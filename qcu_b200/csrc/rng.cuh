// Counter-based random numbers shared by the field generators: SplitMix64's
// output function (Steele, Lea & Flood, OOPSLA 2014) evaluated at (hashed
// seed + counter * golden gamma).  Every field element owns fixed counters,
// so the numbers do not depend on the launch shape, and the CPU generator of
// the tests reproduces them exactly.
#pragma once
#include <stdint.h>

namespace qcu {

__host__ __device__ __forceinline__ uint64_t sm64_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rng_u64(uint64_t seed, uint64_t ctr) {
  const uint64_t s = sm64_mix(seed + 0x9E3779B97F4A7C15ULL);
  return sm64_mix(s + (ctr + 1) * 0x9E3779B97F4A7C15ULL);
}
// uniform in (0, 1]
__device__ __forceinline__ double rng_uniform(uint64_t seed, uint64_t ctr) {
  return (double)((rng_u64(seed, ctr) >> 11) + 1) * (1.0 / 9007199254740992.0);
}

}  // namespace qcu
