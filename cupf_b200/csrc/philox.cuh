// philox.cuh — counter-based random numbers shared by the kernels.
//
// Philox4x32-10 is the published generator of Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3" (SC 2011): ten rounds of
// two 32x32->64 multiplies with Weyl-sequence key bumps.
#pragma once

#include <stdint.h>

namespace cupf {

struct Philox4 {
  uint32_t v[4];
};

__host__ __device__ inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

// Philox4x32-10 of counter (c0..c3) under key (k0, k1).
__host__ __device__ inline Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                 uint32_t c3, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;  // round multipliers
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;  // key increments
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c0, &hi0, &lo0);
    mulhilo32(M1, c2, &hi1, &lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    k0 += W0;
    k1 += W1;
  }
  Philox4 out;
  out.v[0] = c0;
  out.v[1] = c1;
  out.v[2] = c2;
  out.v[3] = c3;
  return out;
}

// Uniform in (0, 1] from 24 bits, like curand_uniform's open-at-zero range.
__host__ __device__ inline float uniform01(uint32_t x) {
  return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

}  // namespace cupf
