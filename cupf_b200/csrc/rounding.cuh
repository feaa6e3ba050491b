// rounding.cuh — stochastic rounding of FP32 values to 16-bit floats.
//
// x goes to the 16-bit value below or above it with probabilities proportional
// to its distance from the other one, so the expected stored value equals the
// FP32 value.  Round-to-nearest drops every per-step change smaller than half a
// 16-bit spacing, which biases slowly varying fields of an explicit time step;
// stochastic rounding does not.  The rounding itself is sm_100a's conversion
// with random bits (cvt.rs); the bits come from mix32 of a counter (cell,
// step), so results are reproducible.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace cupf {

// 32-bit integer finaliser (the "lowbias32" xorshift-multiply constants
// published by C. Wellons, 2018): a counter-based source of rounding bits.
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Stochastic rounding of two FP32 values to a packed pair of 16-bit floats in
// one sm_100a instruction (cvt.rs): the upper half of the result is hi rounded
// with the random bits r[31:16], the lower half lo rounded with r[15:0]; each
// rounds down or up in magnitude with probabilities proportional to its
// distance from the other neighbour (all-zero bits truncate toward zero),
// subnormal results included.  |hi|, |lo| must be at most the largest finite
// value of the format.
__device__ __forceinline__ uint32_t sr_pack_fp16x2(float hi, float lo, uint32_t r) {
  uint32_t d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
  return d;
}
__device__ __forceinline__ uint32_t sr_pack_bf16x2(float hi, float lo, uint32_t r) {
  uint32_t d;
  asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
  return d;
}

}  // namespace cupf
