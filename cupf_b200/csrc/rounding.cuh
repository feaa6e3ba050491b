// rounding.cuh — stochastic rounding of FP32 values to 16-bit floats.
//
// x goes to the 16-bit value below or above it with probabilities proportional
// to its distance from the other one, so the expected stored value equals the
// FP32 value.  Round-to-nearest drops every per-step change smaller than half a
// 16-bit spacing, which biases slowly varying fields of an explicit time step;
// stochastic rounding does not.  The random bits come from mix32 of a counter
// (cell, field, step), so results are reproducible.
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

// BF16 keeps the top 16 bits of the FP32 pattern: add 16 random bits below
// them, then truncate the magnitude.  |x| must be below the largest finite
// BF16 value.
__device__ __forceinline__ unsigned short sr_bf16_bits(float x, uint32_t r) {
  const uint32_t sign = __float_as_uint(x) & 0x80000000u;
  const uint32_t b = (__float_as_uint(fabsf(x)) + (r >> 16)) & 0xFFFF0000u;
  return (unsigned short)((b | sign) >> 16);
}

// FP16: the spacing at |x| is 2^(E-10) for E >= -14 (normal values) and 2^-24
// below; add a uniform fraction of it, then round toward zero.  |x| must be at
// most 65504.
__device__ __forceinline__ unsigned short sr_fp16_bits(float x, uint32_t r) {
  const uint32_t sign = __float_as_uint(x) & 0x80000000u;
  const float a = fabsf(x);
  uint32_t e = __float_as_uint(a) & 0x7F800000u;
  const uint32_t emin = (uint32_t)(127 - 14) << 23;
  e = (e < emin ? emin : e) - (10u << 23);
  // a uniform fraction in [0, 1) from the top 23 bits of r: the float 1.f
  // with those bits as its mantissa, minus 1 (exact)
  const float f = __fsub_rn(__uint_as_float(0x3F800000u | (r >> 9)), 1.0f);
  const float t = __fmaf_rn(f, __uint_as_float(e), a);
  return (unsigned short)(__half_as_ushort(__float2half_rz(t)) | (sign >> 16));
}

}  // namespace cupf
