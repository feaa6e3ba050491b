// apt_storage.cuh — storage formats of one (phi, grain id) slot pair.
//
// PairF32: the reference's own precision, {float phi, int32 id} in 8 bytes.
// PairH16<F>: split precision, {16-bit phi code, int16 id} in 4 bytes, the code
//   in BF16 or FP16 (the step stores with stochastic rounding, set-up paths
//   round to nearest even); ids must fit in int16 (-1 = empty).
// The step computes in FP32 for every format; only the stored pair differs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "apt_common.cuh"
#include "rounding.cuh"

namespace cupf {

struct PairF32 {
  using T = uint2;
  static constexpr int kBytes = 8;
  static constexpr int kBW = 34;  // TMA box width in cells: 34*8 = 272 B (16 B multiple)
  static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT64;
  static constexpr int kPitchAlign = 2;  // pitch in cells so rows start on 16 B
  __host__ __device__ static float phi(T p) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(p.x);
#else
    float f;
    memcpy(&f, &p.x, 4);
    return f;
#endif
  }
  __host__ __device__ static int id(T p) { return (int)p.y; }
  __device__ static T make(float ph, int id) { return make_uint2(__float_as_uint(ph), (uint32_t)id); }
  __device__ static T empty() { return make_uint2(0xBF800000u, 0xFFFFFFFFu); }
  __device__ static bool is_empty(T p) { return p.x == 0xBF800000u && p.y == 0xFFFFFFFFu; }
  static constexpr bool kStochastic = false;
  __device__ static T make_sr(float ph, int id, uint32_t) { return make(ph, id); }
};

enum class Half16 { BF16, FP16 };

// 16-bit phi is stored in one of two bands, told apart by the code's magnitude:
//   |phi| >= 1/2: c = copysign(1 - |phi|, phi), |c| <= 1/2 (the distance to the
//                 nearest bulk value: c = +0 for phi = +1, -0 for phi = -1, so
//                 empty slots stay exact);
//   |phi| <  1/2: c = copysign(1 + K |phi|, phi), K = 4096, |c| in [1, 2049).
// A 16-bit float keeps ~11 (FP16) or 8 (BF16) significant bits of c: relative
// precision of 1 - |phi| in the tanh profile's tails, which approach the bulk
// values and change by less than a plain 16-bit spacing per step, and relative
// precision of |phi| in the interface core, where two grains' phi cross and the
// argmax that gives grain volumes is decided.  The coarsest spacing is 2.4e-4
// (FP16) at |phi| near 1/2; near phi = 0 it is far finer (a distance code alone
// spaces phi = 0 by 4.9e-4).  Values outside [-1, 1] (rounding overshoot) are
// stored as +-1.  Both bands' decodes are exact in FP32.
template <Half16 F>
struct PairH16 {
  using T = uint32_t;
  static constexpr int kBytes = 4;
  static constexpr int kBW = 36;  // 36*4 = 144 B (16 B multiple)
  static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT32;
  static constexpr int kPitchAlign = 4;
  static constexpr float kCore = 4096.0f;
  __device__ static float decode(unsigned short b) {
    const float c = (F == Half16::BF16) ? __bfloat162float(__ushort_as_bfloat16(b))
                                        : __half2float(__ushort_as_half(b));
    // both bands as (c - s) k, s = sign of c: k = 1/K in the core, k = -1 in the
    // tails (s - c exactly); the products are exact
    const float s = copysignf(1.0f, c);
    const float k = fabsf(c) >= 1.0f ? 1.0f / kCore : -1.0f;
    return __fmul_rn(__fsub_rn(c, s), k);
  }
  // the FP32 value of the code before rounding to 16 bits
  __device__ static float code(float ph) {
    const float a = fabsf(ph);
    // 1 - a is exact for a >= 1/2; clamped at 0 for overshoot past the bulk value
    const float m = a >= 0.5f ? fmaxf(__fsub_rn(1.0f, a), 0.0f) : __fmaf_rn(a, kCore, 1.0f);
    return copysignf(m, ph);
  }
  __device__ static unsigned short encode(float ph) {
    const float c = code(ph);
    if (F == Half16::BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(c));
    return __half_as_ushort(__float2half_rn(c));
  }
  static constexpr bool kStochastic = true;
  // The step's store, with stochastic rounding (r: 32 random bits, of which the
  // hardware conversion cvt.rs uses r[31:16]): the code goes to the 16-bit
  // value below or above it with probabilities proportional to its distance
  // from the other one, so the expected stored value equals the FP32 result.
  // Round-to-nearest drops every per-step change smaller than half a 16-bit
  // spacing, which biases slowly moving interfaces; this does not.  The rounded
  // code lands in the upper half of the conversion's result and is moved to the
  // low half of the pair, beside the id.
  __device__ static T make_sr(float ph, int id, uint32_t r) {
    const float c = code(ph);
    const uint32_t d = (F == Half16::BF16) ? sr_pack_bf16x2(c, 0.0f, r) : sr_pack_fp16x2(c, 0.0f, r);
    return __byte_perm(d, (uint32_t)id, 0x5432);
  }
  __device__ static float phi(T p) { return decode((unsigned short)(p & 0xFFFFu)); }
  __device__ static int id(T p) { return (int)(short)(p >> 16); }
  __device__ static T make(float ph, int id) {
    return (uint32_t)encode(ph) | ((uint32_t)(unsigned short)(short)id << 16);
  }
  __device__ static T empty() { return 0xFFFF8000u; }  // c = -0 (phi = -1), id -1
  __device__ static bool is_empty(T p) { return p == 0xFFFF8000u; }
};

using PairBF16 = PairH16<Half16::BF16>;
using PairFP16 = PairH16<Half16::FP16>;

}  // namespace cupf
