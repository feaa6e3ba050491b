// apt_storage.cuh — storage formats of one (phi, grain id) slot pair.
//
// PairF32: the reference's own precision, {float phi, int32 id} in 8 bytes.
// PairH16<F>: split precision, {16-bit phi, int16 id} in 4 bytes, phi in BF16
//   or FP16 (round to nearest even on store); ids must fit in int16 (-1 = empty).
// The step computes in FP32 for every format; only the stored pair differs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "apt_common.cuh"

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
};

enum class Half16 { BF16, FP16 };

template <Half16 F>
struct PairH16 {
  using T = uint32_t;
  static constexpr int kBytes = 4;
  static constexpr int kBW = 36;  // 36*4 = 144 B (16 B multiple)
  static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT32;
  static constexpr int kPitchAlign = 4;
  __device__ static float phi(T p) {
    const unsigned short b = (unsigned short)(p & 0xFFFFu);
    if (F == Half16::BF16) return __bfloat162float(__ushort_as_bfloat16(b));
    return __half2float(__ushort_as_half(b));
  }
  __device__ static int id(T p) { return (int)(short)(p >> 16); }
  __device__ static T make(float ph, int id) {
    unsigned short b;
    if (F == Half16::BF16) b = __bfloat16_as_ushort(__float2bfloat16_rn(ph));
    else b = __half_as_ushort(__float2half_rn(ph));
    return (uint32_t)b | ((uint32_t)(unsigned short)(short)id << 16);
  }
  __device__ static T empty() {
    return F == Half16::BF16 ? 0xFFFFBF80u : 0xFFFFBC00u;  // phi -1, id -1
  }
};

using PairBF16 = PairH16<Half16::BF16>;
using PairFP16 = PairH16<Half16::FP16>;

}  // namespace cupf
