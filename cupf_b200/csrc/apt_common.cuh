// apt_common.cuh — shared device definitions of the B200 APT step.
//
// Device memory layout of one slot buffer ("pair planes"):
//   pair[slot][z][y][x]   with x pitch xp (even, >= fnx), 8-byte pairs
//   pair = { float phi, int32 id }           (id -1 = empty slot)
// i.e. the reference's SoA slot layout (devicefunc.cu_inl:24-29) with phi and
// id interleaved and the x rows padded so every row starts on a 16-byte
// boundary, which is what a TMA tensor map needs.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cupf.h"

namespace cupf {

constexpr double LS = -0.995;     // liquid threshold (APTPhaseField.cu:25)
constexpr double ID_DROP = -0.9999; // id is dropped below this phi (:341)
// The reference compares float phi with these double literals.  For a float f,
//   (double)f > -0.995  <=>  f > 0xbf7eb852 (-0.99500000477...)  (largest float <= -0.995)
//   (double)f < -0.9999 <=>  f < 0xbf7ff972 (-0.99989998340...)  (smallest float >= -0.9999)
// so the kernels compare in single precision with these bit patterns.
constexpr uint32_t kLSFloatBits = 0xbf7eb852u;
constexpr uint32_t kDropFloatBits = 0xbf7ff972u;

// Per-launch arguments of the step kernel (passed by value).
struct StepArgs {
  int fnx, fny, fnz, xp;
  long long slot_stride;  // pairs per slot plane set = xp*fny*fnz
  int bcX, bcY, bcZ;
  int ntx, nty, nzc, zc;  // tile grid and z-chunk length
  int num_theta, thermalType, use_iuc;
  // num_theta as an invariant divisor (invariant_divisor): the orientation index
  // of a nucleated id, id % num_theta + 1, without a divide instruction
  uint32_t nt_magic;
  int nt_sh1, nt_sh2;
  float t;
  // time and height coordinates in FP64 (fp64 != 0: 16-bit storage, whose long
  // runs keep time, the moving-domain offset and the thermal model's
  // coordinates in double); t and z are the reference's FP32 forms
  int fp64;
  double t64;
  const double* z64;
  uint32_t sr_key;  // per-step key of the stochastic-rounding bits (16-bit storage)
  float kin_delta, eps, G, z0, uc, uc0, L_cp, hi, lamd, dt, tau0;
  float lyd, lzd, r0, x0, angle, V, mp_len, order;
  int Nx, Ny, Nz;
  const float* x;
  const float* y;
  const float* z;
  const float* sint;
  const float* cost;
  const float4* orient;  // per orientation index 0..NG: {sint[i], cost[i], sint[i+NG], cost[i+NG]}
  const float* X_mac;
  const float* Y_mac;
  const float* Z_mac;
  const float* psi_mac;
  const void* in;    // pair buffer read this step (storage format of the launch)
  void* out;         // pair buffer written this step
  int* err;          // device error word (0 = ok)
  int* work;         // [next item, CTAs done] of the persistent launch (self-resetting)
  // Quiet-item flags (NULL = off): per work item, bit 0 set when every interior
  // cell of the item holds only exact empty pairs (id -1, phi -1) in that
  // buffer, bits 1 and 2 the same for its bottom and its top plane.  quiet_in describes `in`,
  // quiet_out describes `out` as it stands before this step and is rewritten
  // for every item the step computes.
  const uint8_t* quiet_in;
  uint8_t* quiet_out;
  unsigned long long* active_cells;  // cells of the computed items, accumulated (may be NULL)
  // merge overflows (more than NUM_PF distinct ids in a stencil), accumulated
  // (may be NULL): [0] entries aliased into the next point's slot 0 (s < 6),
  // [1] entries dropped at the last point (s == 6)
  unsigned long long* overflows;
  long long wait_limit;  // SM cycles a stage wait may spin before the step gives up
};

// Unsigned division by a divisor fixed for a launch, by a multiply and shifts
// (T. Granlund and P. Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, fig. 4.1): for 1 <= d < 2^31 and every 32-bit n,
// n / d = (t + ((n - t) >> s1)) >> s2 with t = mulhi(m, n), where
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, s1 = min(l, 1) and
// s2 = max(l - 1, 0).
struct InvariantDivisor {
  uint32_t m;
  int s1, s2;
};
inline InvariantDivisor invariant_divisor(uint32_t d) {
  InvariantDivisor v{0u, 0, 0};
  if (d == 0) return v;
  int l = 0;
  while ((1ull << l) < d) ++l;
  v.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
  v.s1 = l < 1 ? l : 1;
  v.s2 = l > 1 ? l - 1 : 0;
  return v;
}
__host__ __device__ __forceinline__ uint32_t div_invariant(uint32_t n, uint32_t m, int s1,
                                                           int s2) {
#ifdef __CUDA_ARCH__
  const uint32_t t = __umulhi(m, n);
#else
  const uint32_t t = (uint32_t)(((unsigned long long)m * n) >> 32);
#endif
  return (t + ((n - t) >> s1)) >> s2;
}

// Boundary map of one coordinate (APTsetBC3D, APTPhaseField.cu:111-112,134-135,157-158):
// no-flux mirrors about the first/last interior point, periodic wraps.
__host__ __device__ __forceinline__ int bc_map(int c, int fn, int bc) {
  if (c == 0) return bc == 0 ? 2 : fn - 2;
  if (c == fn - 1) return bc == 0 ? fn - 3 : 1;
  return c;
}

enum ErrCode { ERR_TMA_TIMEOUT = 1 };

// Orientation table of the step: entry i (0..num_theta) packs the two angles'
// sines and cosines {sint[i], cost[i], sint[i+NG], cost[i+NG]} so that a slot
// update reads them with one 16-byte load.  sint/cost have 2*NG+1 entries.
inline void pack_orientations(const float* sint, const float* cost, int num_theta, float* out) {
  for (int i = 0; i <= num_theta; ++i) {
    out[4 * i + 0] = sint[i];
    out[4 * i + 1] = cost[i];
    out[4 * i + 2] = sint[i + num_theta];
    out[4 * i + 3] = cost[i + num_theta];
  }
}

}  // namespace cupf
