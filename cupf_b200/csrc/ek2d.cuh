// ek2d.cuh — 2D Echebarria–Karma directional-solidification step (psi/U line
// model of cuPF 2DdendriteMPI/line_model/PF.cu) for sm_100a.
//
// One launch advances the whole grid by one step.  A CTA owns a TW x TH tile of
// output cells and works in four shared-memory phases:
//   0. load the phase field, U, dpsi of the tile plus a one-cell halo, decode
//      psi and phi (phi = tanh(psi/sqrt2)) and compute the anti-trapping flux
//      density jat = (1+(1-k)U)(1-phi^2) dpsi / 2 of every loaded cell;
//   1. plaquette means of psi and phi at the (i+1/2, j+1/2) corners
//      (psipjp .. phimjm of merge_PF, PF.cu:444-453);
//   2. fluxes on every cell edge: the anisotropic psi flux J (atheta/aptheta,
//      PF.cu:119-146, 475-538) and the solute flux of U with its anti-trapping
//      part (PF.cu:460-551).  Each edge is computed once and shared by the two
//      cells it separates (the reference computes it from both sides);
//   3. per cell: U' = U + dt*div(U flux)/tau_U (PF.cu:553-556), then the psi
//      right-hand side with the new U (PF.cu:563-590), dpsi = rhs/tau_psi,
//      psi' = psi + dt*dpsi (+ noise), and the stores.
// The reference's merge_PF (PF.cu:379-610) fuses the same U-then-psi update in
// one kernel over a 128-wide band of a linear index; the pre-loop rhs_psi
// (PF.cu:150-280) is the same psi update with U left unchanged (`prestep`).
//
// Boundary: x periodic, y mirrored about rows 1 and fny-2 (set_BC,
// PF.cu:35-73).  The reference refills the halo of the state it is about to
// read; here every writer of an interior cell that some halo cell copies also
// writes that copy, so each step's output already carries its halo.
//
// Storage S: FP32 (the reference's), FP16 / BF16 (split precision: phi (as its
// distance to the bulk value), U - U0 and dpsi in 16 bits, phi and U stored with
// stochastic rounding, arithmetic in FP32) or FP64 (double arithmetic
// throughout).  Up = (y/W0 - intR)/lT_tilde of each row
// is formed in FP64 from the host's FP64 time integration.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "philox.cuh"
#include "rounding.cuh"

namespace cupf {
namespace ek2d {

constexpr int TW = 64;  // output tile width (x, contiguous in memory)
constexpr int TH = 16;  // output tile height (y)
constexpr int NTHREADS = 256;
constexpr int IW = TW + 2, IH = TH + 2;  // input tile with its one-cell halo

// ---- storage formats -------------------------------------------------------
//
// Every format stores three planes: the phase field, U and dpsi.  ld_pp()
// decodes the phase-field plane into (psi, phi), st_ps()/st_ps_sr() encode a
// new psi; U and dpsi use ld/ldU and st/stU/st_sr.

template <class T>
__device__ __forceinline__ T tanh_t(T x);

// FP32 / FP64: psi itself, as the reference stores it; phi = tanh(psi/sqrt2).
template <class TT>
struct StPlain {
  using V = TT;
  using T = TT;
  static constexpr bool kSR = false;
  __device__ static T ld(V v) { return v; }
  __device__ static T ldU(V v, T) { return v; }
  __device__ static V st(T x) { return x; }
  __device__ static V stU(T x, T) { return x; }
  __device__ static V st_sr(T x, uint32_t) { return x; }
  __device__ static void ld_pp(V v, T inv_sqrt2, T& ps, T& ph) {
    ps = v;
    ph = tanh_t(ps * inv_sqrt2);
  }
  __device__ static V st_ps(T ps) { return ps; }
  __device__ static V st_ps_sr(T ps, uint32_t) { return ps; }
};
using StF32 = StPlain<float>;
using StF64 = StPlain<double>;

// 16-bit storage (split precision) keeps phi, not psi: the phase-field plane
// holds phi's distance to its nearest bulk value, with phi's sign,
//   u = copysign(1 - |phi|, phi),   phi = copysign(1 - |u|, u),
//   |psi| = sqrt2 atanh(1 - |u|) = (ln(2 - |u|) - ln|u|)/sqrt2.
// A 16-bit float keeps |u| to 11 (FP16) or 8 (BF16) significant bits, i.e. psi
// to about 3.5e-4 (FP16) or 2.8e-3 (BF16) wherever |psi| >= 1 and about twice
// that at the interface centre.  psi itself would not do: it is a signed
// distance that reaches thousands of W0 across the domain, where a 16-bit
// spacing exceeds the grid's own psi increments, and rounding noise in
// |grad psi|^2 then drives the far field toward solid.  phi is saturated to
// +-1 beyond a few W0, so psi is held to |psi| <= kPsiClamp (|u| = 0 there).
// U is stored as its offset from the far-field value U0.
constexpr float kPsiClamp = 12.5f;

template <bool BF>
struct StH16 {
  using V = unsigned short;
  using T = float;
  static constexpr bool kSR = true;
  __device__ static T ld(V v) {
    return BF ? __bfloat162float(__ushort_as_bfloat16(v)) : __half2float(__ushort_as_half(v));
  }
  __device__ static T ldU(V v, T U0) { return __fadd_rn(ld(v), U0); }
  __device__ static V st(T x) {
    return BF ? __bfloat16_as_ushort(__float2bfloat16_rn(x)) : __half_as_ushort(__float2half_rn(x));
  }
  __device__ static V stU(T x, T U0) { return st(__fsub_rn(x, U0)); }
  __device__ static V st_sr(T x, uint32_t r) { return BF ? sr_bf16_bits(x, r) : sr_fp16_bits(x, r); }
  __device__ static void ld_pp(V v, T, T& ps, T& ph) {
    const float u = ld(v), a = fabsf(u);
    ph = copysignf(1.0f - a, u);
    const float m = (a > 0.0f) ? fminf(0.70710678f * (__logf(2.0f - a) - __logf(a)), kPsiClamp)
                               : kPsiClamp;
    ps = copysignf(m, u);
  }
  // u of a psi: 1 - tanh(|psi|/sqrt2) = 2/(1 + e^(sqrt2 |psi|)), with psi's sign
  __device__ static float code(float ps) {
    const float x = fabsf(ps);
    const float a = (x >= kPsiClamp) ? 0.0f : __fdividef(2.0f, 1.0f + __expf(1.41421356f * x));
    return copysignf(a, ps);
  }
  __device__ static V st_ps(T ps) { return st(code(ps)); }
  __device__ static V st_ps_sr(T ps, uint32_t r) { return st_sr(code(ps), r); }
};
using StF16 = StH16<false>;
using StBF16 = StH16<true>;

// ---- launch arguments ------------------------------------------------------

struct EkArgs {
  const void* in;     // three planes (psi, U, dpsi), each fny rows of `pitch` values
  void* out;
  long long plane;    // values per plane
  int pitch, fnx, fny;
  int prestep;        // 1: psi update only, U unchanged (rhs_psi)
  float k, hi, Dl_tilde, eps, sqrt2, lamd, dt, cosa, sina, a_s, epsilon, a_12, U0;
  float noise_amp;    // dt_sqrt*hi*eta; 0 disables the noise term
  double up_a, up_b;  // Up of memory row j = up_a + j*up_b
  uint32_t seed, step;
};

template <class T>
struct Consts {
  T k, omk, opk, hi, hiDl_half, eps, sqrt2, inv_sqrt2, lamd, dt, cosa, sina, a_s, epsilon, a_12, U0,
      noise_amp;
};

template <class T>
__device__ __forceinline__ Consts<T> consts(const EkArgs& a) {
  Consts<T> c;
  c.k = (T)a.k;
  c.omk = (T)1 - (T)a.k;
  c.opk = (T)1 + (T)a.k;
  c.hi = (T)a.hi;
  c.hiDl_half = (T)a.hi * (T)a.Dl_tilde * (T)0.5;
  c.eps = (T)a.eps;
  c.sqrt2 = (T)a.sqrt2;
  c.inv_sqrt2 = (T)1 / (T)a.sqrt2;
  c.lamd = (T)a.lamd;
  c.dt = (T)a.dt;
  c.cosa = (T)a.cosa;
  c.sina = (T)a.sina;
  c.a_s = (T)a.a_s;
  c.epsilon = (T)a.epsilon;
  c.a_12 = (T)a.a_12;
  c.U0 = (T)a.U0;
  c.noise_amp = (T)a.noise_amp;
  return c;
}

// Math of the step.  FP64 storage uses correctly rounded double operations
// throughout.  The FP32-arithmetic storages (FP32, FP16, BF16) use the
// hardware approximations (reciprocal, reciprocal square root, 2^x; a few ulp
// each), far below the per-step differences the model's own rounding makes,
// and tanh from its exponential form tanh(x) = 1 - 2/(1 + e^(2x)) (exact limits
// +-1 at large |x|; absolute error of a few 1e-7 near 0).
template <>
__device__ __forceinline__ float tanh_t<float>(float x) {
  return 1.0f - __fdividef(2.0f, 1.0f + __expf(2.0f * x));
}
template <>
__device__ __forceinline__ double tanh_t<double>(double x) {
  return tanh(x);
}
__device__ __forceinline__ float div_t(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double div_t(double a, double b) { return a / b; }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return 1.0 / sqrt(x); }

// |phi| strictly inside the interface band, as the reference's
// (double)phi > -0.995 && (double)phi < 0.995 (PF.cu:592): for a float, that
// is |phi| < 0.995f exactly (0.995f rounds above 0.995).
__device__ __forceinline__ bool in_band(float ph) { return fabsf(ph) < 0.995f; }
__device__ __forceinline__ bool in_band(double ph) { return fabs(ph) < 0.995; }

// Anisotropy of the interface normal (phx, phz) rotated by the misorientation:
// A = atheta (PF.cu:119-131), Ap = aptheta (PF.cu:135-146).
template <class T>
__device__ __forceinline__ void aniso(T phx, T phz, const Consts<T>& c, T& A, T& Ap) {
  const T ux = c.cosa * phx + c.sina * phz;
  const T uz = c.cosa * phz - c.sina * phx;
  const T ux2 = ux * ux, uz2 = uz * uz;
  const T m = ux2 + uz2;
  if (m > c.eps) {
    const T inv = div_t((T)1, m * m);
    A = c.a_s * ((T)1 + c.epsilon * (ux2 * ux2 + uz2 * uz2) * inv);
    Ap = -c.a_12 * ux * uz * (ux2 - uz2) * inv;
  } else {
    A = (T)1;
    Ap = (T)0;
  }
}

template <class T>
__device__ __forceinline__ T aniso_a(T phx, T phz, const Consts<T>& c) {
  const T ux = c.cosa * phx + c.sina * phz;
  const T uz = c.cosa * phz - c.sina * phx;
  const T ux2 = ux * ux, uz2 = uz * uz;
  const T m = ux2 + uz2;
  if (m > c.eps) return c.a_s * ((T)1 + c.epsilon * div_t(ux2 * ux2 + uz2 * uz2, m * m));
  return (T)1;
}

template <class T>
struct Tile {
  T ps[IH][IW], ph[IH][IW], U[IH][IW], jat[IH][IW];
  T qs[TH + 1][TW + 1], qp[TH + 1][TW + 1];  // plaquette means of psi, phi
  T vJ[TH][TW + 1], vU[TH][TW + 1];          // fluxes through x-edges (i+1/2, j)
  T hJ[TH + 1][TW], hU[TH + 1][TW];          // fluxes through y-edges (i, j+1/2)
};

// Write one cell's three values at (j, i) and at every halo cell that copies it:
// column fnx-1 copies column 1 and column 0 copies column fnx-2 (periodic x),
// row 0 copies row 2 and row fny-1 copies row fny-3 (mirrored y), corners both.
template <class V>
__device__ __forceinline__ void put_with_halo(V* ps, V* U, V* D, int pitch, int fnx, int fny,
                                              int j, int i, V vps, V vU, V vD) {
  auto put = [&](int jj, int ii) {
    const long long o = (long long)jj * pitch + ii;
    ps[o] = vps;
    U[o] = vU;
    D[o] = vD;
  };
  put(j, i);
  const bool xl = (i == 1), xr = (i == fnx - 2);
  if (xl) put(j, fnx - 1);
  if (xr) put(j, 0);
  if (j == 2) {
    put(0, i);
    if (xl) put(0, fnx - 1);
    if (xr) put(0, 0);
  }
  if (j == fny - 3) {
    put(fny - 1, i);
    if (xl) put(fny - 1, fnx - 1);
    if (xr) put(fny - 1, 0);
  }
}

template <class S>
__global__ void __launch_bounds__(NTHREADS) ek2d_step_kernel(EkArgs a) {
  using T = typename S::T;
  using V = typename S::V;
  extern __shared__ __align__(16) unsigned char ek_smem[];
  Tile<T>& sm = *reinterpret_cast<Tile<T>*>(ek_smem);
  const Consts<T> c = consts<T>(a);
  const bool merge = !a.prestep;
  const V* in_ps = static_cast<const V*>(a.in);
  const V* in_U = in_ps + a.plane;
  const V* in_D = in_U + a.plane;
  const int x0 = 1 + blockIdx.x * TW;  // memory column / row of the first output cell
  const int y0 = 1 + blockIdx.y * TH;

  // ---- 0. load tile + halo; phi and the anti-trapping density per cell
  for (int e = threadIdx.x; e < IH * IW; e += NTHREADS) {
    const int r = e / IW, q = e - r * IW;
    const int gi = x0 - 1 + q, gj = y0 - 1 + r;
    T ps = 0, ph = 0, U = 0, D = 0;
    if (gi < a.fnx && gj < a.fny) {
      const long long o = (long long)gj * a.pitch + gi;
      S::ld_pp(in_ps[o], c.inv_sqrt2, ps, ph);
      U = S::ldU(in_U[o], c.U0);
      D = S::ld(in_D[o]);
    }
    sm.ps[r][q] = ps;
    sm.ph[r][q] = ph;
    sm.U[r][q] = U;
    sm.jat[r][q] = (T)0.5 * ((T)1 + c.omk * U) * ((T)1 - ph * ph) * D;
  }
  __syncthreads();

  // ---- 1. plaquette means (corner (q+1/2, r+1/2) of the input tile)
  for (int e = threadIdx.x; e < (TH + 1) * (TW + 1); e += NTHREADS) {
    const int r = e / (TW + 1), q = e - r * (TW + 1);
    sm.qs[r][q] = (((sm.ps[r][q] + sm.ps[r][q + 1]) + sm.ps[r + 1][q]) + sm.ps[r + 1][q + 1]) * (T)0.25;
    sm.qp[r][q] = (((sm.ph[r][q] + sm.ph[r][q + 1]) + sm.ph[r + 1][q]) + sm.ph[r + 1][q + 1]) * (T)0.25;
  }
  __syncthreads();

  // ---- 2. edge fluxes
  constexpr int NV = TH * (TW + 1), NHZ = (TH + 1) * TW;
  for (int e = threadIdx.x; e < NV + NHZ; e += NTHREADS) {
    if (e < NV) {
      // x-edge between input cells (b+1, q) and (b+1, q+1)
      const int b = e / (TW + 1), q = e - b * (TW + 1);
      const T psx = sm.ps[b + 1][q + 1] - sm.ps[b + 1][q];
      const T psz = sm.qs[b + 1][q] - sm.qs[b][q];
      const T phx = sm.ph[b + 1][q + 1] - sm.ph[b + 1][q];
      const T phz = sm.qp[b + 1][q] - sm.qp[b][q];
      T A, Ap;
      aniso(phx, phz, c, A, Ap);
      sm.vJ[b][q] = A * (A * psx - Ap * psz);
      if (merge) {
        const T n2 = phx * phx + phz * phz;
        const T nx = (n2 > c.eps) ? phx * rsqrt_t(n2) : (T)0;
        sm.vU[b][q] = c.hiDl_half * ((T)2 - sm.ph[b + 1][q] - sm.ph[b + 1][q + 1]) *
                          (sm.U[b + 1][q + 1] - sm.U[b + 1][q]) +
                      (T)0.5 * (sm.jat[b + 1][q] + sm.jat[b + 1][q + 1]) * nx;
      }
    } else {
      // y-edge between input cells (r, q+1) and (r+1, q+1)
      const int f = e - NV;
      const int r = f / TW, q = f - r * TW;
      const T psz = sm.ps[r + 1][q + 1] - sm.ps[r][q + 1];
      const T psx = sm.qs[r][q + 1] - sm.qs[r][q];
      const T phz = sm.ph[r + 1][q + 1] - sm.ph[r][q + 1];
      const T phx = sm.qp[r][q + 1] - sm.qp[r][q];
      T A, Ap;
      aniso(phx, phz, c, A, Ap);
      sm.hJ[r][q] = A * (A * psz + Ap * psx);
      if (merge) {
        const T n2 = phx * phx + phz * phz;
        const T nz = (n2 > c.eps) ? phz * rsqrt_t(n2) : (T)0;
        sm.hU[r][q] = c.hiDl_half * ((T)2 - sm.ph[r][q + 1] - sm.ph[r + 1][q + 1]) *
                          (sm.U[r + 1][q + 1] - sm.U[r][q + 1]) +
                      (T)0.5 * (sm.jat[r][q + 1] + sm.jat[r + 1][q + 1]) * nz;
      }
    }
  }
  __syncthreads();

  // ---- 3. cell updates
  V* o_ps = static_cast<V*>(a.out);
  V* o_U = o_ps + a.plane;
  V* o_D = o_U + a.plane;
  const uint32_t step_key = mix32(a.step ^ (a.seed * 0x9E3779B9u));
  for (int e = threadIdx.x; e < TH * TW; e += NTHREADS) {
    const int b = e / TW, q = e - b * TW;
    const int gi = x0 + q, gj = y0 + b;
    if (gi > a.fnx - 2 || gj > a.fny - 2) continue;
    const int r = b + 1, s = q + 1;  // input-tile coordinates of the cell
    const T psC = sm.ps[r][s], phC = sm.ph[r][s], UC = sm.U[r][s];
    T Un = UC;
    if (merge) {
      const T rhsU = ((sm.vU[b][q + 1] - sm.vU[b][q]) + (sm.hU[b + 1][q] - sm.hU[b][q])) * c.hi +
                     c.sqrt2 * sm.jat[r][s];
      const T tauU = c.opk - c.omk * phC;
      Un = UC + c.dt * div_t(rhsU, tauU);
    }
    const T phxn = (sm.ph[r][s + 1] - sm.ph[r][s - 1]) * (T)0.5;
    const T phzn = (sm.ph[r + 1][s] - sm.ph[r - 1][s]) * (T)0.5;
    const T psxn = (sm.ps[r][s + 1] - sm.ps[r][s - 1]) * (T)0.5;
    const T pszn = (sm.ps[r + 1][s] - sm.ps[r - 1][s]) * (T)0.5;
    T A2 = aniso_a(phxn, phzn, c);
    A2 = A2 * A2;
    const T gradps2 = psxn * psxn + pszn * pszn;
    const T extra = -c.sqrt2 * A2 * phC * gradps2;
    const T Up = (T)(a.up_a + (double)gj * a.up_b);
    const T rhs = ((sm.vJ[b][q + 1] - sm.vJ[b][q]) + (sm.hJ[b + 1][q] - sm.hJ[b][q]) + extra) * c.hi *
                      c.hi +
                  c.sqrt2 * phC - c.lamd * ((T)1 - phC * phC) * c.sqrt2 * (Un + Up);
    const T tp = (T)1 - c.omk * Up;
    const T tau = ((tp >= c.k) ? tp : c.k) * A2;
    const T dps = div_t(rhs, tau);
    T noise = (T)0;
    if (c.noise_amp != (T)0 && in_band(phC)) {
      const Philox4 rn = philox4x32_10((uint32_t)gi, (uint32_t)gj, a.step, 0x4E4F4953u, a.seed, 0x5EEDu);
      noise = c.noise_amp * ((T)uniform01(rn.v[0]) - (T)0.5);
    }
    const T psn = psC + c.dt * dps + noise;
    V vps, vU, vD;
    if (S::kSR) {
      // one 32-bit draw per cell and step: independent 10-bit fractions for psi
      // and U (1/1024 of a 16-bit spacing is ample); dpsi is rewritten from
      // scratch every step, not accumulated, so it rounds to nearest
      const uint32_t r = mix32((uint32_t)(gi + a.fnx * gj) ^ step_key);
      vps = S::st_ps_sr(psn, r & 0xFFC00000u);
      vU = merge ? S::st_sr(Un - c.U0, (r << 10) & 0xFFC00000u) : S::stU(Un, c.U0);
      vD = S::st(dps);
    } else {
      vps = S::st_ps(psn);
      vU = S::stU(Un, c.U0);
      vD = S::st(dps);
    }
    put_with_halo(o_ps, o_U, o_D, a.pitch, a.fnx, a.fny, gj, gi, vps, vU, vD);
  }
}

// ---- auxiliary kernels -------------------------------------------------------

// Reference-layout floats (psi, U, dpsi) -> storage, interior cells with their
// halo copies.  dpsi may be null (zeros).
template <class S>
__global__ void ek2d_import_kernel(const float* ps, const float* U, const float* D, void* out,
                                   long long plane, int pitch, int fnx, int fny, float U0) {
  using V = typename S::V;
  using T = typename S::T;
  const long long n = (long long)(fnx - 2) * (fny - 2);
  V* o_ps = static_cast<V*>(out);
  V* o_U = o_ps + plane;
  V* o_D = o_U + plane;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(e % (fnx - 2)), j = 1 + (int)(e / (fnx - 2));
    const long long src = (long long)j * fnx + i;
    put_with_halo(o_ps, o_U, o_D, pitch, fnx, fny, j, i, S::st_ps((T)ps[src]), S::stU((T)U[src], (T)U0),
                  S::st(D ? (T)D[src] : (T)0));
  }
}

// Storage -> reference layout (halos included) in float or double;
// phi = tanh(psi/sqrt2).
template <class S, class O>
__global__ void ek2d_export_kernel(const void* in, long long plane, int pitch, int fnx, int fny,
                                   float U0, float sqrt2, O* ps, O* ph, O* U, O* D) {
  using V = typename S::V;
  using T = typename S::T;
  const long long n = (long long)fnx * fny;
  const V* i_ps = static_cast<const V*>(in);
  const V* i_U = i_ps + plane;
  const V* i_D = i_U + plane;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % fnx), j = (int)(e / fnx);
    const long long o = (long long)j * pitch + i;
    T p, q;
    S::ld_pp(i_ps[o], (T)1 / (T)sqrt2, p, q);
    if (ps) ps[e] = (O)p;
    if (ph) ph[e] = (O)q;
    if (U) U[e] = (O)S::ldU(i_U[o], (T)U0);
    if (D) D[e] = (O)S::ld(i_D[o]);
  }
}

// Sum of phi over each row, halo columns included (one CTA per row, FP64).
template <class S>
__global__ void ek2d_row_sums_kernel(const void* in, int pitch, int fnx, float sqrt2, double* out) {
  using V = typename S::V;
  using T = typename S::T;
  const V* row = static_cast<const V*>(in) + (long long)blockIdx.x * pitch;
  double s = 0.0;
  const T inv = (T)1 / (T)sqrt2;
  for (int i = threadIdx.x; i < fnx; i += blockDim.x) {
    T p, q;
    S::ld_pp(row[i], inv, p, q);
    s += (double)q;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double warp_sums[32];
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += warp_sums[w];
    out[blockIdx.x] = t;
  }
}

// Move the frame up by `k` rows (k single-row moves of move_frame/copy_frame,
// PF.cu:625-668): row j takes row j+k; the top k rows continue the linear
// extrapolation psi_new = 2 psi[fny-2] - psi[fny-3] one row at a time, and U
// there is U0.  dpsi is not moved (the reference moves psi, phi and U only).
template <class S>
__global__ void ek2d_shift_kernel(const void* in, void* out, long long plane, int pitch, int fnx,
                                  int fny, int k, float U0) {
  using V = typename S::V;
  using T = typename S::T;
  const long long n = (long long)(fnx - 2) * (fny - 2);
  const V* i_ps = static_cast<const V*>(in);
  const V* i_U = i_ps + plane;
  const V* i_D = i_U + plane;
  V* o_ps = static_cast<V*>(out);
  V* o_U = o_ps + plane;
  V* o_D = o_U + plane;
  const V vU0 = S::stU((T)U0, (T)U0);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(e % (fnx - 2)), j = 1 + (int)(e / (fnx - 2));
    V vps, vU;
    if (j + k <= fny - 2) {
      const long long src = (long long)(j + k) * pitch + i;
      vps = i_ps[src];
      vU = i_U[src];
    } else {
      T em2, em1, q;
      S::ld_pp(i_ps[(long long)(fny - 3) * pitch + i], (T)0.70710678118654752, em2, q);
      S::ld_pp(i_ps[(long long)(fny - 2) * pitch + i], (T)0.70710678118654752, em1, q);
      const int m = j - (fny - 2 - k);
      for (int t = 0; t < m; ++t) {
        const T en = (T)2 * em1 - em2;
        em2 = em1;
        em1 = en;
      }
      vps = S::st_ps(em1);
      vU = vU0;
    }
    put_with_halo(o_ps, o_U, o_D, pitch, fnx, fny, j, i, vps, vU, i_D[(long long)j * pitch + i]);
  }
}

}  // namespace ek2d
}  // namespace cupf
