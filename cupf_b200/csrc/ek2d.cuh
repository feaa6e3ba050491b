// ek2d.cuh — 2D Echebarria–Karma directional-solidification step (psi/U line
// model of cuPF 2DdendriteMPI/line_model/PF.cu) for sm_100a.
//
// One launch advances the whole grid by one step (ek2d_march_kernel, below):
// each warp marches up a strip of 30 columns, computing for every cell
//   - the phase field, U and dpsi of the next row (decoded: psi and
//     phi = tanh(psi/sqrt2)) and the anti-trapping flux density
//     jat = (1+(1-k)U)(1-phi^2) dpsi / 2;
//   - plaquette means of psi and phi at the cell corners (psipjp .. phimjm of
//     merge_PF, PF.cu:444-453);
//   - the fluxes through its right and upper edges: the anisotropic psi flux J
//     (atheta/aptheta, PF.cu:119-146, 475-538) and the solute flux of U with
//     its anti-trapping part (PF.cu:460-551).  Each edge is computed once and
//     shared by the two cells it separates (the reference computes it from
//     both sides);
//   - U' = U + dt*div(U flux)/tau_U (PF.cu:553-556), then the psi right-hand
//     side with the new U (PF.cu:563-590), dpsi = rhs/tau_psi,
//     psi' = psi + dt*dpsi (+ noise), and the stores.
// The reference's merge_PF (PF.cu:379-610) fuses the same U-then-psi update in
// one kernel over a 128-wide band of a linear index; the pre-loop rhs_psi
// (PF.cu:150-280) is the same psi update with U left unchanged (`prestep`).
//
// Boundary: x periodic, y mirrored about rows 1 and fny-2 (set_BC,
// PF.cu:35-73).  The reference refills the halo of the state it is about to
// read; here every writer of an interior cell that some halo cell copies also
// writes that copy, so each step's output already carries its halo.
//
// Storage S: FP32 (the reference's), FP16 / BF16 (split precision: the phase
// field (psi bounded to +-50 W0 in FP16; phi as its distance to the bulk value
// in BF16), U - U0 and dpsi in 16 bits, the phase field and U stored with
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
  __device__ static void st_ps_U_sr(T ps, T u, uint32_t, V& vps, V& vu) {
    vps = ps;
    vu = u;
  }
};
using StF32 = StPlain<float>;
using StF64 = StPlain<double>;

// 16-bit storage (split precision).  psi is a signed distance that reaches
// thousands of W0 across the domain; stored as it is in 16 bits its spacing
// there exceeds the grid's own psi increments, and rounding noise in
// |grad psi|^2 then drives the far field toward solid.  psi is therefore held
// to |psi| <= kPsiClamp = 50 W0 in the 16-bit modes: far enough that the bound
// does not reach back to the front (a bound of 12.5 W0, where phi is already
// +-1 to float precision, moved the front by about a cell in 3000 steps; 25 W0
// by 0.02 cells; 50 W0 by none measurable), and small enough that FP16 keeps a
// spacing of at most 0.03 W0 there.
//   FP16 stores psi itself (spacing 2^-11 |psi|: 5e-4 at the interface centre,
//   4e-3 at |psi| = 4-8).
//   BF16, with 8 significant bits, stores phi as its distance to the nearest
//   bulk value, with phi's sign,
//     u = copysign(1 - |phi|, phi),   phi = copysign(1 - |u|, u),
//     |psi| = sqrt2 atanh(1 - |u|) = (ln(2 - |u|) - ln|u|)/sqrt2,
//   which keeps psi to about 2.8e-3 everywhere (BF16 has FP32's exponent range,
//   so u of |psi| = 50, 4e-31, is representable).
// U is stored as its offset from the far-field value U0.
constexpr float kPsiClamp = 50.0f;

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
  // stochastic rounding by the hardware conversion (cvt.rs): x with r[31:16]
  __device__ static uint32_t sr2(T hi, T lo, uint32_t r) {
    return BF ? sr_pack_bf16x2(hi, lo, r) : sr_pack_fp16x2(hi, lo, r);
  }
  __device__ static V st_sr(T x, uint32_t r) { return (V)(sr2(x, 0.0f, r) >> 16); }
  __device__ static void ld_pp(V v, T inv_sqrt2, T& ps, T& ph) {
    if (!BF) {
      ps = ld(v);
      ph = tanh_t(ps * inv_sqrt2);
      return;
    }
    const float u = ld(v), a = fabsf(u);
    ph = copysignf(1.0f - a, u);
    const float m = (a > 0.0f) ? fminf(0.70710678f * (__logf(2.0f - a) - __logf(a)), kPsiClamp)
                               : kPsiClamp;
    ps = copysignf(m, u);
  }
  // the stored value of a psi: psi bounded to +-kPsiClamp (FP16), or its u:
  // 1 - tanh(|psi|/sqrt2) = 2/(1 + e^(sqrt2 |psi|)) with psi's sign (BF16)
  __device__ static float code(float ps) {
    const float x = fminf(fabsf(ps), kPsiClamp);
    if (!BF) return copysignf(x, ps);
    return copysignf(__fdividef(2.0f, 1.0f + __expf(1.41421356f * x)), ps);
  }
  __device__ static V st_ps(T ps) { return st(code(ps)); }
  __device__ static V st_ps_sr(T ps, uint32_t r) { return st_sr(code(ps), r); }
  // the phase field's code and U - U0 in one conversion: r[31:16] round the
  // first, r[15:0] the second
  __device__ static void st_ps_U_sr(T ps, T u, uint32_t r, V& vps, V& vu) {
    const uint32_t d = sr2(code(ps), u, r);
    vps = (V)(d >> 16);
    vu = (V)(d & 0xFFFFu);
  }
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
  int rows;           // output rows each warp marches over
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

// Fluxes through one cell edge, from the differences across it (normal) and
// along it (tangential, from the plaquette means at its two ends), and the
// values of the two cells it separates (a below/left, b above/right):
// J = A (A dpsi_n -+ Ap dpsi_t), the anisotropic psi flux of merge_PF
// (PF.cu:475-538), and Uf, the solute flux with its anti-trapping part
// (PF.cu:460-551).  kY selects the y-edge form (normal = z).
template <bool kY, class T>
__device__ __forceinline__ void edge_flux(const Consts<T>& c, bool merge, T psx, T psz, T phx,
                                          T phz, T pha, T phb, T Ua, T Ub, T ja, T jb, T& J,
                                          T& Uf) {
  T A, Ap;
  aniso(phx, phz, c, A, Ap);
  J = kY ? A * (A * psz + Ap * psx) : A * (A * psx - Ap * psz);
  if (merge) {
    const T n2 = phx * phx + phz * phz;
    const T nn = (n2 > c.eps) ? (kY ? phz : phx) * rsqrt_t(n2) : (T)0;
    Uf = c.hiDl_half * ((T)2 - pha - phb) * (Ub - Ua) + (T)0.5 * (ja + jb) * nn;
  }
}

template <class T>
__device__ __forceinline__ T jat_of(const Consts<T>& c, T U, T ph, T D) {
  return (T)0.5 * ((T)1 + c.omk * U) * ((T)1 - ph * ph) * D;
}

// One cell's update and stores (PF.cu:553-598): U' from the divergence of the
// solute fluxes, then psi' with the new U, dpsi = rhs/tau_psi, the optional
// noise term, and the stores with their halo copies.
template <class S, class T = typename S::T, class V = typename S::V>
__device__ __forceinline__ void cell_update(const EkArgs& a, const Consts<T>& c, bool merge,
                                            uint32_t step_key, int gi, int gj, T psC, T phC, T UC,
                                            T jatC, T JR, T JL, T JT, T JB, T UR, T UL, T UT, T UB,
                                            T phR, T phL, T phT, T phB, T psR, T psL, T psT,
                                            T psB, V* o_ps, V* o_U, V* o_D) {
  T Un = UC;
  if (merge) {
    const T rhsU = ((UR - UL) + (UT - UB)) * c.hi + c.sqrt2 * jatC;
    const T tauU = c.opk - c.omk * phC;
    Un = UC + c.dt * div_t(rhsU, tauU);
  }
  const T phxn = (phR - phL) * (T)0.5;
  const T phzn = (phT - phB) * (T)0.5;
  const T psxn = (psR - psL) * (T)0.5;
  const T pszn = (psT - psB) * (T)0.5;
  T A2 = aniso_a(phxn, phzn, c);
  A2 = A2 * A2;
  const T gradps2 = psxn * psxn + pszn * pszn;
  const T extra = -c.sqrt2 * A2 * phC * gradps2;
  const T Up = (T)(a.up_a + (double)gj * a.up_b);
  const T rhs = ((JR - JL) + (JT - JB) + extra) * c.hi * c.hi + c.sqrt2 * phC -
                c.lamd * ((T)1 - phC * phC) * c.sqrt2 * (Un + Up);
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
    // one 32-bit draw per cell and step: its two 16-bit halves round the
    // phase field and U independently; dpsi is rewritten from scratch every
    // step, not accumulated, so it rounds to nearest
    const uint32_t r = mix32((uint32_t)(gi + a.fnx * gj) ^ step_key);
    if (merge) {
      S::st_ps_U_sr(psn, Un - c.U0, r, vps, vU);
    } else {
      vps = S::st_ps_sr(psn, r);
      vU = S::stU(Un, c.U0);
    }
    vD = S::st(dps);
  } else {
    vps = S::st_ps(psn);
    vU = S::stU(Un, c.U0);
    vD = S::st(dps);
  }
  put_with_halo(o_ps, o_U, o_D, a.pitch, a.fnx, a.fny, gj, gi, vps, vU, vD);
}

// ---- register-marching step kernel ------------------------------------------
//
// A warp owns a strip of MW = 30 output columns: lane l holds column x0-1+l, so
// lanes 0 and 31 carry the strip's halo columns.  The warp marches up a.rows
// output rows, keeping three rows of its own column (r-1, r, r+1) and two of its right
// neighbour (r, r+1) in registers; the left neighbour's values, plaquette means
// and x-edge fluxes come by warp shuffle.  Each edge flux is computed once: a
// lane computes the x-edge on its right and the y-edge above it, the y-edge
// below it was computed in the previous row.  The next row's loads are issued a
// row ahead of their use.  No shared memory, no barriers.
constexpr int MW = 30;
constexpr int MWARPS = 8;

template <class S>
__global__ void __launch_bounds__(MWARPS * 32) ek2d_march_kernel(EkArgs a) {
  using T = typename S::T;
  using V = typename S::V;
  const Consts<T> c = consts<T>(a);
  const bool merge = !a.prestep;
  const V* in_ps = static_cast<const V*>(a.in);
  const V* in_U = in_ps + a.plane;
  const V* in_D = in_U + a.plane;
  V* o_ps = static_cast<V*>(a.out);
  V* o_U = o_ps + a.plane;
  V* o_D = o_U + a.plane;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int x0 = 1 + (blockIdx.x * MWARPS + warp) * MW;  // first output column of the strip
  if (x0 > a.fnx - 2) return;                              // whole warp: uniform
  const int gi = x0 - 1 + lane;
  const bool col_ok = gi < a.fnx;
  const bool out_col = lane >= 1 && lane <= MW && gi <= a.fnx - 2;
  const int y0 = 1 + blockIdx.y * a.rows;
  const uint32_t step_key = mix32(a.step ^ (a.seed * 0x9E3779B9u));

  // raw values of the next row to decode, loaded one row ahead of their use so
  // that the load latency overlaps the current row's arithmetic
  V raw_ps{}, raw_U{}, raw_D{};
  bool raw_ok = false;
  auto issue = [&](int r) {
    raw_ok = col_ok && r < a.fny;
    if (raw_ok) {
      const long long o = (long long)r * a.pitch + gi;
      raw_ps = in_ps[o];
      raw_U = in_U[o];
      raw_D = in_D[o];
    }
  };
  auto load = [&](T& ps, T& ph, T& U, T& jat) {
    ps = ph = U = jat = (T)0;
    if (raw_ok) {
      S::ld_pp(raw_ps, c.inv_sqrt2, ps, ph);
      U = S::ldU(raw_U, c.U0);
      jat = jat_of(c, U, ph, S::ld(raw_D));
    }
  };
  auto right = [&](T v) { return __shfl_down_sync(FULL, v, 1); };
  auto left = [&](T v) { return __shfl_up_sync(FULL, v, 1); };

  // row r+1 ("c") and its right neighbour; row r ("b"); row r-1 ("a")
  T ps_c, ph_c, U_c, j_c, Rps_c, Rph_c, RU_c, Rj_c;
  T ps_b, ph_b, U_b, j_b, Rps_b, Rph_b, RU_b, Rj_b;
  T ps_a, ph_a;
  auto fetch_c = [&]() {  // decode the issued row into "c"
    load(ps_c, ph_c, U_c, j_c);
    Rps_c = right(ps_c);
    Rph_c = right(ph_c);
    RU_c = right(U_c);
    Rj_c = right(j_c);
  };
  auto shift = [&]() {
    ps_a = ps_b;
    ph_a = ph_b;
    ps_b = ps_c; ph_b = ph_c; U_b = U_c; j_b = j_c;
    Rps_b = Rps_c; Rph_b = Rph_c; RU_b = RU_c; Rj_b = Rj_c;
  };
  // plaquette means at (x+1/2, r+1/2) from rows b and c
  auto plaq = [&](T& qs, T& qp) {
    qs = (((ps_b + Rps_b) + ps_c) + Rps_c) * (T)0.25;
    qp = (((ph_b + Rph_b) + ph_c) + Rph_c) * (T)0.25;
  };
  // y-edge (x, r+1/2) between rows b and c
  auto yedge = [&](T qs, T qp, T& J, T& Uf) {
    const T Lqs = left(qs), Lqp = left(qp);
    edge_flux<true>(c, merge, qs - Lqs, ps_c - ps_b, qp - Lqp, ph_c - ph_b, ph_b, ph_c, U_b, U_c,
                    j_b, j_c, J, Uf);
  };

  issue(y0 - 1);
  fetch_c();
  shift();
  issue(y0);
  fetch_c();
  issue(y0 + 1);
  T qs_hi, qp_hi;
  plaq(qs_hi, qp_hi);
  T yJ_hi, yU_hi = (T)0;
  yedge(qs_hi, qp_hi, yJ_hi, yU_hi);

  for (int t = 0; t < a.rows; ++t) {
    const int r = y0 + t;
    if (r > a.fny - 2) break;  // uniform across the warp
    shift();
    fetch_c();      // row r+1, issued one row earlier
    issue(r + 2);   // in flight during this row's arithmetic
    const T qs_lo = qs_hi, qp_lo = qp_hi;
    plaq(qs_hi, qp_hi);
    // x-edge (x+1/2, r)
    T xJ, xU = (T)0;
    edge_flux<false>(c, merge, Rps_b - ps_b, qs_hi - qs_lo, Rph_b - ph_b, qp_hi - qp_lo, ph_b, Rph_b,
                     U_b, RU_b, j_b, Rj_b, xJ, xU);
    const T yJ_lo = yJ_hi, yU_lo = yU_hi;
    yedge(qs_hi, qp_hi, yJ_hi, yU_hi);
    const T xJ_L = left(xJ), xU_L = left(xU);
    const T Lps = left(ps_b), Lph = left(ph_b);
    if (out_col)
      cell_update<S>(a, c, merge, step_key, gi, r, ps_b, ph_b, U_b, j_b, xJ, xJ_L, yJ_hi, yJ_lo, xU,
                     xU_L, yU_hi, yU_lo, Rph_b, Lph, ph_c, ph_a, Rps_b, Lps, ps_c, ps_a, o_ps, o_U,
                     o_D);
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
