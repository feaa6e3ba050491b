// apt_update.cuh — per-slot explicit update of the APT step (single precision).
//
// Restates the arithmetic of APTrhs_psi (3DgrainMPI/APTPhaseField.cu:254-348),
// kine_ani (:36-52) and the thermal models (:278-327, devicefunc.cu_inl:85-125).
// Every operation is written with an explicit rounding intrinsic, so nvcc
// cannot fuse anything on its own: the sites where the reference's build fuses
// a product into a sum (nvcc's default -fmad=true) are chosen by the Contract
// constants below, which are pinned bit-for-bit against the reference kernels
// compiled for sm_100a.  Site order and meaning match oracle/apt_oracle.c.
#pragma once

#include <type_traits>

#include "apt_common.cuh"

namespace cupf {

struct Contract {
  // 0 = separate multiply and add, 1 = fuse the left product, 2 = fuse the right one.
  // Pinned: with these choices every step of the reference kernels recorded on a
  // B200 is reproduced bit for bit (AS and TD are indistinguishable on those
  // inputs and keep the compiler's usual left fusion).
  static constexpr int AS = 1, UX_IN = 1, UX_OUT = 1, UY = 2, UZ_IN = 1, UZ_OUT = 1,
                       MAG_IN = 0, MAG_OUT = 0, Q_IN = 2, Q_OUT = 1, DIFF = 1, REP = 1, W = 1,
                       E1 = 2, INNER = 1, RHS = 1, NEW = 1, TD = 1;
};

// The full-PF kernel (PhaseField.cu:168-301), pinned the same way against its own
// dumps: the sums of its rotation (X/Y/Z, PhaseField.cu:37-44) and, of the sums it
// shares in shape with the APT kernel, the quartic and E1 sums fused on the other
// side.
struct ContractFull : Contract {
  static constexpr int Q_IN = 1, E1 = 1;
  static constexpr int X_IN = 2, X_OUT = 1, Y_IN = 2, Y_OUT = 1, Z_OUT = 1;
};

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// x*y + u*v under contraction mode M
template <int M>
__device__ __forceinline__ float sop(float x, float y, float u, float v) {
  if (M == 1) return ffma(x, y, fmul(u, v));
  if (M == 2) return ffma(u, v, fmul(x, y));
  return fadd(fmul(x, y), fmul(u, v));
}

// a_s = 1 + 3 kd and epsilon = -4 kd / a_s of kine_ani (APTPhaseField.cu:38-39),
// which depend only on the launch's kin_delta: formed once per work item with
// the same operations the reference repeats per call.
struct KineConst {
  float a_s, epsilon;
};
__device__ __forceinline__ KineConst kine_const(float kd) {
  using K = Contract;
  KineConst k;
  k.a_s = K::AS ? ffma(3.0f, kd, 1.0f) : fadd(1.0f, fmul(3.0f, kd));
  k.epsilon = __fdiv_rn(fmul(-4.0f, kd), k.a_s);
  return k;
}

// Normal rotated into the grain frame.  APT kernel (APTPhaseField.cu:41-46):
//   ( ca*cb*ux + sa*cb*uy - sb*uz,  -sa*ux + ca*uy + 0,  ca*sb*ux + sa*sb*uy + cb*uz );
// full-PF kernel (kFull, PhaseField.cu:37-44), a different rotation:
//   ( ca*cb*ux + sa*uy + ca*sb*uz,  -sa*cb*ux + ca*uy - sa*sb*uz,  -sb*ux + 0 + cb*uz ).
template <bool kFull>
__device__ __forceinline__ void rotate_normal(float ux, float uy, float uz, float cosa, float sina,
                                              float cosb, float sinb, float& rx, float& ry,
                                              float& rz) {
  if (!kFull) {
    using K = Contract;
    float s = sop<K::UX_IN>(fmul(cosa, cosb), ux, fmul(sina, cosb), uy);
    rx = K::UX_OUT ? ffma(-sinb, uz, s) : fsub(s, fmul(sinb, uz));
    ry = fadd(sop<K::UY>(-sina, ux, cosa, uy), 0.0f);
    s = sop<K::UZ_IN>(fmul(cosa, sinb), ux, fmul(sina, sinb), uy);
    rz = K::UZ_OUT ? ffma(cosb, uz, s) : fadd(s, fmul(cosb, uz));
  } else {
    using K = ContractFull;
    float s = sop<K::X_IN>(fmul(cosa, cosb), ux, sina, uy);
    rx = K::X_OUT ? ffma(fmul(cosa, sinb), uz, s) : fadd(s, fmul(fmul(cosa, sinb), uz));
    s = sop<K::Y_IN>(fmul(-sina, cosb), ux, cosa, uy);
    ry = K::Y_OUT ? ffma(-fmul(sina, sinb), uz, s) : fsub(s, fmul(fmul(sina, sinb), uz));
    s = fadd(fmul(-sinb, ux), 0.0f);
    rz = K::Z_OUT ? ffma(cosb, uz, s) : fadd(s, fmul(cosb, uz));
  }
}

// 4-fold kinetic anisotropy of the rotated normal (APTPhaseField.cu:36-52,
// PhaseField.cu:32-50).
template <bool kFull = false>
__device__ __forceinline__ float kine_ani(float ux, float uy, float uz, float cosa, float sina,
                                          float cosb, float sinb, KineConst kc, float eps) {
  using K = typename std::conditional<kFull, ContractFull, Contract>::type;
  const float a_s = kc.a_s, epsilon = kc.epsilon;
  float rx, ry, rz;
  rotate_normal<kFull>(ux, uy, uz, cosa, sina, cosb, sinb, rx, ry, rz);
  float ux2 = fmul(rx, rx), uy2 = fmul(ry, ry), uz2 = fmul(rz, rz);
  float mag = sop<K::MAG_IN>(rx, rx, ry, ry);
  mag = K::MAG_OUT ? ffma(rz, rz, mag) : fadd(mag, uz2);
  float mag2 = fmul(mag, mag);
  if (mag > eps) {
    float q = sop<K::Q_IN>(ux2, ux2, uy2, uy2);
    q = K::Q_OUT ? ffma(uz2, uz2, q) : fadd(q, fmul(uz2, uz2));
    return fmul(a_s, fadd(1.0f, __fdiv_rn(fmul(epsilon, q), mag2)));
  }
  return 1.0f;
}

// interp3Dtemperature (devicefunc.cu_inl:85-125).
__device__ __forceinline__ float interp3d(const float* __restrict__ u, float x, float y, float z,
                                          int Nx, int Ny, int Nz, float Dx) {
  int kx = (int)__fdiv_rn(x, Dx), ky = (int)__fdiv_rn(y, Dx), kz = (int)__fdiv_rn(z, Dx);
  float dx = fsub(__fdiv_rn(x, Dx), (float)kx);
  float dy = fsub(__fdiv_rn(y, Dx), (float)ky);
  float dz = fsub(__fdiv_rn(z, Dx), (float)kz);
  if (kx == Nx - 1) { kx = Nx - 2; dx = 1.0f; }
  if (ky == Ny - 1) { ky = Ny - 2; dy = 1.0f; }
  if (kz == Nz - 1) { kz = Nz - 2; dz = 1.0f; }
  long long o = kx + (long long)ky * Nx + (long long)kz * Nx * Ny;
  long long on = kx + (long long)ky * Nx + (long long)(kz + 1) * Nx * Ny;
  float a = fmul(fsub(1.0f, dx), fsub(1.0f, dy)), b = fmul(fsub(1.0f, dx), dy);
  float c = fmul(dx, fsub(1.0f, dy)), d = fmul(dx, dy);
  // the reference's build fuses the first pair of the two brackets on opposite
  // sides (pinned on dumps of the paraboloid case): lower a*u0 + b*u1 fuses the
  // right product, upper the left one; the rest of each sum and the z blend fuse
  // as written left to right
  float p0 = ffma(b, __ldg(u + o + Nx), fmul(a, __ldg(u + o)));
  p0 = ffma(c, __ldg(u + o + 1), p0);
  p0 = ffma(d, __ldg(u + o + Nx + 1), p0);
  float p1 = ffma(a, __ldg(u + on), fmul(b, __ldg(u + on + Nx)));
  p1 = ffma(c, __ldg(u + on + 1), p1);
  p1 = ffma(d, __ldg(u + on + Nx + 1), p1);
  return ffma(p0, fsub(1.0f, dz), fmul(p1, dz));
}

// Undercooling at (i,j,k) and time t (APTPhaseField.cu:278-327).  Returns false
// where the reference skips the update (`continue`: the slot keeps what the
// output buffer already holds).
// The thermal models with time and height in FP64 (16-bit storage): the same
// formulas as tinterp below, every product and sum in double, the coordinates
// x, y (fixed, exact in float) promoted and z from the FP64 copy; the
// trilinear table lookup of thermalType 4 interpolates the float table at the
// double coordinates rounded to float.
__device__ __forceinline__ bool tinterp64(const StepArgs& a, int i, int j, int k, float* T) {
  const double t = a.t64;
  const double uct = (double)a.uc * 1e6 * t;
  if (a.use_iuc) {
    *T = (float)(-(double)a.uc0 * 1e6 * t);
    return true;
  }
  const double z = a.z64[k];
  if (a.thermalType == 1) {
    *T = (float)((double)a.G * (z - (double)a.z0) - uct);
    return true;
  }
  if (a.thermalType == 2) {
    const double u = (double)__ldg(a.y + j) - 0.5 * (double)a.lyd;
    const double v = z - (double)a.z0 - (double)a.lzd;
    *T = (float)(-(double)a.G * (sqrt(u * u + v * v) - (double)a.r0) - uct);
    return true;
  }
  if (a.thermalType == 3) {
    const double lm = ((double)a.r0 - (double)a.z0) / tan((double)a.angle);
    const double xl = (double)__ldg(a.x + i);
    const double r0x = (double)a.z0 + ((double)a.r0 - (double)a.z0) * xl / lm;
    const double u = (double)__ldg(a.y + j) - 0.5 * (double)a.lyd;
    const double zt = (double)a.z0 + (double)a.lzd - z;
    const double dist = cos((double)a.angle) * (sqrt(zt * zt + u * u) - r0x);
    if (xl > (double)a.V * 1e6 * t + lm) return false;
    *T = (float)(-(double)a.G * dist - uct);
    return true;
  }
  if (a.thermalType == 5) {
    const double xi = (double)a.x0 + (double)a.V * 1e6 * t - (double)__ldg(a.x + i);
    const double u = (double)__ldg(a.y + j) - 0.5 * (double)a.lyd;
    const double w = (double)a.z0 + (double)a.lzd - z;
    const double rr = u * u + w * w;
    double dist;
    if (xi <= 0.0) dist = sqrt(rr + xi * xi) - (double)a.r0;
    else if (xi < (double)a.mp_len) dist = sqrt(rr) - (double)a.r0 * sqrt(1.0 - xi / (double)a.mp_len);
    else dist = sqrt(rr);
    *T = (float)(-(double)a.G * dist - uct);
    return true;
  }
  if (a.thermalType == 4) {
    const double xq = (double)__ldg(a.x + i) - (double)a.V * 1e6 * t;
    if (xq > (double)a.mp_len + (double)a.x0 || xq < 0.0) return false;
    const float Dx = fsub(__ldg(a.X_mac + 1), __ldg(a.X_mac));
    const float v = interp3d(a.psi_mac, (float)(xq - (double)__ldg(a.X_mac)),
                             (float)((double)__ldg(a.y + j) - (double)__ldg(a.Y_mac)),
                             (float)(z - (double)__ldg(a.Z_mac)), a.Nx, a.Ny, a.Nz, Dx);
    *T = (a.order == 100.0f) ? -v : (float)(-(double)a.G * (double)v);
    return true;
  }
  *T = 0.0f;
  return true;
}

__device__ __forceinline__ bool tinterp(const StepArgs& a, int i, int j, int k, float* T) {
  if (a.fp64) return tinterp64(a, i, j, k, T);
  const float t = a.t;
  if (a.use_iuc) {
    *T = __double2float_rn(__dmul_rn(__dmul_rn((double)(-a.uc0), 1e6), (double)t));
    return true;
  }
  if (a.thermalType == 1) {
    float g = fmul(a.G, fsub(__ldg(a.z + k), a.z0));
    double m = __dmul_rn((double)a.uc, 1e6);
    double r = Contract::TD ? __fma_rn(-m, (double)t, (double)g)
                            : __dsub_rn((double)g, __dmul_rn(m, (double)t));
    *T = __double2float_rn(r);
    return true;
  }
  if (a.thermalType == 2) {
    float u = fsub(__ldg(a.y + j), fmul(0.5f, a.lyd));
    float v = fsub(fsub(__ldg(a.z + k), a.z0), a.lzd);
    float dist = fsub(__fsqrt_rn(ffma(u, u, fmul(v, v))), a.r0);
    double m = __dmul_rn((double)a.uc, 1e6);
    *T = __double2float_rn(__fma_rn(-m, (double)t, (double)fmul(-a.G, dist)));
    return true;
  }
  if (a.thermalType == 3) {
    float lm = __fdiv_rn(fsub(a.r0, a.z0), tanf(a.angle));
    float xl = fsub(__ldg(a.x + i), 0.0f);
    float r0x = fadd(a.z0, __fdiv_rn(fmul(fsub(a.r0, a.z0), xl), lm));
    float u = fsub(__ldg(a.y + j), fmul(0.5f, a.lyd));
    float zt = fsub(fadd(a.z0, a.lzd), __ldg(a.z + k));
    float dist = fmul(cosf(a.angle), fsub(__fsqrt_rn(ffma(zt, zt, fmul(u, u))), r0x));
    if ((double)xl > __fma_rn((double)fmul(a.V, t), 1e6, (double)lm)) return false;
    double m = __dmul_rn((double)a.uc, 1e6);
    *T = __double2float_rn(__fma_rn(-m, (double)t, (double)fmul(-a.G, dist)));
    return true;
  }
  if (a.thermalType == 4) {
    float xq = __double2float_rn(
        __dsub_rn((double)__ldg(a.x + i), __dmul_rn((double)fmul(a.V, t), 1e6)));
    if (xq > fadd(a.mp_len, a.x0) || xq < 0.0f) return false;
    float Dx = fsub(__ldg(a.X_mac + 1), __ldg(a.X_mac));
    float v = interp3d(a.psi_mac, fsub(xq, __ldg(a.X_mac)), fsub(__ldg(a.y + j), __ldg(a.Y_mac)),
                       fsub(__ldg(a.z + k), __ldg(a.Z_mac)), a.Nx, a.Ny, a.Nz, Dx);
    *T = (a.order == 100.0f) ? -v : fmul(-a.G, v);
    return true;
  }
  if (a.thermalType == 5) {
    // analytic paraboloid melt pool (no counterpart in the reference, which
    // tabulates its pool, thermalType 4): a beam at x_b = x0 + V 1e6 t moving in
    // +x along the axis y = lyd/2, z = z0 + lzd; behind it the pool's radius
    // about the axis is R = r0 sqrt(1 - xi/mp_len) at distance xi, ahead of it
    // the pool ends in a hemisphere of radius r0; dist = distance from the axis
    // minus R (the axis itself past the tail), T = -G dist - UC 1e6 t as the cone
    const float xb = __double2float_rn(
        __dadd_rn((double)a.x0, __dmul_rn((double)fmul(a.V, t), 1e6)));
    const float xi = fsub(xb, __ldg(a.x + i));
    const float u = fsub(__ldg(a.y + j), fmul(0.5f, a.lyd));
    const float w = fsub(fadd(a.z0, a.lzd), __ldg(a.z + k));
    const float rr = fadd(fmul(u, u), fmul(w, w));
    float dist;
    if (xi <= 0.0f) dist = fsub(__fsqrt_rn(fadd(rr, fmul(xi, xi))), a.r0);
    else if (xi < a.mp_len)
      dist = fsub(__fsqrt_rn(rr), fmul(a.r0, __fsqrt_rn(fsub(1.0f, __fdiv_rn(xi, a.mp_len)))));
    else dist = __fsqrt_rn(rr);
    const double m = __dmul_rn((double)a.uc, 1e6);
    *T = __double2float_rn(__dsub_rn((double)fmul(-a.G, dist), __dmul_rn(m, (double)t)));
    return true;
  }
  *T = 0.0f;
  return true;
}

// New phi of one active slot (APTPhaseField.cu:254-340; the full-PF kernel's
// PhaseField.cu:195-297 is the same arithmetic with its own rotation, kFull).
// ph[0..6] are the slot's values at D,B,L,C,R,T,U; repul the repulsion sum;
// Up = T/L_cp.  A: launch arguments with eps, hi, lamd and dt.
template <bool kFull = false, class A>
__device__ __forceinline__ float slot_update(const A& a, KineConst kc, const float ph[7],
                                             float sina, float cosa, float sinb, float cosb,
                                             float repul, float Up) {
  using K = typename std::conditional<kFull, ContractFull, Contract>::type;
  const float phD = ph[0], phB = ph[1], phL = ph[2], phC = ph[3], phR = ph[4], phT = ph[5],
              phU = ph[6];
  float phx = fmul(fsub(phR, phL), 0.5f);
  float phy = fmul(fsub(phT, phB), 0.5f);
  float phz = fmul(fsub(phU, phD), 0.5f);
  float A2 = kine_ani<kFull>(phx, phy, phz, cosa, sina, cosb, sinb, kc, a.eps);
  float sum = fadd(fadd(fadd(fadd(fadd(phR, phL), phT), phB), phU), phD);
  float diff = K::DIFF ? ffma(-6.0f, phC, sum) : fsub(sum, fmul(6.0f, phC));
  float w = K::W ? ffma(-phC, phC, 1.0f) : fsub(1.0f, fmul(phC, phC));
  float dh = fmul(diff, a.hi);
  float E1 = sop<K::E1>(dh, a.hi, w, phC);
  float m6 = fmul(6.0f, fadd(phC, 1.0f));
  float inner;
  if (K::INNER == 1) inner = ffma(w, w, -fmul(m6, repul));
  else if (K::INNER == 2) inner = ffma(-m6, repul, fmul(w, w));
  else inner = fsub(fmul(w, w), fmul(m6, repul));
  float lu = fmul(a.lamd, Up);
  float rhs = K::RHS ? ffma(-lu, inner, E1) : fsub(E1, fmul(lu, inner));
  float dphi = __fdiv_rn(rhs, A2);
  return K::NEW ? ffma(a.dt, dphi, phC) : fadd(phC, fmul(a.dt, dphi));
}

__device__ __forceinline__ float repul_add(float repul, float phc) {
  float q = fadd(phc, 1.0f);
  return Contract::REP ? ffma(fmul(0.25f, q), q, repul) : fadd(repul, fmul(fmul(0.25f, q), q));
}

}  // namespace cupf
