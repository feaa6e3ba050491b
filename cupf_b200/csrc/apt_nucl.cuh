// apt_nucl.cuh — nucleation of new grains (add_nucl, APTPhaseField.cu:413-536).
//
// The reference draws from a curand XORWOW state per coarse cell; here every
// decision comes from a counter-based Philox4x32-10 stream keyed on
// (seed, coarse cell, step), so the integer outcomes (which cell nucleates,
// which grain id it gets) are reproducible and identical in the CPU oracle
// (generator in philox.cuh).
#pragma once

#include "apt_storage.cuh"
#include "philox.cuh"

namespace cupf {

struct NuclArgs {
  int fnx, fny, fnz, xp;
  long long slot_stride;
  int np;
  int cnx, cny, cnz;  // coarse cells per axis
  int pts;            // pts_cell: half width of the nucleus cube
  int num_theta;      // ids of new grains start above num_theta
  int id_space;       // new ids: num_theta + 1 + (draw % id_space)
  int use_iuc;
  float uc0, nmax0, nmax, mean, std, rad, dt2, t;
  uint32_t seed;
  uint32_t step;
  const float* T_3D;  // 4-D temperature table (may be NULL: no table nucleation)
  const float *X_mac, *Y_mac, *Z_mac, *t_mac;
  const float *x, *y, *z;
  int Nx, Ny, Nz, Nt;
  const float* sphere;  // (2*pts+1)^3 nucleus profile: tanh(dx*((1+pts)/2 - r)/sqrt2)
  int* status;          // per coarse cell: 1 = solid / already nucleated
  int* count;           // nucleation events (accumulated)
  // quiet-item flags of the buffer written (NULL = none kept): the items a
  // nucleus reaches are marked not quiet; tile tw x th cells, z chunk zc
  uint8_t* quiet;
  int tw, th, zc, ntx, nty;
};

// interp4Dtemperature (devicefunc.cu_inl:32-83): quadrilinear in (x, y, z, t),
// single precision, every operation rounded separately (no fused multiply-add)
// so the CPU oracle reproduces it bit for bit.
__device__ __forceinline__ float interp4d(const float* __restrict__ u, float x, float y, float z,
                                          float t, int Nx, int Ny, int Nz, int Nt, float Dx,
                                          float Dt) {
  const float fx = __fdiv_rn(x, Dx), fy = __fdiv_rn(y, Dx), fz = __fdiv_rn(z, Dx),
              ft = __fdiv_rn(t, Dt);
  int kx = (int)fx, ky = (int)fy, kz = (int)fz, kt = (int)ft;
  float dx = __fsub_rn(fx, (float)kx), dy = __fsub_rn(fy, (float)ky);
  float dz = __fsub_rn(fz, (float)kz), dtt = __fsub_rn(ft, (float)kt);
  if (kx == Nx - 1) { kx = Nx - 2; dx = 1.0f; }
  if (ky == Ny - 1) { ky = Ny - 2; dy = 1.0f; }
  if (kz == Nz - 1) { kz = Nz - 2; dz = 1.0f; }
  if (kt == Nt - 1) { kt = Nt - 2; dtt = 1.0f; }
  kx = min(max(kx, 0), Nx - 2);
  ky = min(max(ky, 0), Ny - 2);
  kz = min(max(kz, 0), Nz - 2);
  kt = min(max(kt, 0), Nt - 2);
  const long long sx = 1, sy = Nx, sz = (long long)Nx * Ny, st = sz * Nz;
  const float ex = __fsub_rn(1.0f, dx), ey = __fsub_rn(1.0f, dy);
  const float wa = __fmul_rn(ex, ey), wb = __fmul_rn(ex, dy), wc = __fmul_rn(dx, ey),
              wd = __fmul_rn(dx, dy);
  auto quad = [&](long long o) {
    float r = __fmul_rn(wa, u[o]);
    r = __fadd_rn(r, __fmul_rn(wb, u[o + sy]));
    r = __fadd_rn(r, __fmul_rn(wc, u[o + sx]));
    return __fadd_rn(r, __fmul_rn(wd, u[o + sy + sx]));
  };
  auto tri = [&](long long o) {
    return __fadd_rn(__fmul_rn(quad(o), __fsub_rn(1.0f, dz)), __fmul_rn(quad(o + sz), dz));
  };
  const long long o = kx + ky * sy + kz * sz + kt * st;
  return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, dtt), tri(o)), __fmul_rn(dtt, tri(o + st)));
}

// Nucleation probability of a coarse cell (nuncl_possibility, APTPhaseField.cu:446-455):
// Gaussian density in the undercooling times its increment times the nucleus
// volume 8 r^3.  Evaluated in double so the decision `u < P` is the same on the
// GPU and in the CPU oracle.
__host__ __device__ inline double nucl_probability(double delT, double d_delT, double nmax,
                                                   double mean, double std, double rad) {
  const double q = (delT - mean) / std;
  const double density = nmax / (sqrt(2.0 * 3.14159265358979323846) * std) * exp(-0.5 * q * q) * d_delT;
  return 8.0 * rad * rad * rad * density;
}

// One pass over the coarse cells (add_nucl, APTPhaseField.cu:459-536): a coarse
// cell still marked liquid is re-checked at its centre (any slot above LS makes
// it solid); otherwise it nucleates with the probability above, writing a
// nucleus into slot 0 of its (2*pts+1)^3 cube with a new grain id.
template <class S>
__global__ void nucleate_kernel(typename S::T* buf, NuclArgs a) {
  const long long ncell = (long long)a.cnx * a.cny * a.cnz;
  const float kLS = __uint_as_float(kLSFloatBits);
  const float kDrop = __uint_as_float(kDropFloatBits);
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < ncell;
       C += (long long)gridDim.x * blockDim.x) {
    if (a.status[C]) continue;
    const int i = (int)(C % a.cnx), j = (int)((C / a.cnx) % a.cny), k = (int)(C / ((long long)a.cnx * a.cny));
    const int w = 2 * a.pts + 1;
    const int gi = w * i + a.pts + 1, gj = w * j + a.pts + 1, gk = w * k + a.pts + 1;
    const long long g = (long long)gk * a.xp * a.fny + (long long)gj * a.xp + gi;
    bool solid = false;
    for (int p = 0; p < a.np; ++p) solid |= S::phi(buf[p * a.slot_stride + g]) > kLS;
    if (solid) {
      a.status[C] = 1;
      continue;
    }
    double P;
    if (a.use_iuc) {
      // delT = UC0*1e6*(t+dt), d_delT = UC0*1e6*dt (APTPhaseField.cu:491-495)
      const float delT = __double2float_rn((double)a.uc0 * 1e6 * (double)__fadd_rn(a.t, a.dt2));
      const float d_delT = __double2float_rn((double)a.uc0 * 1e6 * (double)a.dt2);
      P = nucl_probability(delT, d_delT, a.nmax0, a.mean, a.std, a.rad);
    } else if (a.T_3D) {
      // delT = -T(t+dt), d_delT = T(t) - T(t+dt) from the 4-D table (:497-505)
      const float Dx = __fsub_rn(a.X_mac[1], a.X_mac[0]), Dt = __fsub_rn(a.t_mac[1], a.t_mac[0]);
      const float xq = __fsub_rn(a.x[gi], a.X_mac[0]), yq = __fsub_rn(a.y[gj], a.Y_mac[0]);
      const float zq = __fsub_rn(a.z[gk], a.Z_mac[0]);
      const float T0 = interp4d(a.T_3D, xq, yq, zq, __fsub_rn(a.t, a.t_mac[0]), a.Nx, a.Ny, a.Nz,
                                a.Nt, Dx, Dt);
      const float T1 = interp4d(a.T_3D, xq, yq, zq, __fsub_rn(__fadd_rn(a.t, a.dt2), a.t_mac[0]),
                                a.Nx, a.Ny, a.Nz, a.Nt, Dx, Dt);
      P = nucl_probability(-T1, __fsub_rn(T0, T1), a.nmax, a.mean, a.std, a.rad);
    } else {
      continue;
    }
    const Philox4 r = philox4x32_10((uint32_t)C, a.step, 0x4E55434Cu, 0u, a.seed, 0x5EEDu);
    if (!((double)uniform01(r.v[0]) < P)) continue;
    const int id = a.num_theta + 1 + (int)(r.v[1] % (uint32_t)a.id_space);
    for (int dk = -a.pts; dk <= a.pts; ++dk)
      for (int dj = -a.pts; dj <= a.pts; ++dj)
        for (int di = -a.pts; di <= a.pts; ++di) {
          const float v = a.sphere[((dk + a.pts) * w + (dj + a.pts)) * w + (di + a.pts)];
          const long long o = g + (long long)dk * a.xp * a.fny + (long long)dj * a.xp + di;
          const typename S::T old = buf[o];
          // `ph > -0.9999f` (a float literal, APTPhaseField.cu:524) == v > kDrop
          buf[o] = S::make(v, v > kDrop ? id : S::id(old));
        }
    if (a.quiet) {
      for (int qz = (gk - a.pts - 1) / a.zc; qz <= (gk + a.pts - 1) / a.zc; ++qz)
        for (int qy = (gj - a.pts - 1) / a.th; qy <= (gj + a.pts - 1) / a.th; ++qy)
          for (int qx = (gi - a.pts - 1) / a.tw; qx <= (gi + a.pts - 1) / a.tw; ++qx)
            a.quiet[((long long)qz * a.nty + qy) * a.ntx + qx] = 0;
    }
    a.status[C] = 1;
    atomicAdd(a.count, 1);
  }
}

// init_nucl_status (APTPhaseField.cu:420-444): a coarse cell starts solid when
// slot 0 at its centre is above LS.  The reference indexes that centre without
// the halo offset add_nucl uses (:429-431 vs :474-476); kept as is.
template <class S>
__global__ void nucl_status_init_kernel(const typename S::T* __restrict__ buf, NuclArgs a) {
  const long long ncell = (long long)a.cnx * a.cny * a.cnz;
  const float kLS = __uint_as_float(kLSFloatBits);
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < ncell;
       C += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(C % a.cnx), j = (int)((C / a.cnx) % a.cny), k = (int)(C / ((long long)a.cnx * a.cny));
    const int w = 2 * a.pts + 1;
    const long long g = (long long)(w * k + a.pts) * a.xp * a.fny + (long long)(w * j + a.pts) * a.xp +
                        (w * i + a.pts);
    a.status[C] = S::phi(buf[g]) > kLS ? 1 : 0;
  }
}

}  // namespace cupf
