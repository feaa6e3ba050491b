// dense.cuh — kernels of the full (non-APT) phase-field mode: one phi field per
// grain, phi[grain][z][y][x] in float (the reference's layout, PhaseField.cu).
//
// Each buffer has per-cell lists: the grains whose phi differs from -1 at the
// cell, ascending, with their values (capacity K per cell; the count is stored in
// full so a longer list is detected).  A step is one launch:
//   dense_update_kernel  per interior cell: the grains the output buffer's lists
//                        name (its content of two steps ago) are reset to -1, then
//                        the reference's update (rhs_psi, PhaseField.cu:168-301) is
//                        evaluated for each grain in the union of the seven stencil
//                        cells' lists of the input buffer, with the repulsion summed
//                        over the centre list in ascending grain order; the results
//                        that differ from -1 form the output buffer's new lists.
// Every grain outside that union is exactly -1 at all seven stencil points; its
// update is exactly -1 and its repulsion term exactly zero, so skipping them
// reproduces the reference's floats while the step touches only the grains present
// near each cell.  A cell whose stencil meets a list longer than K is evaluated
// from the phi buffer over every grain instead.  dense_list_kernel builds the lists
// of a buffer from scratch (one read of every grain) after the state is replaced
// (init, set_slots, moving frame); while a buffer's lists are not valid the step
// resets all of its grains.
//
// Boundary: set_BC_3D (PhaseField.cu:111-166) mirrors every face (halo 0 takes
// cell 2, halo fn-1 takes cell fn-3) whatever the -b digits; the update reads
// neighbours through that map, so the halo of the buffer being read is never
// needed by the step, and is filled only before read-back, argmax and tip scan.
#pragma once

#include "apt_aux.cuh"
#include "apt_update.cuh"

namespace cupf {

constexpr int kDenseListMax = 16;

// phi-only storage for the shared halo / layer-sum / copy kernels of apt_aux.cuh
struct DensePhi {
  using T = float;
  __host__ __device__ static float phi(float v) { return v; }
};

struct DenseArgs {
  int fnx, fny, fnz, np, K;
  long long len;   // cells per grain field = fnx*fny*fnz
  float t;         // physical time of the step (s)
  double Rm;       // R * 1e6 (double, exact)
  float G, L_cp, hi, lamd, dt, eps, kin_delta;
  const float* z;
  const float4* orient;  // pack_orientations: entry g+1 is grain g
  const float* in;
  float* out;
  const int* cnt;             // lists of `in`: [len] length (may exceed K)
  const unsigned short* lid;  // [K][len] grain of list entry
  const float* lval;          // [K][len] its phi
  int* cnt_o;                 // lists of `out`: read for the reset, then rewritten
  unsigned short* lid_o;
  float* lval_o;
  int reset_from_lists;       // 1: out's lists are valid (reset only the grains they name)
  unsigned long long* overflow;  // cells evaluated over every grain this step
};

__device__ __forceinline__ int mirror(int c, int fn) {
  return c == 0 ? 2 : (c == fn - 1 ? fn - 3 : c);
}

// Per interior cell: grains with phi != -1, ascending.
__global__ void dense_list_kernel(const float* __restrict__ ph, int fnx, int fny, int fnz, int np,
                                  int K, long long len, int* cnt, unsigned short* lid,
                                  float* lval) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > fnx - 2 || j > fny - 2) return;
  const long long C = i + (long long)fnx * (j + (long long)fny * k);
  int c = 0;
  int q = 0;
  for (; q + 4 <= np; q += 4) {
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = __ldg(ph + (q + u) * len + C);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (v[u] != -1.0f) {
        if (c < K) {
          lid[c * len + C] = (unsigned short)(q + u);
          lval[c * len + C] = v[u];
        }
        ++c;
      }
  }
  for (; q < np; ++q) {
    const float v = __ldg(ph + q * len + C);
    if (v != -1.0f) {
      if (c < K) {
        lid[c * len + C] = (unsigned short)q;
        lval[c * len + C] = v;
      }
      ++c;
    }
  }
  cnt[C] = c;
}

// Line undercooling of the full-PF kernel, Up = G*(z - R*1e6*t - 2) / L_cp
// (PhaseField.cu:277-278): the bracket in double, as the reference's double
// literal promotes it, the product fused into the difference (pinned).
__device__ __forceinline__ float dense_up(const DenseArgs& a, int k) {
  const double zk = (double)__ldg(a.z + k);
  double r = ContractFull::TD ? __fma_rn(-a.Rm, (double)a.t, zk)
                              : __dsub_rn(zk, __dmul_rn(a.Rm, (double)a.t));
  r = __dsub_rn(r, 2.0);
  const float T = __double2float_rn(__dmul_rn((double)a.G, r));
  return __fdiv_rn(T, a.L_cp);
}

// The update of grain g from its seven stencil values (D,B,L,C,R,T,U).
__device__ __forceinline__ float dense_grain(const DenseArgs& a, KineConst kc, int g,
                                             const float v7[7], float repul, float Up) {
  float sina = 0.0f, cosa = 1.0f, sinb = 0.0f, cosb = 1.0f;
  if (v7[3] > __uint_as_float(kLSFloatBits)) {  // (double)ph[C] > LS
    const float4 o = __ldg(a.orient + g + 1);  // sint[g+1], cost[g+1], sint[g+1+NG], cost[g+1+NG]
    sina = o.x;
    cosa = o.y;
    sinb = o.z;
    cosb = o.w;
  }
  return slot_update<true>(a, kc, v7, sina, cosa, sinb, cosb, repul, Up);
}

__global__ void __launch_bounds__(128) dense_update_kernel(const DenseArgs a) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > a.fnx - 2 || j > a.fny - 2) return;
  const long long plane = (long long)a.fnx * a.fny;
  const long long C = i + (long long)a.fnx * j + plane * k;
  // stencil cells D,B,L,C,R,T,U through the mirror map of the halo
  long long nb[7];
  nb[0] = i + (long long)a.fnx * j + plane * mirror(k - 1, a.fnz);
  nb[1] = i + (long long)a.fnx * mirror(j - 1, a.fny) + plane * k;
  nb[2] = mirror(i - 1, a.fnx) + (long long)a.fnx * j + plane * k;
  nb[3] = C;
  nb[4] = mirror(i + 1, a.fnx) + (long long)a.fnx * j + plane * k;
  nb[5] = i + (long long)a.fnx * mirror(j + 1, a.fny) + plane * k;
  nb[6] = i + (long long)a.fnx * j + plane * mirror(k + 1, a.fnz);

  const KineConst kc = kine_const(a.kin_delta);
  const float Up = dense_up(a, k);
  int c7[7];
  bool over = false;
#pragma unroll
  for (int s = 0; s < 7; ++s) {
    c7[s] = __ldg(a.cnt + nb[s]);
    over = over || c7[s] > a.K;
  }

  // the output's grains that are not -1 (its content of two steps ago) back to -1
  {
    const int co = a.reset_from_lists ? a.cnt_o[C] : a.K + 1;
    if (over || co > a.K) {
      if (!over)
        for (int g = 0; g < a.np; ++g) a.out[g * a.len + C] = -1.0f;
    } else {
      for (int e = 0; e < co; ++e) a.out[(long long)a.lid_o[e * a.len + C] * a.len + C] = -1.0f;
    }
  }

  int cn = 0;  // the output's new list at C
  auto emit = [&](int g, float v) {
    if (v != -1.0f) {
      if (cn < a.K) {
        a.lid_o[cn * a.len + C] = (unsigned short)g;
        a.lval_o[cn * a.len + C] = v;
      }
      ++cn;
    }
  };

  if (!over) {
    // centre list in registers (the repulsion sums run over it for every grain)
    int cid[kDenseListMax];
    float cval[kDenseListMax];
#pragma unroll
    for (int e = 0; e < kDenseListMax; ++e) {
      cid[e] = -1;
      cval[e] = -1.0f;
      if (e < c7[3]) {
        cid[e] = __ldg(a.lid + e * a.len + C);
        cval[e] = __ldg(a.lval + e * a.len + C);
      }
    }
    // seven-way merge of the ascending lists: every grain of the union once
    int pos[7], head[7];
#pragma unroll
    for (int s = 0; s < 7; ++s) {
      pos[s] = 0;
      head[s] = c7[s] > 0 ? (int)__ldg(a.lid + nb[s]) : 0x10000;
    }
    for (;;) {
      int g = head[0];
#pragma unroll
      for (int s = 1; s < 7; ++s) g = min(g, head[s]);
      if (g == 0x10000) break;
      float v7[7];
#pragma unroll
      for (int s = 0; s < 7; ++s) {
        v7[s] = -1.0f;
        if (head[s] == g) {
          v7[s] = __ldg(a.lval + pos[s] * a.len + nb[s]);
          ++pos[s];
          head[s] = pos[s] < c7[s] ? (int)__ldg(a.lid + pos[s] * a.len + nb[s]) : 0x10000;
        }
      }
      // repul over every other grain in ascending order; the grains not in the
      // centre list are -1 there and add exactly zero (PhaseField.cu:280-286)
      float repul = 0.0f;
#pragma unroll
      for (int e = 0; e < kDenseListMax; ++e) {
        if (e >= c7[3]) break;
        if (cid[e] != g) repul = repul_add(repul, cval[e]);
      }
      const float v = dense_grain(a, kc, g, v7, repul, Up);
      a.out[g * a.len + C] = v;
      emit(g, v);
    }
  } else {
    // a list past capacity somewhere in the stencil: every grain from the buffer
    atomicAdd(a.overflow, 1ull);
    for (int g = 0; g < a.np; ++g) {
      float v7[7];
      bool any = false;
#pragma unroll
      for (int s = 0; s < 7; ++s) {
        v7[s] = __ldg(a.in + g * a.len + nb[s]);
        any = any || v7[s] != -1.0f;
      }
      float v = -1.0f;
      if (any) {
        float repul = 0.0f;
        for (int q = 0; q < a.np; ++q)
          if (q != g) repul = repul_add(repul, __ldg(a.in + q * a.len + C));
        v = dense_grain(a, kc, g, v7, repul, Up);
      }
      a.out[g * a.len + C] = v;
      emit(g, v);
    }
  }
  a.cnt_o[C] = cn;
}

// set_minus1 x2 + ini_PF x2 (PhaseField.cu:51-57, 91-107): every grain -1, then
// grain alpha-1 = phi where phi > LS; the argmax phi field -1, argmax index 0.
__global__ void dense_init_kernel(float* A, float* B, const float* __restrict__ phi,
                                  const int* __restrict__ alpha, float* phi_m, int* argmax, int np,
                                  long long len) {
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < len;
       C += (long long)gridDim.x * blockDim.x) {
    const float v = phi[C];
    const int g0 = ((double)v > LS) ? alpha[C] - 1 : -1;
    for (int g = 0; g < np; ++g) {
      const float o = (g == g0) ? v : -1.0f;
      A[g * len + C] = o;
      B[g * len + C] = o;
    }
    phi_m[C] = -1.0f;
    argmax[C] = 0;
  }
}

// collect_PF (PhaseField.cu:60-88): the argmax starts from the previous call's
// (a grain replaces it only when strictly larger), and phi / alpha change only
// where the max is above LS.
__global__ void dense_collect_kernel(const float* __restrict__ ph, float* phi, int* alpha,
                                     int* argmax, int np, long long len) {
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < len;
       C += (long long)gridDim.x * blockDim.x) {
    int am = argmax[C];
    float best = ph[am * len + C];
    for (int g = 0; g < np; ++g) {
      const float v = ph[g * len + C];
      if (v > best) {
        am = g;
        best = v;
      }
    }
    argmax[C] = am;
    if ((double)best > LS) {
      phi[C] = best;
      alpha[C] = am + 1;
    }
  }
}

// move_frame's field part (PhaseField.cu:331-337): interior layers k <- k+1 for
// k < fnz-2, the top interior layer extrapolated as 2*phi[top] - phi[top-1].
__global__ void dense_shift_kernel(const float* __restrict__ src, float* dst, int fnx, int fny,
                                   int fnz, int np) {
  const int ni = fnx - 2, nj = fny - 2, nk = fnz - 2;
  const long long plane = (long long)fnx * fny, len = plane * fnz;
  const long long total = (long long)ni * nj * nk * np;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    const int i = 1 + (int)(r % ni);
    r /= ni;
    const int j = 1 + (int)(r % nj);
    r /= nj;
    const int k = 1 + (int)(r % nk);
    const int g = (int)(r / nk);
    const long long d = g * len + i + (long long)fnx * j + plane * k;
    dst[d] = (k < fnz - 2) ? src[d + plane] : __fsub_rn(__fmul_rn(2.0f, src[d]), src[d - plane]);
  }
}

}  // namespace cupf
