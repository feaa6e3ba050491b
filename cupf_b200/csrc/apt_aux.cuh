// apt_aux.cuh — the non-step kernels of the B200 APT solver.
//
// All operate on the pair-plane buffers described in apt_common.cuh.  None of
// them is on the per-step hot path; they run at init, at QoI / moving-domain
// events and on read-back.
#pragma once

#include "apt_common.cuh"

namespace cupf {

struct Grid {
  int fnx, fny, fnz, xp, np;
  long long ss;  // slot stride in pairs
  __host__ __device__ long long plane() const { return (long long)xp * fny; }
  __host__ __device__ long long at(int i, int j, int k) const {
    return (long long)k * plane() + (long long)j * xp + i;
  }
  __host__ __device__ long long length() const { return (long long)fnx * fny * fnz; }
};

__device__ __forceinline__ uint2 empty_pair() {
  return make_uint2(__float_as_uint(-1.0f), 0xFFFFFFFFu);
}

// Materialise the halo: every cell with a coordinate on the boundary takes the
// record of its mapped interior source (each coordinate mapped independently,
// = sequential z, y, x face fills of APTsetBC3D, APTPhaseField.cu:93-174).
// Cells are enumerated face by face without repetition.
__global__ void fill_halo_kernel(uint2* buf, Grid g, int bcX, int bcY, int bcZ) {
  const long long nz2 = 2ll * g.fnx * g.fny;
  const long long ny2 = 2ll * g.fnx * (g.fnz - 2);
  const long long nx2 = 2ll * (g.fny - 2) * (g.fnz - 2);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < nz2 + ny2 + nx2;
       idx += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    long long r = idx;
    if (r < nz2) {
      k = (r < nz2 / 2) ? 0 : g.fnz - 1;
      r %= (long long)g.fnx * g.fny;
      j = (int)(r / g.fnx);
      i = (int)(r % g.fnx);
    } else if ((r -= nz2) < ny2) {
      j = (r < ny2 / 2) ? 0 : g.fny - 1;
      r %= (long long)g.fnx * (g.fnz - 2);
      k = 1 + (int)(r / g.fnx);
      i = (int)(r % g.fnx);
    } else {
      r -= ny2;
      i = (r < nx2 / 2) ? 0 : g.fnx - 1;
      r %= (long long)(g.fny - 2) * (g.fnz - 2);
      k = 1 + (int)(r / (g.fny - 2));
      j = 1 + (int)(r % (g.fny - 2));
    }
    const long long d = g.at(i, j, k);
    const long long s = g.at(bc_map(i, g.fnx, bcX), bc_map(j, g.fny, bcY), bc_map(k, g.fnz, bcZ));
    for (int p = 0; p < g.np; ++p) buf[p * g.ss + d] = buf[p * g.ss + s];
  }
}

// set_minus1 + APTini_PF on both buffers (PhaseField.cu:51-57, APTPhaseField.cu:78-89):
// every slot (-1, -1), then slot 0 = (phi, alpha) where phi > LS.  phi/alpha in
// reference layout (index i + j*fnx + k*fnx*fny).
__global__ void init_kernel(uint2* A, uint2* B, const float* __restrict__ phi,
                            const int* __restrict__ alpha, Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L;
       C += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(C % g.fnx);
    const int j = (int)((C / g.fnx) % g.fny);
    const int k = (int)(C / ((long long)g.fnx * g.fny));
    const long long d = g.at(i, j, k);
    const float v = phi[C];
    uint2 s0 = empty_pair();
    if ((double)v > LS) s0 = make_uint2(__float_as_uint(v), (uint32_t)alpha[C]);
    A[d] = s0;
    B[d] = s0;
    for (int p = 1; p < g.np; ++p) {
      A[p * g.ss + d] = empty_pair();
      B[p * g.ss + d] = empty_pair();
    }
  }
}

// APTcollect_PF (APTPhaseField.cu:55-75): argmax over slots, first max wins; the
// outputs change only where the max is above LS.
__global__ void collect_kernel(const uint2* __restrict__ buf, float* phi, int* alpha, Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L;
       C += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(C % g.fnx);
    const int j = (int)((C / g.fnx) % g.fny);
    const int k = (int)(C / ((long long)g.fnx * g.fny));
    const long long d = g.at(i, j, k);
    uint2 best = buf[d];
    for (int p = 1; p < g.np; ++p) {
      const uint2 v = buf[p * g.ss + d];
      if (__uint_as_float(v.x) > __uint_as_float(best.x)) best = v;
    }
    if ((double)__uint_as_float(best.x) > LS) {
      phi[C] = __uint_as_float(best.x);
      alpha[C] = (int)best.y;
    }
  }
}

// pair planes -> reference layout (ph[slot*length + C], ids[slot*length + C])
__global__ void export_kernel(const uint2* __restrict__ buf, float* ph, int* ids, Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L * g.np;
       C += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(C / L);
    const long long c = C - p * L;
    const int i = (int)(c % g.fnx);
    const int j = (int)((c / g.fnx) % g.fny);
    const int k = (int)(c / ((long long)g.fnx * g.fny));
    const uint2 v = buf[p * g.ss + g.at(i, j, k)];
    ph[C] = __uint_as_float(v.x);
    ids[C] = (int)v.y;
  }
}

__global__ void import_kernel(uint2* buf, const float* __restrict__ ph, const int* __restrict__ ids,
                              Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L * g.np;
       C += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(C / L);
    const long long c = C - p * L;
    const int i = (int)(c % g.fnx);
    const int j = (int)((c / g.fnx) % g.fny);
    const int k = (int)(c / ((long long)g.fnx * g.fny));
    buf[p * g.ss + g.at(i, j, k)] = make_uint2(__float_as_uint(ph[C]), (uint32_t)ids[C]);
  }
}

// Per-layer sum of phi over every slot and cell (halo included), one block per
// layer, double accumulation in a fixed order (deterministic; the reference
// accumulates with float atomics, PhaseField.cu:366-378).
__global__ void layer_sum_kernel(const uint2* __restrict__ buf, double* sums, Grid g) {
  const int k = blockIdx.x;
  double acc = 0.0;
  const long long n = (long long)g.fnx * g.fny;
  for (int p = 0; p < g.np; ++p)
    for (long long c = threadIdx.x; c < n; c += blockDim.x) {
      const int i = (int)(c % g.fnx), j = (int)(c / g.fnx);
      acc += (double)__uint_as_float(buf[p * g.ss + g.at(i, j, k)].x);
    }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[k] = red[0];
}

// One-layer shift of the interior (APTmove_frame + APTcopy_frame,
// APTPhaseField.cu:357-410): dst[k] = src[k+1] for k < fnz-2, top interior layer
// (-1, -1).  Halo cells are not touched.
__global__ void shift_kernel(const uint2* __restrict__ src, uint2* dst, Grid g) {
  const int ni = g.fnx - 2, nj = g.fny - 2, nk = g.fnz - 2;
  const long long total = (long long)ni * nj * nk * g.np;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    const int i = 1 + (int)(r % ni);
    r /= ni;
    const int j = 1 + (int)(r % nj);
    r /= nj;
    const int k = 1 + (int)(r % nk);
    const int p = (int)(r / nk);
    const long long d = p * g.ss + g.at(i, j, k);
    dst[d] = (k < g.fnz - 2) ? src[p * g.ss + g.at(i, j, k + 1)] : empty_pair();
  }
}

__global__ void copy_interior_kernel(const uint2* __restrict__ src, uint2* dst, Grid g) {
  const int ni = g.fnx - 2, nj = g.fny - 2, nk = g.fnz - 2;
  const long long total = (long long)ni * nj * nk * g.np;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    const int i = 1 + (int)(r % ni);
    r /= ni;
    const int j = 1 + (int)(r % nj);
    r /= nj;
    const int k = 1 + (int)(r % nk);
    const int p = (int)(r / nk);
    const long long d = p * g.ss + g.at(i, j, k);
    dst[d] = src[d];
  }
}

// Archive the bottom interior layer of the argmax map and count it into the
// lost area (APTPhaseField.cu:383-388): alpha_full[move*plane + C] = alpha[C] for
// C in layer 1 (all i, j), loss_area[alpha-1] += 1 for alpha in 1..num_theta.
__global__ void archive_kernel(const int* __restrict__ alpha, int* alpha_full, int* loss_area,
                               int fnx, int fny, int move_count, int num_theta) {
  const long long plane = (long long)fnx * fny;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < plane;
       c += (long long)gridDim.x * blockDim.x) {
    const int a = alpha[plane + c];
    alpha_full[move_count * plane + plane + c] = a;
    if (a >= 1 && a <= num_theta) atomicAdd(loss_area + a - 1, 1);
  }
}

// Voxel count per grain id over the interior of the argmax map, plus the first
// (k, j, i)-order index where each id occurs (for the reference's first-seen
// ordering, QOI.cpp:198-231).  counts[0] = interior cells with no grain.
__global__ void volume_kernel(const int* __restrict__ alpha, int fnx, int fny, int fnz, int ng,
                              unsigned long long* counts, long long* first) {
  const long long ni = fnx - 2, nj = fny - 2, nk = fnz - 2;
  const long long total = ni * nj * nk;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = 1 + idx % ni, j = 1 + (idx / ni) % nj, k = 1 + idx / (ni * nj);
    const long long C = k * fnx * fny + j * fnx + i;
    const int a = alpha[C];
    if (a >= 1 && a <= ng) {
      atomicAdd(counts + a, 1ull);
      atomicMin(first + a, C);
    } else {
      atomicAdd(counts, 1ull);
    }
  }
}

}  // namespace cupf
