// apt_aux.cuh — the non-step kernels of the B200 APT solver.
//
// All operate on the pair-plane buffers described in apt_common.cuh.  None of
// them is on the per-step hot path; they run at init, at QoI / moving-domain
// events and on read-back.
#pragma once

#include "apt_storage.cuh"

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

// Materialise the halo: every cell with a coordinate on the boundary takes the
// record of its mapped interior source (each coordinate mapped independently,
// = sequential z, y, x face fills of APTsetBC3D, APTPhaseField.cu:93-174).
// Cells are enumerated face by face without repetition.
__host__ __device__ __forceinline__ long long halo_cells(const Grid& g) {
  return 2ll * g.fnx * g.fny + 2ll * g.fnx * (g.fnz - 2) + 2ll * (g.fny - 2) * (g.fnz - 2);
}

// Halo cell idx (0 .. halo_cells-1): the two z planes, then the two y faces of
// the interior planes, then the two x faces of the interior rows.
__device__ __forceinline__ void halo_cell(long long idx, const Grid& g, int& i, int& j, int& k) {
  const long long nz2 = 2ll * g.fnx * g.fny;
  const long long ny2 = 2ll * g.fnx * (g.fnz - 2);
  const long long nx2 = 2ll * (g.fny - 2) * (g.fnz - 2);
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
}

template <class S>
__global__ void fill_halo_kernel(typename S::T* buf, Grid g, int bcX, int bcY, int bcZ) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < halo_cells(g);
       idx += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    halo_cell(idx, g, i, j, k);
    const long long d = g.at(i, j, k);
    const long long s = g.at(bc_map(i, g.fnx, bcX), bc_map(j, g.fny, bcY), bc_map(k, g.fnz, bcZ));
    for (int p = 0; p < g.np; ++p) buf[p * g.ss + d] = buf[p * g.ss + s];
  }
}

// The halo cells of every slot, copied from src to dst unchanged.
template <class S>
__global__ void copy_halo_kernel(const typename S::T* __restrict__ src, typename S::T* dst,
                                 Grid g) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < halo_cells(g);
       idx += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    halo_cell(idx, g, i, j, k);
    const long long d = g.at(i, j, k);
    for (int p = 0; p < g.np; ++p) dst[p * g.ss + d] = src[p * g.ss + d];
  }
}

// set_minus1 + APTini_PF on both buffers (PhaseField.cu:51-57, APTPhaseField.cu:78-89):
// every slot (-1, -1), then slot 0 = (phi, alpha) where phi > LS.  phi/alpha in
// reference layout (index i + j*fnx + k*fnx*fny).
template <class S>
__global__ void init_kernel(typename S::T* A, typename S::T* B, const float* __restrict__ phi,
                            const int* __restrict__ alpha, Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L;
       C += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(C % g.fnx);
    const int j = (int)((C / g.fnx) % g.fny);
    const int k = (int)(C / ((long long)g.fnx * g.fny));
    const long long d = g.at(i, j, k);
    const float v = phi[C];
    typename S::T s0 = S::empty();
    if ((double)v > LS) s0 = S::make(v, alpha[C]);
    A[d] = s0;
    B[d] = s0;
    for (int p = 1; p < g.np; ++p) {
      A[p * g.ss + d] = S::empty();
      B[p * g.ss + d] = S::empty();
    }
  }
}

// APTcollect_PF (APTPhaseField.cu:55-75): argmax over slots, first max wins; the
// outputs change only where the max is above LS.
template <class S>
__global__ void collect_kernel(const typename S::T* __restrict__ buf, float* phi, int* alpha,
                               Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L;
       C += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(C % g.fnx);
    const int j = (int)((C / g.fnx) % g.fny);
    const int k = (int)(C / ((long long)g.fnx * g.fny));
    const long long d = g.at(i, j, k);
    typename S::T best = buf[d];
    float bv = S::phi(best);
    for (int p = 1; p < g.np; ++p) {
      const typename S::T v = buf[p * g.ss + d];
      const float f = S::phi(v);
      if (f > bv) {
        best = v;
        bv = f;
      }
    }
    if ((double)bv > LS) {
      phi[C] = bv;
      alpha[C] = S::id(best);
    }
  }
}

// pair planes -> reference layout (ph[slot*length + C], ids[slot*length + C])
template <class S>
__global__ void export_kernel(const typename S::T* __restrict__ buf, float* ph, int* ids, Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L * g.np;
       C += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(C / L);
    const long long c = C - p * L;
    const int i = (int)(c % g.fnx);
    const int j = (int)((c / g.fnx) % g.fny);
    const int k = (int)(c / ((long long)g.fnx * g.fny));
    const typename S::T v = buf[p * g.ss + g.at(i, j, k)];
    ph[C] = S::phi(v);
    ids[C] = S::id(v);
  }
}

template <class S>
__global__ void import_kernel(typename S::T* buf, const float* __restrict__ ph,
                              const int* __restrict__ ids, Grid g) {
  const long long L = g.length();
  for (long long C = blockIdx.x * (long long)blockDim.x + threadIdx.x; C < L * g.np;
       C += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(C / L);
    const long long c = C - p * L;
    const int i = (int)(c % g.fnx);
    const int j = (int)((c / g.fnx) % g.fny);
    const int k = (int)(c / ((long long)g.fnx * g.fny));
    buf[p * g.ss + g.at(i, j, k)] = S::make(ph[C], ids[C]);
  }
}

// Per-layer sum of phi over every slot and cell (halo included), one block per
// layer, double accumulation in a fixed order (deterministic; the reference
// accumulates with float atomics, PhaseField.cu:366-378).
template <class S>
__global__ void layer_sum_kernel(const typename S::T* __restrict__ buf, double* sums, Grid g) {
  const int k = blockIdx.x;
  double acc = 0.0;
  const long long n = (long long)g.fnx * g.fny;
  for (int p = 0; p < g.np; ++p)
    for (long long c = threadIdx.x; c < n; c += blockDim.x) {
      const int i = (int)(c % g.fnx), j = (int)(c / g.fnx);
      acc += (double)S::phi(buf[p * g.ss + g.at(i, j, k)]);
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
template <class S>
__global__ void shift_kernel(const typename S::T* __restrict__ src, typename S::T* dst, Grid g) {
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
    dst[d] = (k < g.fnz - 2) ? src[p * g.ss + g.at(i, j, k + 1)] : S::empty();
  }
}

// Quiet-item flags after the domain moved down by m planes (new plane k holds old
// plane k + m, planes past the top are empty): an item is quiet when every item
// that held its new planes was (bit 0; bits 1 and 2, its bottom and top plane,
// are set only with bit 0).  src: flags before the move, dst: after.
static __global__ void quiet_shift_kernel(const uint8_t* __restrict__ src, uint8_t* dst, int per_chunk,
                                          int nzc, int zc, int fnz, int m) {
  const long long n = (long long)per_chunk * nzc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / per_chunk), t = (int)(i - (long long)c * per_chunk);
    const int k0 = 1 + zc * c, k1 = min(k0 + zc, fnz - 1);  // planes [k0, k1)
    const int lo = k0 + m, hi = min(k1 - 1 + m, fnz - 2);   // old planes they hold
    uint8_t q = 1;
    for (int cc = (lo - 1) / zc; lo <= hi && cc <= (hi - 1) / zc; ++cc)
      q &= src[(long long)cc * per_chunk + t] & 1;
    dst[i] = q ? 7 : 0;  // plane bits only from a wholly empty item
  }
}

template <class S>
__global__ void copy_interior_kernel(const typename S::T* __restrict__ src, typename S::T* dst,
                                     Grid g) {
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
static __global__ void archive_kernel(const int* __restrict__ alpha, int* alpha_full, int* loss_area,
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
// Neighbouring cells mostly share a grain, so the lanes of a warp holding the
// same id add their count in one atomic from the lowest of them, which also
// holds their smallest index (a warp's lanes take consecutive interior cells,
// whose reference-layout indices increase with the lane).
static __global__ void volume_kernel(const int* __restrict__ alpha, int fnx, int fny, int fnz, int ng,
                              unsigned long long* counts, long long* first) {
  const long long ni = fnx - 2, nj = fny - 2, nk = fnz - 2;
  const long long total = ni * nj * nk;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = 1 + idx % ni, j = 1 + (idx / ni) % nj, k = 1 + idx / (ni * nj);
    const long long C = k * fnx * fny + j * fnx + i;
    const int a = alpha[C];
    const int key = (a >= 1 && a <= ng) ? a : 0;
    const unsigned peers = __match_any_sync(__activemask(), key);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) {
      atomicAdd(counts + key, (unsigned long long)__popc(peers));
      if (key) atomicMin(first + key, C);
    }
  }
}

// Candidate cells of the 3D junction search (QOI3D::searchJunctionsOnImage,
// QOI.cpp:233-311): a solid cell (alpha != 0) whose 19-point neighbourhood
// (offsets with di^2 + dj^2 + dk^2 <= 2, itself included) holds no liquid cell,
// exactly four distinct grain ids and no id more than ten times.  The indices
// (reference layout) are appended in arbitrary order; `count` receives how many
// cells qualify even past `cap`.  `distinct[idx]` (interior cells in (k, j, i)
// order) receives the number of distinct values, liquid included, that the
// reference's scan inserts into its hash map at that cell (0 where alpha == 0):
// the host needs their running maximum to reproduce the map's bucket count,
// which fixes the order of the grain ids in each record.
static __global__ void junction_candidates_kernel(const int* __restrict__ alpha, int fnx, int fny,
                                                  int fnz, long long* out, long long cap,
                                                  unsigned long long* count,
                                                  unsigned char* distinct) {
  const long long ni = fnx - 2, nj = fny - 2, nk = fnz - 2;
  const long long total = ni * nj * nk, plane = (long long)fnx * fny;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = 1 + idx % ni, j = 1 + (idx / ni) % nj, k = 1 + idx / (ni * nj);
    const long long C = k * plane + j * fnx + i;
    if (alpha[C] == 0) {
      distinct[idx] = 0;
      continue;
    }
    int vals[19], cnt[19];
    int nd = 0, maxc = 0;
    bool zero = false;
    for (int dk = -1; dk <= 1; ++dk)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          if (di * di + dj * dj + dk * dk > 2) continue;
          const int v = alpha[C + dk * plane + dj * fnx + di];
          zero |= (v == 0);
          int f = -1;
          for (int q = 0; q < nd; ++q)
            if (vals[q] == v) f = q;
          if (f < 0) {
            vals[nd] = v;
            cnt[nd] = 0;
            f = nd++;
          }
          maxc = max(maxc, ++cnt[f]);
        }
    distinct[idx] = (unsigned char)nd;
    if (zero || nd != 4 || maxc > 10) continue;
    const unsigned long long slot = atomicAdd(count, 1ull);
    if ((long long)slot < cap) out[slot] = C;
  }
}

// Candidate cells of the line-configuration junction search
// (QOILine::searchJunctionsOnImage, QOI.cpp:103-160) over `nl` stacked x-y
// layers of an argmax map (the layers at the sampled tip heights): interior
// cells whose 3x3 in-plane neighbourhood holds at least three distinct values,
// none more than five times.  out receives the cells' indices in the stacked
// layers (layer * fnx * fny + j * fnx + i) in no particular order, up to cap;
// count receives their number.
static __global__ void line_junction_kernel(const int* __restrict__ layers, int nl, int fnx,
                                            int fny, long long* out, long long cap,
                                            unsigned long long* count) {
  const long long ni = fnx - 2, nj = fny - 2;
  const long long total = ni * nj * nl, plane = (long long)fnx * fny;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = 1 + idx % ni, j = 1 + (idx / ni) % nj, l = idx / (ni * nj);
    const long long C = l * plane + j * fnx + i;
    int v[9];
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
      for (int di = -1; di <= 1; ++di) v[(dj + 1) * 3 + di + 1] = __ldg(layers + C + dj * fnx + di);
    int nd = 0, maxc = 0;
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      bool first = true;
      int c = 0;
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        c += (v[b] == v[a]);
        if (b < a && v[b] == v[a]) first = false;
      }
      nd += first;
      maxc = max(maxc, c);
    }
    if (nd < 3 || maxc > 5) continue;
    const unsigned long long slot = atomicAdd(count, 1ull);
    if ((long long)slot < cap) out[slot] = C;
  }
}

// FP64 interface QoIs over the interior, from m = max-over-slots phi of each cell:
//   part[2*b]   = sum (1 + m) / 2              (solid volume, cell units)
//   part[2*b+1] = sum |grad m| / 2             (interface area, cell units; a
//                 diffuse interface integrates |grad phi| to 2 across its width)
// with central differences of m on the 6 neighbours (halo cells filled first).
// One partial pair per block; the host adds the partials in block order.
template <class S>
__device__ __forceinline__ float max_phi(const typename S::T* __restrict__ buf, const Grid& g,
                                         long long d) {
  float m = S::phi(buf[d]);
  for (int p = 1; p < g.np; ++p) m = fmaxf(m, S::phi(buf[p * g.ss + d]));
  return m;
}

template <class S>
__global__ void qoi_sums_kernel(const typename S::T* __restrict__ buf, Grid g, double* part) {
  const long long ni = g.fnx - 2, nj = g.fny - 2, nk = g.fnz - 2;
  const long long total = ni * nj * nk;
  double vol = 0.0, area = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(idx % ni), j = 1 + (int)((idx / ni) % nj), k = 1 + (int)(idx / (ni * nj));
    const long long d = g.at(i, j, k);
    const double m = max_phi<S>(buf, g, d);
    vol += 0.5 * (1.0 + m);
    const double gx = 0.5 * ((double)max_phi<S>(buf, g, d + 1) - max_phi<S>(buf, g, d - 1));
    const double gy = 0.5 * ((double)max_phi<S>(buf, g, d + g.xp) - max_phi<S>(buf, g, d - g.xp));
    const double gz =
        0.5 * ((double)max_phi<S>(buf, g, d + g.plane()) - max_phi<S>(buf, g, d - g.plane()));
    area += 0.5 * sqrt(gx * gx + gy * gy + gz * gz);
  }
  __shared__ double rv[256], ra[256];
  rv[threadIdx.x] = vol;
  ra[threadIdx.x] = area;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      rv[threadIdx.x] += rv[threadIdx.x + s];
      ra[threadIdx.x] += ra[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = rv[0];
    part[2 * blockIdx.x + 1] = ra[0];
  }
}

}  // namespace cupf
