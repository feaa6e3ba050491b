// cupf_dense.cu — C ABI of the full (non-APT) phase-field mode (include/cupf_dense.h).
//
// The handle owns two phi buffers of num_theta grain fields (reference layout),
// the per-cell lists of the step, the argmax fields with the persistent argmax
// index of collect_PF, the moving-domain archive and one CUDA stream.  Every CUDA
// call is checked and mapped to a status code.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/cupf_dense.h"
#include "capi_internal.h"
#include "dense.cuh"

using namespace cupf;

struct cupf_dense_handle {
  cupf_apt_params p;
  int device = 0;
  int np = 0;
  long long len = 0;
  Grid g;  // phi-only view for the shared halo / layer-sum / copy kernels
  float R = 0.0f;
  float* buf[2] = {nullptr, nullptr};
  int cur = 0;                // buffer the next step reads
  bool halo_ok[2] = {false, false};
  int K = kDenseListMax;
  // per-buffer lists of the grains that are not -1 at each cell (dense.cuh)
  int* cnt[2] = {nullptr, nullptr};
  unsigned short* lid[2] = {nullptr, nullptr};
  float* lval[2] = {nullptr, nullptr};
  bool list_ok[2] = {false, false};  // lists describe the buffer's current content
  unsigned long long* overflow = nullptr;
  float *x = nullptr, *y = nullptr, *z = nullptr, *orient = nullptr;
  std::vector<float> z_host;
  float* phi_m = nullptr;
  int* alpha_m = nullptr;
  int* argmax = nullptr;
  double* layer_sums = nullptr;
  int* alpha_full = nullptr;
  int fnz_f = 0;
  int* loss_area = nullptr;
  int64_t steps_done = 0;
  bool initialised = false;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

int grid_for(long long n, int block = 256) {
  long long b = (n + block - 1) / block;
  return (int)std::max(1ll, std::min(b, 148ll * 32));
}

void free_handle(cupf_dense_handle* h) {
  void* ptrs[] = {h->buf[0], h->buf[1], h->cnt[0], h->cnt[1], h->lid[0], h->lid[1], h->lval[0],
                  h->lval[1], h->overflow, h->x, h->y, h->z,
                  h->orient, h->phi_m, h->alpha_m, h->argmax, h->layer_sums, h->alpha_full,
                  h->loss_area};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

cupf_status upload(float** dst, const float* src, size_t n, cudaStream_t s) {
  CK(cudaMalloc((void**)dst, std::max<size_t>(n, 1) * sizeof(float)));
  if (n) CK(cudaMemcpyAsync(*dst, src, n * sizeof(float), cudaMemcpyHostToDevice, s));
  return CUPF_OK;
}

cupf_status fill_halo(cupf_dense_handle* h, int b) {
  if (h->halo_ok[b]) return CUPF_OK;
  const Grid& g = h->g;
  const long long nh = 2ll * g.fnx * g.fny + 2ll * g.fnx * (g.fnz - 2) + 2ll * (g.fny - 2) * (g.fnz - 2);
  fill_halo_kernel<DensePhi><<<grid_for(nh), 256, 0, h->stream>>>(h->buf[b], g, 0, 0, 0);
  CK(cudaGetLastError());
  h->halo_ok[b] = true;
  return CUPF_OK;
}

// One update of the current buffer into the other at time t.
cupf_status launch_step(cupf_dense_handle* h, float t) {
  const cupf_apt_params& p = h->p;
  const dim3 blk(32, 4);
  const dim3 grd((p.fnx - 2 + 31) / 32, (p.fny - 2 + 3) / 4, p.fnz - 2);
  const int ci = h->cur, co = h->cur ^ 1;
  if (!h->list_ok[ci]) {  // the state was replaced: lists from one read of every grain
    dense_list_kernel<<<grd, blk, 0, h->stream>>>(h->buf[ci], p.fnx, p.fny, p.fnz, h->np, h->K,
                                                  h->len, h->cnt[ci], h->lid[ci], h->lval[ci]);
    CK(cudaGetLastError());
    h->list_ok[ci] = true;
  }
  CK(cudaMemsetAsync(h->overflow, 0, sizeof(unsigned long long), h->stream));
  DenseArgs a;
  std::memset(&a, 0, sizeof(a));
  a.fnx = p.fnx;
  a.fny = p.fny;
  a.fnz = p.fnz;
  a.np = h->np;
  a.K = h->K;
  a.len = h->len;
  a.t = t;
  a.Rm = (double)h->R * 1e6;
  a.G = p.G;
  a.L_cp = p.L_cp;
  a.hi = p.hi;
  a.lamd = p.lamd;
  a.dt = p.dt;
  a.eps = p.eps;
  a.kin_delta = p.kin_delta;
  a.z = h->z;
  a.orient = reinterpret_cast<const float4*>(h->orient);
  a.in = h->buf[ci];
  a.out = h->buf[co];
  a.cnt = h->cnt[ci];
  a.lid = h->lid[ci];
  a.lval = h->lval[ci];
  a.cnt_o = h->cnt[co];
  a.lid_o = h->lid[co];
  a.lval_o = h->lval[co];
  a.reset_from_lists = h->list_ok[co] ? 1 : 0;
  a.overflow = h->overflow;
  dense_update_kernel<<<grd, blk, 0, h->stream>>>(a);
  CK(cudaGetLastError());
  h->list_ok[co] = true;
  h->cur ^= 1;
  h->halo_ok[h->cur] = false;
  return CUPF_OK;
}

// collect_PF on the current buffer; fill = false reads the halo as it stands
// (inside the moving-domain loop, where the reference does not refill it).
cupf_status collect(cupf_dense_handle* h, bool clear, bool fill = true) {
  if (fill) {
    cupf_status st = fill_halo(h, h->cur);
    if (st) return st;
  }
  if (clear) CK(cudaMemsetAsync(h->alpha_m, 0, h->len * sizeof(int), h->stream));
  dense_collect_kernel<<<grid_for(h->len), 256, 0, h->stream>>>(h->buf[h->cur], h->phi_m,
                                                                h->alpha_m, h->argmax, h->np, h->len);
  CK(cudaGetLastError());
  return CUPF_OK;
}

}  // namespace

#define TRY(x)                  \
  do {                          \
    cupf_status s_ = (x);       \
    if (s_ != CUPF_OK) {        \
      free_handle(h);           \
      return s_;                \
    }                           \
  } while (0)

extern "C" cupf_status cupf_dense_create(const cupf_apt_params* p, const cupf_apt_inputs* in,
                                         float R, int device, cupf_dense_handle** out) {
  if (!p || !in || !out) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->fnx < 4 || p->fny < 4 || p->fnz < 4)
    return cupf_fail(CUPF_ERR_INVALID, "grid %dx%dx%d too small (>= 4 points per axis)", p->fnx,
                     p->fny, p->fnz);
  if (p->num_theta < 1 || p->num_theta > 65535)
    return cupf_fail(CUPF_ERR_INVALID, "num_theta=%d outside 1..65535", p->num_theta);
  if (!in->z || !in->sint || !in->cost)
    return cupf_fail(CUPF_ERR_INVALID, "z, sint and cost are required");
  cupf_dense_handle* h = new cupf_dense_handle();
  h->p = *p;
  h->device = device;
  h->np = p->num_theta;
  h->len = (long long)p->fnx * p->fny * p->fnz;
  h->R = R;
  h->g.fnx = p->fnx;
  h->g.fny = p->fny;
  h->g.fnz = p->fnz;
  h->g.xp = p->fnx;
  h->g.np = h->np;
  h->g.ss = h->len;
  auto cuda = [&](cudaError_t e, const char* what) -> cupf_status {
    if (e == cudaSuccess) return CUPF_OK;
    return cupf_fail(e == cudaErrorMemoryAllocation ? CUPF_ERR_OOM : CUPF_ERR_CUDA, "%s: %s", what,
                     cudaGetErrorString(e));
  };
  TRY(cuda(cudaSetDevice(device), "cudaSetDevice"));
  TRY(cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream"));
  TRY(cuda(cudaEventCreate(&h->ev0), "event"));
  TRY(cuda(cudaEventCreate(&h->ev1), "event"));
  const size_t fbytes = (size_t)h->len * h->np * sizeof(float);
  for (int b = 0; b < 2; ++b) TRY(cuda(cudaMalloc((void**)&h->buf[b], fbytes), "phi buffer"));
  for (int b = 0; b < 2; ++b) {
    TRY(cuda(cudaMalloc((void**)&h->cnt[b], h->len * sizeof(int)), "list counts"));
    TRY(cuda(cudaMemsetAsync(h->cnt[b], 0, h->len * sizeof(int), h->stream), "memset"));
    TRY(cuda(cudaMalloc((void**)&h->lid[b], (size_t)kDenseListMax * h->len * sizeof(unsigned short)),
             "lists"));
    TRY(cuda(cudaMalloc((void**)&h->lval[b], (size_t)kDenseListMax * h->len * sizeof(float)),
             "lists"));
  }
  TRY(cuda(cudaMalloc((void**)&h->overflow, sizeof(unsigned long long)), "overflow counter"));
  TRY(cuda(cudaMemsetAsync(h->overflow, 0, sizeof(unsigned long long), h->stream), "memset"));
  if (in->x) TRY(upload(&h->x, in->x, p->fnx, h->stream));
  if (in->y) TRY(upload(&h->y, in->y, p->fny, h->stream));
  TRY(upload(&h->z, in->z, p->fnz, h->stream));
  h->z_host.assign(in->z, in->z + p->fnz);
  {
    std::vector<float> ot(4 * (size_t)(p->num_theta + 1));
    pack_orientations(in->sint, in->cost, p->num_theta, ot.data());
    TRY(upload(&h->orient, ot.data(), ot.size(), h->stream));
  }
  TRY(cuda(cudaMalloc((void**)&h->phi_m, h->len * sizeof(float)), "phi field"));
  TRY(cuda(cudaMalloc((void**)&h->alpha_m, h->len * sizeof(int)), "alpha field"));
  TRY(cuda(cudaMalloc((void**)&h->argmax, h->len * sizeof(int)), "argmax"));
  TRY(cuda(cudaMemsetAsync(h->argmax, 0, h->len * sizeof(int), h->stream), "memset"));
  TRY(cuda(cudaMalloc((void**)&h->layer_sums, p->fnz * sizeof(double)), "layer sums"));
  TRY(cuda(cudaStreamSynchronize(h->stream), "sync"));
  *out = h;
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_destroy(cupf_dense_handle* h) {
  if (!h) return CUPF_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_handle(h);
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_init_from_argmax(cupf_dense_handle* h, const float* phi,
                                                   const int32_t* alpha) {
  if (!h || !phi || !alpha) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  struct Stage {  // device copy of phi for the init kernel, freed on every path
    float* p = nullptr;
    ~Stage() {
      if (p) cudaFree(p);
    }
  } stage;
  CK(cudaMalloc((void**)&stage.p, h->len * sizeof(float)));
  CK(cudaMemcpyAsync(stage.p, phi, h->len * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->alpha_m, alpha, h->len * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  dense_init_kernel<<<grid_for(h->len), 256, 0, h->stream>>>(h->buf[0], h->buf[1], stage.p,
                                                             h->alpha_m, h->phi_m, h->argmax, h->np,
                                                             h->len);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  h->cur = 0;
  h->halo_ok[0] = h->halo_ok[1] = false;
  h->list_ok[0] = h->list_ok[1] = false;
  cupf_status st = fill_halo(h, 0);
  if (st) return st;
  if ((st = fill_halo(h, 1))) return st;
  h->steps_done = 0;
  h->initialised = true;
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_prestep(cupf_dense_handle* h) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->initialised) return cupf_fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  return launch_step(h, 0.0f);
}

extern "C" cupf_status cupf_dense_step(cupf_dense_handle* h, int32_t nsteps) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->initialised) return cupf_fail(CUPF_ERR_STATE, "state not initialised");
  if (nsteps < 0) return cupf_fail(CUPF_ERR_INVALID, "nsteps < 0");
  CK(cudaSetDevice(h->device));
  for (int n = 0; n < nsteps; ++n) {
    // (2*kt+1)*dt*tau0 of evolve: integer step times dt, then tau0, in float
    const float t = (float)(h->steps_done + 1) * h->p.dt * h->p.tau0;
    cupf_status st = launch_step(h, t);
    if (st) return st;
    h->steps_done += 1;
  }
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_steps_done(cupf_dense_handle* h, int64_t* steps) {
  if (!h || !steps) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  *steps = h->steps_done;
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_collect(cupf_dense_handle* h, int32_t clear, float* phi_out,
                                          int32_t* alpha_out) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->initialised) return cupf_fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  cupf_status st = collect(h, clear != 0);
  if (st) return st;
  if (phi_out)
    CK(cudaMemcpyAsync(phi_out, h->phi_m, h->len * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (alpha_out)
    CK(cudaMemcpyAsync(alpha_out, h->alpha_m, h->len * sizeof(int), cudaMemcpyDeviceToHost,
                       h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_get_slots(cupf_dense_handle* h, float* ph) {
  if (!h || !ph) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  if (!h->initialised) return cupf_fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  cupf_status st = fill_halo(h, h->cur);
  if (st) return st;
  CK(cudaMemcpyAsync(ph, h->buf[h->cur], (size_t)h->len * h->np * sizeof(float),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_set_slots(cupf_dense_handle* h, const float* ph,
                                            int64_t steps_done) {
  if (!h || !ph) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->buf[h->cur], ph, (size_t)h->len * h->np * sizeof(float),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->halo_ok[h->cur] = false;
  h->list_ok[h->cur] = false;
  h->steps_done = steps_done;
  h->initialised = true;
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_move_domain(cupf_dense_handle* h, int32_t* tip_front,
                                              int32_t tip_thres, int32_t* move_count,
                                              int32_t* moved) {
  if (!h || !tip_front || !move_count || !moved) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  if (!h->initialised) return cupf_fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  const cupf_apt_params& p = h->p;
  if (*tip_front < 0 || *tip_front >= p.fnz)
    return cupf_fail(CUPF_ERR_INVALID, "tip_front=%d outside 0..%d", *tip_front, p.fnz - 1);
  const long long plane = (long long)p.fnx * p.fny;
  if (!h->alpha_full) {
    h->fnz_f = p.fnz * 4 + 8;
    CK(cudaMalloc((void**)&h->alpha_full, (size_t)plane * h->fnz_f * sizeof(int)));
    CK(cudaMemsetAsync(h->alpha_full, 0, (size_t)plane * h->fnz_f * sizeof(int), h->stream));
    CK(cudaMalloc((void**)&h->loss_area, p.num_theta * sizeof(int)));
    CK(cudaMemsetAsync(h->loss_area, 0, p.num_theta * sizeof(int), h->stream));
  }
  cupf_status st = fill_halo(h, h->cur);
  if (st) return st;
  layer_sum_kernel<DensePhi><<<p.fnz, 256, 0, h->stream>>>(h->buf[h->cur], h->layer_sums, h->g);
  CK(cudaGetLastError());
  std::vector<double> sums(p.fnz);
  CK(cudaMemcpyAsync(sums.data(), h->layer_sums, p.fnz * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // tip_mvf (PhaseField.cu:382-399): the first layer whose mean is not above LS
  const float denom = (float)((long long)h->np * p.fnx * p.fny);
  while (((double)((float)sums[*tip_front] / denom) > LS) && (*tip_front < p.fnz - 1))
    (*tip_front)++;
  *moved = 0;
  // collect_PF before the loop (PhaseField.cu:587)
  if ((st = collect(h, false))) return st;
  while (*tip_front >= tip_thres) {
    if (*move_count + 2 > h->fnz_f) {  // grow the archive
      const int nf = h->fnz_f * 2;
      int* na = nullptr;
      CK(cudaMalloc((void**)&na, (size_t)plane * nf * sizeof(int)));
      CK(cudaMemsetAsync(na, 0, (size_t)plane * nf * sizeof(int), h->stream));
      CK(cudaMemcpyAsync(na, h->alpha_full, (size_t)plane * h->fnz_f * sizeof(int),
                         cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaStreamSynchronize(h->stream));
      cudaFree(h->alpha_full);
      h->alpha_full = na;
      h->fnz_f = nf;
    }
    if ((st = collect(h, false, false))) return st;
    archive_kernel<<<grid_for(plane), 256, 0, h->stream>>>(h->alpha_m, h->alpha_full, h->loss_area,
                                                           p.fnx, p.fny, *move_count, p.num_theta);
    const long long ni = (long long)(p.fnx - 2) * (p.fny - 2) * (p.fnz - 2) * h->np;
    dense_shift_kernel<<<grid_for(ni), 256, 0, h->stream>>>(h->buf[h->cur], h->buf[h->cur ^ 1], p.fnx,
                                                            p.fny, p.fnz, h->np);
    copy_interior_kernel<DensePhi><<<grid_for(ni), 256, 0, h->stream>>>(h->buf[h->cur ^ 1],
                                                                        h->buf[h->cur], h->g);
    CK(cudaGetLastError());
    // z shift (move_frame :322-326 then copy_frame :355-356)
    std::vector<float>& z = h->z_host;
    const float ztop = 2.0f * z[p.fnz - 2] - z[p.fnz - 3];
    for (int k = 1; k < p.fnz - 2; ++k) z[k] = z[k + 1];
    z[p.fnz - 2] = ztop;
    CK(cudaMemcpyAsync(h->z, z.data(), p.fnz * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->halo_ok[h->cur] = false;
    h->halo_ok[h->cur ^ 1] = false;
    h->list_ok[0] = h->list_ok[1] = false;
    *move_count += 1;
    *tip_front -= 1;
    *moved += 1;
  }
  if ((st = fill_halo(h, h->cur))) return st;
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_get_archive(cupf_dense_handle* h, int32_t fnz_f,
                                              int32_t* alpha_full, int32_t* loss_area) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  CK(cudaSetDevice(h->device));
  const long long plane = (long long)h->p.fnx * h->p.fny;
  if (alpha_full) {
    std::memset(alpha_full, 0, (size_t)plane * fnz_f * sizeof(int));
    if (h->alpha_full)
      CK(cudaMemcpyAsync(alpha_full, h->alpha_full,
                         (size_t)plane * std::min(fnz_f, h->fnz_f) * sizeof(int),
                         cudaMemcpyDeviceToHost, h->stream));
  }
  if (loss_area) {
    std::memset(loss_area, 0, h->p.num_theta * sizeof(int));
    if (h->loss_area)
      CK(cudaMemcpyAsync(loss_area, h->loss_area, h->p.num_theta * sizeof(int),
                         cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_get_z(cupf_dense_handle* h, float* z) {
  if (!h || !z) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  std::memcpy(z, h->z_host.data(), h->p.fnz * sizeof(float));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_sync(cupf_dense_handle* h, int32_t timeout_ms) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  CK(cudaSetDevice(h->device));
  if (timeout_ms <= 0) {
    CK(cudaStreamSynchronize(h->stream));
    return CUPF_OK;
  }
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(h->stream);
    if (e == cudaSuccess) return CUPF_OK;
    if (e != cudaErrorNotReady) CK(e);
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0)
                  .count();
    if (ms > timeout_ms) return cupf_fail(CUPF_ERR_TIMEOUT, "stream not idle after %d ms", timeout_ms);
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

extern "C" cupf_status cupf_dense_time_steps(cupf_dense_handle* h, int32_t nsteps, float* ms) {
  if (!h || !ms) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaEventRecord(h->ev0, h->stream));
  cupf_status st = cupf_dense_step(h, nsteps);
  if (st) return st;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_set_tuning(cupf_dense_handle* h, int32_t list_cap) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (list_cap < 1 || list_cap > kDenseListMax)
    return cupf_fail(CUPF_ERR_INVALID, "list_cap=%d outside 1..%d", list_cap, kDenseListMax);
  h->K = list_cap;
  h->list_ok[0] = h->list_ok[1] = false;  // lists hold at most the old capacity
  return CUPF_OK;
}

extern "C" cupf_status cupf_dense_overflow_cells(cupf_dense_handle* h, int64_t* overflow_cells) {
  if (!h || !overflow_cells) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, h->overflow, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *overflow_cells = (int64_t)v;
  return CUPF_OK;
}
