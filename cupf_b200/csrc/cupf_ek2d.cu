// cupf_ek2d.cu — C ABI of the 2D Echebarria–Karma line-model step
// (include/cupf_ek2d.h).  Host side of setup() in cuPF
// 2DdendriteMPI/line_model/PF.cu:699-842: buffers, the FP64 varGR time
// integration, the step loop and the tip search / moving frame.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/cupf_ek2d.h"
#include "capi_internal.h"
#include "ek2d.cuh"

using namespace cupf::ek2d;

struct cupf_ek2d_handle {
  cupf_ek2d_params p;
  int prec = CUPF_PREC_FP32;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int fnx = 0, fny = 0, pitch = 0;
  int rows = 32;  // rows per warp of the step kernel
  long long plane = 0;
  size_t vbytes = 4;
  void* buf[2] = {nullptr, nullptr};
  int cur = 0;
  float* stage = nullptr;  // 4 reference-layout float planes for import/export
  double* d_rows = nullptr;
  std::vector<double> h_rows;
  std::vector<double> t_mac, Gt, Rt;
  bool have_state = false;
  int64_t steps = 0, shifts = 0;
  int cur_tip = 1, tip_thres = 0;
  double t = 0.0, intR = 0.0, lT_tilde = 0.0;
};

namespace {

template <class F>
cupf_status with_ek_storage(int prec, F&& f) {
  switch (prec) {
    case CUPF_PREC_FP32: return f(StF32{});
    case CUPF_PREC_FP16: return f(StF16{});
    case CUPF_PREC_BF16: return f(StBF16{});
    case CUPF_PREC_FP64: return f(StF64{});
    default: return cupf_fail(CUPF_ERR_INVALID, "unknown precision %d", prec);
  }
}

size_t value_bytes(int prec) {
  return prec == CUPF_PREC_FP64 ? 8 : (prec == CUPF_PREC_FP32 ? 4 : 2);
}

int grid_1d(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (int)std::max(1LL, b);
}

// R and G of the macro tables at time t (s): linear in the interval holding t,
// the last interval past the end (varGR, PF.cu:685-697).
void table_at(const cupf_ek2d_handle* h, double t, double* R, double* G) {
  const int nt = (int)h->t_mac.size();
  const double Dt = h->t_mac[1] - h->t_mac[0];
  const double x = (t - h->t_mac[0]) / Dt;
  int kt = (int)std::floor(x);
  kt = std::min(std::max(kt, 0), nt - 2);
  const double d = x - kt;
  *R = (1.0 - d) * h->Rt[kt] + d * h->Rt[kt + 1];
  *G = (1.0 - d) * h->Gt[kt] + d * h->Gt[kt + 1];
}

double thermal_length(const cupf_ek2d_params& p, double G) {
  return ((double)p.c_infm * (1.0 / (double)p.k - 1.0) / G) / (double)p.W0;
}

EkArgs make_args(const cupf_ek2d_handle* h, int prestep, uint32_t step) {
  const cupf_ek2d_params& p = h->p;
  EkArgs a;
  memset(&a, 0, sizeof(a));
  a.in = h->buf[h->cur];
  a.out = h->buf[h->cur ^ 1];
  a.plane = h->plane;
  a.pitch = h->pitch;
  a.fnx = h->fnx;
  a.fny = h->fny;
  a.prestep = prestep;
  a.k = p.k;
  a.hi = p.hi;
  a.Dl_tilde = p.Dl_tilde;
  a.eps = p.eps;
  a.sqrt2 = p.sqrt2;
  a.lamd = p.lamd;
  a.dt = p.dt;
  a.cosa = p.cosa;
  a.sina = p.sina;
  a.a_s = p.a_s;
  a.epsilon = p.epsilon;
  a.a_12 = p.a_12;
  a.U0 = p.U0;
  a.noise_amp = p.dt_sqrt * p.hi * p.eta;
  // Up of memory row j = (y_j/W0 - intR)/lT, y_j = y0 + (j - 1 + shifts)*dx*W0
  const double W0 = p.W0, dxd = (double)p.dx * (double)p.W0;
  a.up_a = ((p.y0 + ((double)h->shifts - 1.0) * dxd) / W0 - h->intR) / h->lT_tilde;
  a.up_b = (dxd / W0) / h->lT_tilde;
  a.seed = (uint32_t)p.seed_val;
  a.step = step;
  return a;
}

// Rows each warp marches over: 32, halved (down to 8) while the grid would give
// fewer than about two waves of resident warps (32 per SM at 8 warps per CTA).
int march_rows(const cupf_ek2d_handle* h) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const long long strips = (h->fnx - 2 + MW - 1) / MW;
  int rows = 32;
  while (rows > 8 && strips * ((h->fny - 2 + rows - 1) / rows) < 2LL * 32 * nsm) rows /= 2;
  return rows;
}

cupf_status launch_step(cupf_ek2d_handle* h, int prestep, uint32_t step) {
  EkArgs a = make_args(h, prestep, step);
  a.rows = h->rows;
  const int nstrips = (h->fnx - 2 + MW - 1) / MW;
  const dim3 grid((nstrips + MWARPS - 1) / MWARPS, (h->fny - 2 + a.rows - 1) / a.rows);
  return with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    ek2d_march_kernel<S><<<grid, MWARPS * 32, 0, h->stream>>>(a);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
}

// Tip search and moving frame after a multiple of tipp steps (tip_mvf and the
// while loop of PF.cu:811-818): advance cur_tip while the row mean of phi is
// above LS, then move the frame one row per row the tip has reached past
// tip_thres.
cupf_status tip_and_frame(cupf_ek2d_handle* h) {
  cupf_status st = with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    ek2d_row_sums_kernel<S><<<h->fny, 256, 0, h->stream>>>(h->buf[h->cur], h->pitch, h->fnx,
                                                          h->p.sqrt2, h->d_rows);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  if (st) return st;
  CK(cudaMemcpyAsync(h->h_rows.data(), h->d_rows, h->fny * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  while (h->h_rows[h->cur_tip] / h->fnx > (double)h->p.ls && h->cur_tip < h->fny - 1) h->cur_tip += 1;
  int k = 0;
  while (h->cur_tip >= h->tip_thres) {
    k += 1;
    h->cur_tip -= 1;
  }
  if (k == 0) return CUPF_OK;
  st = with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    const long long n = (long long)(h->fnx - 2) * (h->fny - 2);
    ek2d_shift_kernel<S><<<grid_1d(n), 256, 0, h->stream>>>(h->buf[h->cur], h->buf[h->cur ^ 1], h->plane,
                                                           h->pitch, h->fnx, h->fny, k, h->p.U0);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  if (st) return st;
  h->cur ^= 1;
  h->shifts += k;
  return CUPF_OK;
}

}  // namespace

extern "C" cupf_status cupf_ek2d_create(const cupf_ek2d_params* p, int32_t precision, int32_t device,
                                        cupf_ek2d_handle** out) {
  if (!p || !out) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  *out = nullptr;
  if (precision != CUPF_PREC_FP32 && precision != CUPF_PREC_FP16 && precision != CUPF_PREC_BF16 &&
      precision != CUPF_PREC_FP64)
    return cupf_fail(CUPF_ERR_INVALID, "unknown precision %d", precision);
  if (p->nx < 2 || p->ny < 2) return cupf_fail(CUPF_ERR_INVALID, "nx, ny must be >= 2");
  if ((long long)(p->nx + 2) * (p->ny + 3) > (1LL << 31))
    return cupf_fail(CUPF_ERR_INVALID, "grid larger than 2^31 points");
  if (p->tipp < 1) return cupf_fail(CUPF_ERR_INVALID, "tipp must be >= 1");
  if (!(p->dt > 0.0f) || !(p->W0 > 0.0f) || !(p->k > 0.0f) || !(p->dx > 0.0f))
    return cupf_fail(CUPF_ERR_INVALID, "dt, W0, k, dx must be positive");
  CK(cudaSetDevice(device));
  cupf_ek2d_handle* h = new cupf_ek2d_handle();
  h->p = *p;
  h->prec = precision;
  h->device = device;
  h->fnx = p->nx + 2;
  h->fny = p->ny + 3;
  h->vbytes = value_bytes(precision);
  const int align = (int)(128 / h->vbytes);  // rows start on 128 B
  h->pitch = (h->fnx + align - 1) / align * align;
  h->plane = (long long)h->pitch * h->fny;
  h->tip_thres = (int)((1.0 - (double)p->blank) * h->fny);
  h->rows = march_rows(h);
  h->h_rows.assign(h->fny, 0.0);
  auto bail = [&](cupf_status st) {
    cupf_ek2d_destroy(h);
    return st;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaMalloc(&h->buf[b], 3 * h->plane * h->vbytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->stage, 4 * (size_t)h->fnx * h->fny * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_rows, h->fny * sizeof(double));
  for (int b = 0; b < 2 && e == cudaSuccess; ++b)
    e = cudaMemsetAsync(h->buf[b], 0, 3 * h->plane * h->vbytes, h->stream);
  if (e != cudaSuccess)
    return bail(cupf_fail(e == cudaErrorMemoryAllocation ? CUPF_ERR_OOM : CUPF_ERR_CUDA,
                          "2D set-up failed: %s", cudaGetErrorString(e)));
  *out = h;
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_destroy(cupf_ek2d_handle* h) {
  if (!h) return CUPF_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int b = 0; b < 2; ++b)
    if (h->buf[b]) cudaFree(h->buf[b]);
  if (h->stage) cudaFree(h->stage);
  if (h->d_rows) cudaFree(h->d_rows);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_set_thermal(cupf_ek2d_handle* h, int32_t Nt, const float* t_mac,
                                             const float* Gt, const float* Rt) {
  if (!h || !t_mac || !Gt || !Rt) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  if (Nt < 2) return cupf_fail(CUPF_ERR_INVALID, "need at least two table times");
  if (!(t_mac[1] > t_mac[0])) return cupf_fail(CUPF_ERR_INVALID, "table times must increase");
  for (int i = 0; i < Nt; ++i)
    if (!(Gt[i] > 0.0f)) return cupf_fail(CUPF_ERR_INVALID, "G must be positive (entry %d)", i);
  h->t_mac.assign(t_mac, t_mac + Nt);
  h->Gt.assign(Gt, Gt + Nt);
  h->Rt.assign(Rt, Rt + Nt);
  h->lT_tilde = thermal_length(h->p, h->Gt[0]);
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_set_state(cupf_ek2d_handle* h, const float* psi, const float* U,
                                           const float* dpsi) {
  if (!h || !psi || !U) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  const size_t n = (size_t)h->fnx * h->fny;
  float* d_ps = h->stage;
  float* d_U = h->stage + n;
  float* d_D = dpsi ? h->stage + 2 * n : nullptr;
  CK(cudaMemcpyAsync(d_ps, psi, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(d_U, U, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  if (dpsi) CK(cudaMemcpyAsync(d_D, dpsi, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  cupf_status st = with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    const long long m = (long long)(h->fnx - 2) * (h->fny - 2);
    ek2d_import_kernel<S><<<grid_1d(m), 256, 0, h->stream>>>(d_ps, d_U, d_D, h->buf[h->cur], h->plane,
                                                            h->pitch, h->fnx, h->fny, h->p.U0);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  if (st) return st;
  CK(cudaStreamSynchronize(h->stream));
  h->have_state = true;
  h->steps = 0;
  h->shifts = 0;
  h->cur_tip = 1;
  h->t = 0.0;
  h->intR = 0.0;
  if (!h->Gt.empty()) h->lT_tilde = thermal_length(h->p, h->Gt[0]);
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_prestep(cupf_ek2d_handle* h) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->have_state) return cupf_fail(CUPF_ERR_STATE, "prestep before set_state");
  if (h->t_mac.empty()) return cupf_fail(CUPF_ERR_STATE, "prestep before set_thermal");
  CK(cudaSetDevice(h->device));
  // rhs_psi at PF.cu:745: pulling distance 0, thermal length of the first gradient
  const double intR = h->intR, lT = h->lT_tilde;
  h->intR = 0.0;
  h->lT_tilde = thermal_length(h->p, h->Gt[0]);
  cupf_status st = launch_step(h, 1, 0u);
  if (st) {
    h->intR = intR;
    h->lT_tilde = lT;
    return st;
  }
  h->cur ^= 1;
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_step(cupf_ek2d_handle* h, int32_t nsteps) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->have_state) return cupf_fail(CUPF_ERR_STATE, "step before set_state");
  if (h->t_mac.empty()) return cupf_fail(CUPF_ERR_STATE, "step before set_thermal");
  if (nsteps < 0) return cupf_fail(CUPF_ERR_INVALID, "nsteps < 0");
  CK(cudaSetDevice(h->device));
  const cupf_ek2d_params& p = h->p;
  for (int n = 0; n < nsteps; ++n) {
    // varGR before step m (PF.cu:794, 805): t = m*dt*tau0, intR += R*tau0/W0*dt
    const int64_t m = h->steps + 1;
    const double t = (double)m * (double)p.dt * (double)p.tau0;
    double R, G;
    table_at(h, t, &R, &G);
    h->intR += (R * (double)p.tau0 / (double)p.W0) * (double)p.dt;
    h->lT_tilde = thermal_length(p, G);
    h->t = t;
    cupf_status st = launch_step(h, 0, (uint32_t)m);
    if (st) return st;
    h->cur ^= 1;
    h->steps = m;
    if (m % p.tipp == 0) {
      st = tip_and_frame(h);
      if (st) return st;
    }
  }
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_get_state(cupf_ek2d_handle* h, float* psi, float* phi, float* U,
                                           float* dpsi) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->have_state) return cupf_fail(CUPF_ERR_STATE, "get_state before set_state");
  CK(cudaSetDevice(h->device));
  const size_t n = (size_t)h->fnx * h->fny;
  float* d[4] = {h->stage, h->stage + n, h->stage + 2 * n, h->stage + 3 * n};
  cupf_status st = with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    ek2d_export_kernel<S, float><<<grid_1d((long long)n), 256, 0, h->stream>>>(
        h->buf[h->cur], h->plane, h->pitch, h->fnx, h->fny, h->p.U0, h->p.sqrt2, psi ? d[0] : nullptr,
        phi ? d[1] : nullptr, U ? d[2] : nullptr, dpsi ? d[3] : nullptr);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  if (st) return st;
  float* host[4] = {psi, phi, U, dpsi};
  for (int f = 0; f < 4; ++f)
    if (host[f]) CK(cudaMemcpyAsync(host[f], d[f], n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_get_state_f64(cupf_ek2d_handle* h, double* psi, double* phi,
                                               double* U, double* dpsi) {
  if (!h) return cupf_fail(CUPF_ERR_INVALID, "null handle");
  if (!h->have_state) return cupf_fail(CUPF_ERR_STATE, "get_state before set_state");
  CK(cudaSetDevice(h->device));
  const size_t n = (size_t)h->fnx * h->fny;
  double* d = nullptr;
  CK(cudaMalloc((void**)&d, 4 * n * sizeof(double)));
  double* part[4] = {d, d + n, d + 2 * n, d + 3 * n};
  cupf_status st = with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    ek2d_export_kernel<S, double><<<grid_1d((long long)n), 256, 0, h->stream>>>(
        h->buf[h->cur], h->plane, h->pitch, h->fnx, h->fny, h->p.U0, h->p.sqrt2,
        psi ? part[0] : nullptr, phi ? part[1] : nullptr, U ? part[2] : nullptr,
        dpsi ? part[3] : nullptr);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  double* host[4] = {psi, phi, U, dpsi};
  for (int f = 0; f < 4 && !st; ++f)
    if (host[f]) {
      cudaError_t e = cudaMemcpyAsync(host[f], part[f], n * sizeof(double), cudaMemcpyDeviceToHost,
                                      h->stream);
      if (e != cudaSuccess) st = cupf_fail(CUPF_ERR_CUDA, "copy out: %s", cudaGetErrorString(e));
    }
  cudaError_t e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (st) return st;
  if (e != cudaSuccess) return cupf_fail(CUPF_ERR_CUDA, "sync: %s", cudaGetErrorString(e));
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_get_y(cupf_ek2d_handle* h, double* y) {
  if (!h || !y) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  const double dxd = (double)h->p.dx * (double)h->p.W0;
  for (int j = 0; j < h->fny; ++j) y[j] = h->p.y0 + ((double)(j - 1) + (double)h->shifts) * dxd;
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_info_get(cupf_ek2d_handle* h, cupf_ek2d_info* info) {
  if (!h || !info) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  info->steps = h->steps;
  info->shifts = h->shifts;
  info->cur_tip = h->cur_tip;
  info->tip_thres = h->tip_thres;
  info->t = h->t;
  info->intR = h->intR;
  info->lT_tilde = h->lT_tilde;
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_row_means(cupf_ek2d_handle* h, double* meanx) {
  if (!h || !meanx) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  if (!h->have_state) return cupf_fail(CUPF_ERR_STATE, "row_means before set_state");
  CK(cudaSetDevice(h->device));
  cupf_status st = with_ek_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    ek2d_row_sums_kernel<S><<<h->fny, 256, 0, h->stream>>>(h->buf[h->cur], h->pitch, h->fnx,
                                                          h->p.sqrt2, h->d_rows);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  if (st) return st;
  CK(cudaMemcpyAsync(meanx, h->d_rows, h->fny * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int j = 0; j < h->fny; ++j) meanx[j] /= h->fnx;
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_time_steps(cupf_ek2d_handle* h, int32_t nsteps, float* ms) {
  if (!h || !ms) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaEventRecord(h->ev0, h->stream));
  cupf_status st = cupf_ek2d_step(h, nsteps);
  if (st) return st;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_stream(cupf_ek2d_handle* h, void** stream) {
  if (!h || !stream) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  *stream = (void*)h->stream;
  return CUPF_OK;
}
