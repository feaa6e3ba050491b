// cupf_server.cu — continuous-batching server of APT simulations (include/cupf.h).
//
// Requests (independent simulations of any grid size) wait in a FIFO queue.
// Each pump of the server:
//   1. retires simulations that reached their step target: argmax map,
//      per-grain volumes and FP64 interface sums go to host memory and the
//      device memory is released;
//   2. admits queued requests while a slot and HBM within the budget are free:
//      buffers, tensor maps, inputs and the initial state go to the device;
//   3. when the resident set changed, rebuilds the work-item list (every
//      (simulation, column tile, z chunk)) and captures a CUDA graph of
//      steps_per_round (batched step, finish) launch pairs;
//   4. replays the graph: every resident simulation advances together, in one
//      persistent kernel launch per step.
// A simulation retires at its exact target even mid-round (the finish kernel
// deactivates it), so results do not depend on the round length or on what
// else is resident.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "../../include/cupf.h"
#include "apt_aux.cuh"
#include "apt_batch.cuh"
#include "capi_internal.h"

using namespace cupf;

typedef CUresult (*EncodeTiledFn2)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn2 encode_fn() {
  static EncodeTiledFn2 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn2)p;
  }
  return fn;
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

namespace {

enum ReqState { PENDING = 0, RUNNING = 1, DONE = 2, FAILED = 3 };

// A page-locked host buffer the server recycles between requests (a request's
// initial fields and its argmax result): no page faults on refill, and copies
// to and from the device run at full speed without the driver's staging.
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Request {
  int64_t id = 0;
  cupf_apt_params p;
  std::vector<float> x, y, z, sint, cost, orient;
  HostBuf hphi, halpha;  // initial argmax fields, L values each (until retired)
  int64_t nsteps = 0;
  int state = PENDING;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // device
  int slot = -1;
  Grid g;
  void* buf[2] = {nullptr, nullptr};
  float *dx = nullptr, *dy = nullptr, *dz = nullptr, *dsint = nullptr, *dcost = nullptr;
  double* dz64 = nullptr;  // heights in FP64 (16-bit storage)
  float* dorient = nullptr;
  float* dphi = nullptr;
  int* dalpha = nullptr;
  float* ddummy = nullptr;
  uint8_t* dquiet[2] = {nullptr, nullptr};  // quiet-item flags of each buffer
  size_t bytes = 0;
  int zc = 64, ty = 8, ntx = 0, nty = 0, nzc = 0;
  // results
  HostBuf hres;  // argmax grain ids, res_len values
  size_t res_len = 0;
  std::vector<long long> res_volumes;
  double res_qoi[3] = {0, 0, 0};
};

}  // namespace

struct cupf_server {
  cupf_server_config cfg;
  cudaStream_t stream = nullptr;
  int pair_bytes = 8;
  int64_t next_id = 1;
  std::deque<int64_t> queue;
  std::map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<int64_t> slots;  // request id per slot (0 = free)
  size_t used_bytes = 0;
  size_t budget = 0;
  BatchSim* d_sims = nullptr;
  CUtensorMap* d_tmaps = nullptr;
  int4* d_items = nullptr;
  int items_cap = 0;
  int nitems = 0;
  int* d_next = nullptr;
  int* d_err = nullptr;
  unsigned long long* d_counts = nullptr;
  long long* d_first = nullptr;
  int counts_cap = 0;
  double* d_part = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  // the requests' device memory: a stream-ordered pool that keeps what retired
  // requests free for the next admissions (no release to the driver until the
  // server is destroyed), so admitting and retiring cost no device-wide
  // allocation or synchronising free
  cudaMemPool_t pool = nullptr;
  // recycled page-locked host buffers, at most kHostCacheBytes in all
  std::vector<HostBuf> host_cache;
  size_t host_cache_bytes = 0;
  bool dirty = true;
  // (fnx, fny, fnz) -> (tile height, z chunk)
  std::map<std::tuple<int, int, int>, std::pair<int, int>> tile_cache;
  int64_t steps_replayed = 0;
  // device time of the rounds: events around each graph launch, summed when the
  // next pump has waited for it
  cudaEvent_t ev_round[2] = {nullptr, nullptr};
  bool round_open = false;
  double busy_ms = 0;
};

template <class F>
static cupf_status with_fmt(int prec, F&& f) {
  switch (prec) {
    case CUPF_PREC_FP32: return f(PairF32{});
    case CUPF_PREC_BF16: return f(PairBF16{});
    case CUPF_PREC_FP16: return f(PairFP16{});
  }
  return cupf_fail(CUPF_ERR_UNSUPPORTED, "precision %d", prec);
}

static int gridn(long long n) {
  long long b = (n + 255) / 256;
  return (int)std::max(1ll, std::min(b, 148ll * 16));
}

constexpr size_t kHostCacheBytes = (size_t)4 << 30;

// A page-locked host buffer of at least n bytes: the smallest cached one that
// fits, else a new one.
static cupf_status get_host(cupf_server* s, size_t n, HostBuf* out) {
  size_t best = s->host_cache.size();
  for (size_t i = 0; i < s->host_cache.size(); ++i)
    if (s->host_cache[i].cap >= n &&
        (best == s->host_cache.size() || s->host_cache[i].cap < s->host_cache[best].cap))
      best = i;
  if (best < s->host_cache.size()) {
    *out = s->host_cache[best];
    s->host_cache.erase(s->host_cache.begin() + best);
    s->host_cache_bytes -= out->cap;
    return CUPF_OK;
  }
  out->cap = std::max<size_t>(n, 1);
  if (cudaHostAlloc(&out->p, out->cap, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    *out = HostBuf();
    return cupf_fail(CUPF_ERR_OOM, "page-locked host buffer of %zu bytes", n);
  }
  return CUPF_OK;
}

// Give a host buffer back (no copy may still use it): kept for reuse while the
// cache stays under its limit, else freed.
static void put_host(cupf_server* s, HostBuf* b) {
  if (!b->p) return;
  if (s->host_cache_bytes + b->cap <= kHostCacheBytes) {
    s->host_cache.push_back(*b);
    s->host_cache_bytes += b->cap;
  } else {
    cudaFreeHost(b->p);
  }
  *b = HostBuf();
}

// A request's device buffer from the server's pool, ordered on its stream.
static cudaError_t pool_alloc(cupf_server* s, void** p, size_t n) {
  return cudaMallocFromPoolAsync(p, n, s->pool, s->stream);
}

// Return a request's buffers to the pool (ordered after the work queued on the
// server's stream that reads them).
static void free_request_device(cupf_server* s, Request* r) {
  void* ptrs[] = {r->buf[0], r->buf[1], r->dx, r->dy, r->dz, r->dz64, r->dsint, r->dcost, r->dorient, r->dphi,
                  r->dalpha, r->ddummy, r->dquiet[0], r->dquiet[1]};
  for (void* p : ptrs)
    if (p) cudaFreeAsync(p, s->stream);
  r->buf[0] = r->buf[1] = nullptr;
  r->dx = r->dy = r->dz = r->dsint = r->dcost = r->dorient = r->dphi = nullptr;
  r->dz64 = nullptr;
  r->dalpha = nullptr;
  r->ddummy = nullptr;
  r->dquiet[0] = r->dquiet[1] = nullptr;
}

static size_t request_bytes(const cupf_apt_params& p, int pair_bytes, int num_pf) {
  const int palign = pair_bytes == 8 ? 2 : 4;
  const size_t xp = (p.fnx + palign - 1) / palign * palign;
  const size_t L = (size_t)p.fnx * p.fny * p.fnz;
  // quiet flags for the most items a tile shape gives (32x4 tiles, z chunks of 1)
  const size_t quiet = 2 * (size_t)((p.fnx - 2 + TX - 1) / TX) * ((p.fny - 2 + 4 - 1) / 4) * (p.fnz - 2);
  return 2 * xp * p.fny * p.fnz * num_pf * pair_bytes + L * 8 + quiet + 4096;
}

// Pick the work items' tile shape of a grid shape -- the column-tile height
// (32x8 or 32x4) and the z chunk -- by timing the single-simulation step on a
// scratch handle (same shape, precision, slot count) for each candidate.
static std::pair<int, int> autotune_tile(cupf_server* s, const Request* r) {
  const auto key = std::make_tuple(r->p.fnx, r->p.fny, r->p.fnz);
  auto it = s->tile_cache.find(key);
  if (it != s->tile_cache.end()) return it->second;
  const int fixed_ty = s->cfg.tile_y;
  std::pair<int, int> best(fixed_ty ? fixed_ty : 8, 64);
  if (s->cfg.autotune) {
    cupf_apt_inputs in;
    std::memset(&in, 0, sizeof(in));
    in.x = r->x.data();
    in.y = r->y.data();
    in.z = r->z.data();
    in.sint = r->sint.data();
    in.cost = r->cost.data();
    float best_ms = 1e30f;
    const int nz = r->p.fnz - 2;
    const int cand[] = {8, 16, 32, 64, 128, 256};
    cupf_apt_handle* h = nullptr;
    if (cupf_apt_create(&r->p, &in, s->cfg.device, (cupf_precision)s->cfg.precision, &h) ==
        CUPF_OK) {
      for (int ty : {8, 4}) {
        if (fixed_ty && ty != fixed_ty) continue;
        if (cupf_apt_set_tile(h, ty) != CUPF_OK) continue;
        for (int zc : cand) {
          if (zc > 2 * nz && zc != cand[0]) break;
          // the fastest of three timings of 4 steps, after 2 untimed ones (a
          // single short timing picked different chunks from run to run)
          float ms = 1e30f;
          bool ok = cupf_apt_set_tuning(h, zc) == CUPF_OK &&
                    cupf_apt_init_from_argmax(h, static_cast<const float*>(r->hphi.p),
                                              static_cast<const int32_t*>(r->halpha.p)) ==
                        CUPF_OK &&
                    cupf_apt_step(h, 2, 0) == CUPF_OK;
          for (int rep = 0; ok && rep < 3; ++rep) {
            float m = 0;
            ok = cupf_apt_time_steps(h, 4, &m) == CUPF_OK;
            ms = std::min(ms, m);
          }
          if (ok && ms < best_ms) {
            best_ms = ms;
            best = std::make_pair(ty, zc);
          }
        }
      }
      cupf_apt_destroy(h);
    }
  }
  s->tile_cache[key] = best;
  return best;
}

static cupf_status admit(cupf_server* s, Request* r, int slot) {
  const cupf_apt_params& p = r->p;
  const int np = s->cfg.num_pf;
  const int palign = s->pair_bytes == 8 ? 2 : 4;
  r->g.fnx = p.fnx;
  r->g.fny = p.fny;
  r->g.fnz = p.fnz;
  r->g.np = np;
  r->g.xp = (p.fnx + palign - 1) / palign * palign;
  r->g.ss = (long long)r->g.xp * p.fny * p.fnz;
  const std::pair<int, int> tile = autotune_tile(s, r);
  r->ty = tile.first;
  r->zc = tile.second;
  const int nz = p.fnz - 2;
  r->zc = std::min(r->zc, nz);
  r->ntx = (p.fnx - 2 + TX - 1) / TX;
  r->nty = (p.fny - 2 + r->ty - 1) / r->ty;
  r->nzc = (nz + r->zc - 1) / r->zc;
  const size_t bb = (size_t)r->g.ss * np * s->pair_bytes;
  const size_t L = (size_t)p.fnx * p.fny * p.fnz;
  const int nth = 2 * p.num_theta + 1;
  cudaStream_t st = s->stream;
  auto up = [&](float** d, const std::vector<float>& h) -> cupf_status {
    CK(pool_alloc(s, (void**)d, h.size() * sizeof(float)));
    CK(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    return CUPF_OK;
  };
  for (int b = 0; b < 2; ++b) CK(pool_alloc(s, &r->buf[b], bb));
  cupf_status e;
  if ((e = up(&r->dx, r->x)) || (e = up(&r->dy, r->y)) || (e = up(&r->dz, r->z)) ||
      (e = up(&r->dsint, r->sint)) || (e = up(&r->dcost, r->cost)) ||
      (e = up(&r->dorient, r->orient)))
    return e;
  CK(pool_alloc(s, (void**)&r->dphi, L * sizeof(float)));
  CK(cudaMemcpyAsync(r->dphi, r->hphi.p, L * sizeof(float), cudaMemcpyHostToDevice, st));
  (void)nth;
  {
    std::vector<double> z64(r->z.begin(), r->z.end());
    CK(pool_alloc(s, (void**)&r->dz64, z64.size() * sizeof(double)));
    CK(cudaMemcpyAsync(r->dz64, z64.data(), z64.size() * sizeof(double), cudaMemcpyHostToDevice,
                       st));
  }
  CK(pool_alloc(s, (void**)&r->dalpha, L * sizeof(int)));
  CK(cudaMemcpyAsync(r->dalpha, r->halpha.p, L * sizeof(int), cudaMemcpyHostToDevice, st));
  CK(pool_alloc(s, (void**)&r->ddummy, 64 * sizeof(float)));
  CK(cudaMemsetAsync(r->ddummy, 0, 64 * sizeof(float), st));
  const size_t nq = (size_t)r->ntx * r->nty * r->nzc;
  for (int b = 0; b < 2; ++b) {
    CK(pool_alloc(s, (void**)&r->dquiet[b], nq));
    CK(cudaMemsetAsync(r->dquiet[b], 0, nq, st));
  }
  r->bytes = request_bytes(p, s->pair_bytes, np);
  // initial state in both buffers
  e = with_fmt(s->cfg.precision, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    init_kernel<S><<<gridn(L), 256, 0, st>>>(static_cast<typename S::T*>(r->buf[0]),
                                             static_cast<typename S::T*>(r->buf[1]), r->dphi,
                                             r->dalpha, r->g);
    // the step reads x/y halo cells from the buffer: fill them on both
    const long long nh = 2ll * r->g.fnx * r->g.fny + 2ll * r->g.fnx * (r->g.fnz - 2) +
                         2ll * (r->g.fny - 2) * (r->g.fnz - 2);
    for (int b = 0; b < 2; ++b)
      fill_halo_kernel<S><<<gridn(nh), 256, 0, st>>>(static_cast<typename S::T*>(r->buf[b]), r->g,
                                                     p.bcX, p.bcY, p.bcZ);
    CK(cudaGetLastError());
    // tensor maps of both buffers
    EncodeTiledFn2 enc = encode_fn();
    if (!enc) return cupf_fail(CUPF_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    CUtensorMap tm[2];
    for (int b = 0; b < 2; ++b) {
      const cuuint64_t eb = S::kBytes;
      cuuint64_t dims[4] = {(cuuint64_t)p.fnx, (cuuint64_t)p.fny, (cuuint64_t)p.fnz,
                            (cuuint64_t)np};
      cuuint64_t strides[3] = {(cuuint64_t)r->g.xp * eb, (cuuint64_t)r->g.xp * p.fny * eb,
                               (cuuint64_t)r->g.ss * eb};
      cuuint32_t box[4] = {(cuuint32_t)S::kBW, (cuuint32_t)(r->ty + 2), 1u, (cuuint32_t)np};
      cuuint32_t es[4] = {1, 1, 1, 1};
      if (enc(&tm[b], S::kTmaType, 4, r->buf[b], dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cupf_fail(CUPF_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    }
    CK(cudaMemcpyAsync(s->d_tmaps + 2 * slot, tm, sizeof(tm), cudaMemcpyHostToDevice, st));
    return CUPF_OK;
  });
  if (e) return e;
  BatchSim bs;
  std::memset(&bs, 0, sizeof(bs));
  StepArgs& a = bs.a;
  a.fnx = p.fnx;
  a.fny = p.fny;
  a.fnz = p.fnz;
  a.xp = r->g.xp;
  a.slot_stride = r->g.ss;
  a.bcX = p.bcX;
  a.bcY = p.bcY;
  a.bcZ = p.bcZ;
  a.ntx = r->ntx;
  a.nty = r->nty;
  a.nzc = r->nzc;
  a.zc = r->zc;
  a.num_theta = p.num_theta;
  {
    const InvariantDivisor dv = invariant_divisor((uint32_t)p.num_theta);
    a.nt_magic = dv.m;
    a.nt_sh1 = dv.s1;
    a.nt_sh2 = dv.s2;
  }
  a.thermalType = p.thermalType;
  a.kin_delta = p.kin_delta;
  a.eps = p.eps;
  a.G = p.G;
  a.z0 = p.z0;
  a.uc = p.underCoolingRate;
  a.uc0 = p.underCoolingRate0;
  a.L_cp = p.L_cp;
  a.hi = p.hi;
  a.lamd = p.lamd;
  a.dt = p.dt;
  a.tau0 = p.tau0;
  a.lyd = p.lyd;
  a.lzd = p.lzd;
  a.r0 = p.r0;
  a.x0 = p.x0;
  a.angle = p.angle;
  a.V = p.V;
  a.mp_len = p.mp_len;
  a.order = p.order;
  a.Nx = 2;
  a.Ny = 2;
  a.Nz = 2;
  a.x = r->dx;
  a.y = r->dy;
  a.z = r->dz;
  a.z64 = r->dz64;
  a.fp64 = s->cfg.precision != CUPF_PREC_FP32;
  a.sint = r->dsint;
  a.cost = r->dcost;
  a.orient = reinterpret_cast<const float4*>(r->dorient);
  a.X_mac = r->ddummy;
  a.Y_mac = r->ddummy;
  a.Z_mac = r->ddummy;
  a.psi_mac = r->ddummy;
  a.err = s->d_err;
  a.wait_limit = kWaitCycles;
  bs.buf[0] = r->buf[0];
  bs.buf[1] = r->buf[1];
  bs.quiet[0] = r->dquiet[0];
  bs.quiet[1] = r->dquiet[1];
  bs.steps = 0;
  bs.target = r->nsteps;
  bs.cur = 0;
  bs.active = r->nsteps > 0 ? 1 : 0;
  CK(cudaMemcpyAsync(s->d_sims + slot, &bs, sizeof(bs), cudaMemcpyHostToDevice, st));
  r->slot = slot;
  r->state = RUNNING;
  r->t_admit = now_s();
  s->slots[slot] = r->id;
  s->used_bytes += r->bytes;
  s->dirty = true;
  return CUPF_OK;
}

static cupf_status retire(cupf_server* s, Request* r, int cur) {
  cudaStream_t st = s->stream;
  const size_t L = (size_t)r->g.length();
  const int ng = r->p.num_theta;
  // argmax map (cleared first), volumes, FP64 interface sums of the final state
  CK(cudaMemsetAsync(r->dphi, 0, L * sizeof(float), st));
  CK(cudaMemsetAsync(r->dalpha, 0, L * sizeof(int), st));
  if (s->counts_cap < ng + 1) {
    if (s->d_counts) cudaFree(s->d_counts);
    if (s->d_first) cudaFree(s->d_first);
    CK(cudaMalloc((void**)&s->d_counts, (ng + 1) * sizeof(unsigned long long)));
    CK(cudaMalloc((void**)&s->d_first, (ng + 1) * sizeof(long long)));
    s->counts_cap = ng + 1;
  }
  CK(cudaMemsetAsync(s->d_counts, 0, (ng + 1) * sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(s->d_first, 0x7F, (ng + 1) * sizeof(long long), st));
  const int nb = 148 * 4;
  const Grid& g = r->g;
  cupf_status e = with_fmt(s->cfg.precision, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    auto* b = static_cast<typename S::T*>(r->buf[cur]);
    const long long nh =
        2ll * g.fnx * g.fny + 2ll * g.fnx * (g.fnz - 2) + 2ll * (g.fny - 2) * (g.fnz - 2);
    fill_halo_kernel<S><<<gridn(nh), 256, 0, st>>>(b, g, r->p.bcX, r->p.bcY, r->p.bcZ);
    collect_kernel<S><<<gridn(L), 256, 0, st>>>(b, r->dphi, r->dalpha, g);
    const long long ni = (long long)(g.fnx - 2) * (g.fny - 2) * (g.fnz - 2);
    volume_kernel<<<gridn(ni), 256, 0, st>>>(r->dalpha, g.fnx, g.fny, g.fnz, ng, s->d_counts,
                                             s->d_first);
    qoi_sums_kernel<S><<<nb, 256, 0, st>>>(b, g, s->d_part);
    CK(cudaGetLastError());
    return CUPF_OK;
  });
  if (e) return e;
  cupf_status he = get_host(s, L * sizeof(int), &r->hres);
  if (he) return he;
  r->res_len = L;
  std::vector<unsigned long long> c(ng + 1);
  std::vector<double> part(2 * nb);
  CK(cudaMemcpyAsync(r->hres.p, r->dalpha, L * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(c.data(), s->d_counts, c.size() * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(part.data(), s->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                     st));
  CK(cudaStreamSynchronize(st));
  r->res_volumes.assign(c.begin(), c.end());
  double v = 0, a = 0;
  for (int b2 = 0; b2 < nb; ++b2) {
    v += part[2 * b2];
    a += part[2 * b2 + 1];
  }
  r->res_qoi[0] = v;
  r->res_qoi[1] = a;
  r->res_qoi[2] = v / ((double)(g.fnx - 2) * (g.fny - 2));
  free_request_device(s, r);
  s->used_bytes -= r->bytes;
  s->slots[r->slot] = 0;
  r->slot = -1;
  r->state = DONE;
  r->t_done = now_s();
  r->x.clear();
  // the uploads of the initial fields finished long ago (the stream was waited on)
  put_host(s, &r->hphi);
  put_host(s, &r->halpha);
  s->dirty = true;
  return CUPF_OK;
}

// Work items of every resident simulation, grouped by tile height (32x8 first,
// then 32x4): per step one persistent batched launch per group present, each
// with its own range of the item list and its own work counter, then the
// finish kernel.
static const int kTileHeights[2] = {8, 4};

static cupf_status rebuild(cupf_server* s) {
  std::vector<int4> items;
  int off[3] = {0, 0, 0};
  for (int gi = 0; gi < 2; ++gi) {
    off[gi] = (int)items.size();
    for (size_t slot = 0; slot < s->slots.size(); ++slot) {
      if (!s->slots[slot]) continue;
      const Request* r = s->reqs[s->slots[slot]].get();
      if (r->ty != kTileHeights[gi]) continue;
      for (int tyi = 0; tyi < r->nty; ++tyi)
        for (int txi = 0; txi < r->ntx; ++txi)
          for (int zci = 0; zci < r->nzc; ++zci)
            items.push_back(make_int4((int)slot, txi, tyi, zci));
    }
  }
  off[2] = (int)items.size();
  s->nitems = (int)items.size();
  if (s->nitems > s->items_cap) {
    if (s->d_items) cudaFree(s->d_items);
    s->items_cap = std::max(s->nitems, 2 * s->items_cap);
    CK(cudaMalloc((void**)&s->d_items, s->items_cap * sizeof(int4)));
  }
  if (s->nitems)
    CK(cudaMemcpyAsync(s->d_items, items.data(), items.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemsetAsync(s->d_next, 0, 4 * sizeof(int), s->stream));
  if (s->gexec) {
    cudaGraphExecDestroy(s->gexec);
    s->gexec = nullptr;
  }
  if (s->graph) {
    cudaGraphDestroy(s->graph);
    s->graph = nullptr;
  }
  if (!s->nitems) {
    s->dirty = false;
    return CUPF_OK;
  }
  // persistent grids: the resident CTAs of each step kernel, never more than items
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->cfg.device);
  const int nsims = (int)s->slots.size();
  cupf_status e = with_fmt(s->cfg.precision, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    switch (s->cfg.num_pf) {
#define CASE(N)                                                                                 \
  case N: {                                                                                     \
    int grid[2] = {0, 0};                                                                       \
    const int bytes8 = StepSmem<N, S, 8>::kBytes, bytes4 = StepSmem<N, S, 4>::kBytes;           \
    CK(cudaFuncSetAttribute(apt_batch_step_kernel<N, S, 8>,                                     \
                            cudaFuncAttributeMaxDynamicSharedMemorySize, bytes8));              \
    CK(cudaFuncSetAttribute(apt_batch_step_kernel<N, S, 4>,                                     \
                            cudaFuncAttributeMaxDynamicSharedMemorySize, bytes4));              \
    for (int gi = 0; gi < 2; ++gi) {                                                            \
      int per_sm = 2;                                                                           \
      if (gi == 0)                                                                              \
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                       \
            &per_sm, apt_batch_step_kernel<N, S, 8>, tile_threads<8>(), bytes8));               \
      else                                                                                      \
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                       \
            &per_sm, apt_batch_step_kernel<N, S, 4>, tile_threads<4>(), bytes4));               \
      grid[gi] = std::min(off[gi + 1] - off[gi], std::max(1, per_sm) * nsm);                    \
    }                                                                                           \
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));                    \
    for (int k = 0; k < s->cfg.steps_per_round; ++k) {                                          \
      if (grid[0] > 0)                                                                          \
        apt_batch_step_kernel<N, S, 8><<<grid[0], tile_threads<8>(), bytes8, s->stream>>>(      \
            s->d_sims, s->d_tmaps, s->d_items + off[0], off[1] - off[0], s->d_next, s->d_err);  \
      if (grid[1] > 0)                                                                          \
        apt_batch_step_kernel<N, S, 4><<<grid[1], tile_threads<4>(), bytes4, s->stream>>>(      \
            s->d_sims, s->d_tmaps, s->d_items + off[1], off[2] - off[1], s->d_next + 2,         \
            s->d_err);                                                                          \
      batch_finish_kernel<<<(nsims + 127) / 128, 128, 0, s->stream>>>(s->d_sims, nsims);        \
    }                                                                                           \
    CK(cudaStreamEndCapture(s->stream, &s->graph));                                             \
    return CUPF_OK;                                                                             \
  }
      CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
#undef CASE
      default:
        return cupf_fail(CUPF_ERR_UNSUPPORTED, "num_pf=%d not built", s->cfg.num_pf);
    }
  });
  if (e) return e;
  CK(cudaGraphInstantiate(&s->gexec, s->graph, 0));
  s->dirty = false;
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_create(const cupf_server_config* cfg, cupf_server** out) {
  if (!cfg || !out) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  *out = nullptr;
  if (cfg->num_pf < 1 || cfg->num_pf > 8)
    return cupf_fail(CUPF_ERR_UNSUPPORTED, "num_pf=%d not built (1..8)", cfg->num_pf);
  if (cfg->max_active < 1 || cfg->max_active > 4096)
    return cupf_fail(CUPF_ERR_INVALID, "max_active must be in 1..4096");
  if (cfg->steps_per_round < 1) return cupf_fail(CUPF_ERR_INVALID, "steps_per_round must be >= 1");
  if (cfg->tile_y != 0 && !tile_height_built(cfg->tile_y))
    return cupf_fail(CUPF_ERR_INVALID, "tile_y must be 0, 4 or 8");
  if (cfg->precision < 0 || cfg->precision > 2)
    return cupf_fail(CUPF_ERR_UNSUPPORTED, "precision %d", cfg->precision);
  std::unique_ptr<cupf_server> s(new cupf_server());
  s->cfg = *cfg;
  s->pair_bytes = cfg->precision == CUPF_PREC_FP32 ? 8 : 4;
  CK(cudaSetDevice(cfg->device));
  CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = cfg->device;
    CK(cudaMemPoolCreate(&s->pool, &props));
    uint64_t keep = UINT64_MAX;  // hold freed memory for reuse until destroy
    CK(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  CK(cudaEventCreate(&s->ev_round[0]));
  CK(cudaEventCreate(&s->ev_round[1]));
  s->slots.assign(cfg->max_active, 0);
  CK(cudaMalloc((void**)&s->d_sims, cfg->max_active * sizeof(BatchSim)));
  CK(cudaMemset(s->d_sims, 0, cfg->max_active * sizeof(BatchSim)));
  CK(cudaMalloc((void**)&s->d_tmaps, 2 * cfg->max_active * sizeof(CUtensorMap)));
  CK(cudaMalloc((void**)&s->d_next, 4 * sizeof(int)));  // a work counter pair per tile height
  CK(cudaMemset(s->d_next, 0, 4 * sizeof(int)));
  CK(cudaMalloc((void**)&s->d_err, sizeof(int)));
  CK(cudaMemset(s->d_err, 0, sizeof(int)));
  CK(cudaMalloc((void**)&s->d_part, 2 * 148 * 4 * sizeof(double)));
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  const size_t reserve = (size_t)2 << 30;
  const size_t avail = fr > reserve ? fr - reserve : 0;
  s->budget = cfg->hbm_budget_bytes > 0 ? std::min((size_t)cfg->hbm_budget_bytes, avail) : avail;
  *out = s.release();
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_destroy(cupf_server* s) {
  if (!s) return cupf_fail(CUPF_ERR_INVALID, "null server");
  cudaSetDevice(s->cfg.device);
  cudaStreamSynchronize(s->stream);
  for (auto& kv : s->reqs) free_request_device(s, kv.second.get());
  cudaStreamSynchronize(s->stream);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  for (auto& kv : s->reqs)
    for (HostBuf* b : {&kv.second->hphi, &kv.second->halpha, &kv.second->hres})
      if (b->p) cudaFreeHost(b->p);
  for (HostBuf& b : s->host_cache) cudaFreeHost(b.p);
  for (cudaEvent_t e : s->ev_round)
    if (e) cudaEventDestroy(e);
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  if (s->graph) cudaGraphDestroy(s->graph);
  void* ptrs[] = {s->d_sims, s->d_tmaps, s->d_items, s->d_next, s->d_err, s->d_counts, s->d_first,
                  s->d_part};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  cudaStreamDestroy(s->stream);
  delete s;
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_submit(cupf_server* s, const cupf_apt_params* p,
                                          const cupf_apt_inputs* in, const float* phi,
                                          const int32_t* alpha, int64_t nsteps,
                                          int64_t* request_id) {
  if (!s || !p || !in || !phi || !alpha || !request_id)
    return cupf_fail(CUPF_ERR_INVALID, "null argument");
  if (p->num_pf != s->cfg.num_pf)
    return cupf_fail(CUPF_ERR_INVALID, "request num_pf %d != server num_pf %d", p->num_pf,
                     s->cfg.num_pf);
  if (p->fnx < 4 || p->fny < 4 || p->fnz < 4 || p->num_theta < 1 || p->haloWidth != 1)
    return cupf_fail(CUPF_ERR_INVALID, "bad grid or grain count");
  if (p->thermalType != 0 && p->thermalType != 1 && p->thermalType != 2)
    return cupf_fail(CUPF_ERR_UNSUPPORTED, "the server runs thermal types 0-2");
  if (s->cfg.precision != CUPF_PREC_FP32 && p->num_theta > 32767)
    return cupf_fail(CUPF_ERR_UNSUPPORTED, "16-bit storage needs num_theta <= 32767");
  if (!in->x || !in->y || !in->z || !in->sint || !in->cost)
    return cupf_fail(CUPF_ERR_INVALID, "x, y, z, sint and cost are required");
  if (nsteps < 0) return cupf_fail(CUPF_ERR_INVALID, "nsteps < 0");
  const size_t need = request_bytes(*p, s->pair_bytes, s->cfg.num_pf);
  if (need > s->budget)
    return cupf_fail(CUPF_ERR_OOM, "request needs %zu bytes, budget is %zu", need, s->budget);
  std::unique_ptr<Request> r(new Request());
  r->id = s->next_id++;
  r->p = *p;
  r->x.assign(in->x, in->x + p->fnx);
  r->y.assign(in->y, in->y + p->fny);
  r->z.assign(in->z, in->z + p->fnz);
  const int nth = 2 * p->num_theta + 1;
  r->sint.assign(in->sint, in->sint + nth);
  r->cost.assign(in->cost, in->cost + nth);
  r->orient.resize(4 * (size_t)(p->num_theta + 1));
  pack_orientations(in->sint, in->cost, p->num_theta, r->orient.data());
  const size_t L = (size_t)p->fnx * p->fny * p->fnz;
  cupf_status e;
  if ((e = get_host(s, L * sizeof(float), &r->hphi))) return e;
  if ((e = get_host(s, L * sizeof(int32_t), &r->halpha))) {
    put_host(s, &r->hphi);
    return e;
  }
  std::memcpy(r->hphi.p, phi, L * sizeof(float));
  std::memcpy(r->halpha.p, alpha, L * sizeof(int32_t));
  r->nsteps = nsteps;
  r->t_submit = now_s();
  *request_id = r->id;
  s->queue.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_pump(cupf_server* s, int32_t* n_running, int32_t* n_pending,
                                        int32_t* n_done) {
  if (!s) return cupf_fail(CUPF_ERR_INVALID, "null server");
  CK(cudaSetDevice(s->cfg.device));
  cupf_status e;
  // 1. retire finished simulations
  std::vector<BatchSim> host(s->slots.size());
  CK(cudaMemcpyAsync(host.data(), s->d_sims, host.size() * sizeof(BatchSim),
                     cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (s->round_open) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, s->ev_round[0], s->ev_round[1]));
    s->busy_ms += ms;
    s->round_open = false;
  }
  int err = 0;
  CK(cudaMemcpy(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return cupf_fail(CUPF_ERR_TIMEOUT, "batched step reported error %d", err);
  for (size_t slot = 0; slot < s->slots.size(); ++slot) {
    if (!s->slots[slot]) continue;
    Request* r = s->reqs[s->slots[slot]].get();
    if (!host[slot].active && host[slot].steps >= r->nsteps)
      if ((e = retire(s, r, host[slot].cur))) return e;
  }
  // 2. admit from the queue (FIFO) while a slot and memory are free
  while (!s->queue.empty()) {
    Request* r = s->reqs[s->queue.front()].get();
    int slot = -1;
    for (size_t k = 0; k < s->slots.size(); ++k)
      if (!s->slots[k]) {
        slot = (int)k;
        break;
      }
    const size_t need = request_bytes(r->p, s->pair_bytes, s->cfg.num_pf);
    if (slot < 0 || s->used_bytes + need > s->budget) break;
    s->queue.pop_front();
    if ((e = admit(s, r, slot))) {
      free_request_device(s, r);
      r->state = FAILED;
      return e;
    }
  }
  // 3. re-plan and capture when the resident set changed
  if (s->dirty && (e = rebuild(s))) return e;
  // 4. advance every resident simulation steps_per_round steps
  // (not waited for here: the next pump's read-back of the simulation states
  // waits, so the caller's work between rounds overlaps the device)
  if (s->gexec) {
    CK(cudaEventRecord(s->ev_round[0], s->stream));
    CK(cudaGraphLaunch(s->gexec, s->stream));
    CK(cudaEventRecord(s->ev_round[1], s->stream));
    s->round_open = true;
    s->steps_replayed += s->cfg.steps_per_round;
  }
  int running = 0, done = 0;
  for (auto& kv : s->reqs) {
    running += kv.second->state == RUNNING;
    done += kv.second->state == DONE;
  }
  if (n_running) *n_running = running;
  if (n_pending) *n_pending = (int32_t)s->queue.size();
  if (n_done) *n_done = done;
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_result(cupf_server* s, int64_t id, int32_t* status,
                                          int32_t* alpha_out, int64_t* volumes_out,
                                          int32_t num_grains, double* qoi_out, double* times_out) {
  if (!s || !status) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return cupf_fail(CUPF_ERR_INVALID, "unknown request %lld", (long long)id);
  Request* r = it->second.get();
  *status = r->state;
  if (r->state != DONE) return CUPF_OK;
  if (alpha_out && r->hres.p) std::memcpy(alpha_out, r->hres.p, r->res_len * sizeof(int));
  if (volumes_out) {
    const int n = std::min<int>(num_grains + 1, (int)r->res_volumes.size());
    for (int i = 0; i < n; ++i) volumes_out[i] = r->res_volumes[i];
  }
  if (qoi_out) std::memcpy(qoi_out, r->res_qoi, sizeof(r->res_qoi));
  if (times_out) {
    times_out[0] = r->t_submit;
    times_out[1] = r->t_admit;
    times_out[2] = r->t_done;
  }
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_stats(cupf_server* s, double* busy_ms, int64_t* rounds) {
  if (!s) return cupf_fail(CUPF_ERR_INVALID, "null server");
  if (busy_ms) *busy_ms = s->busy_ms;
  if (rounds) *rounds = s->steps_replayed / std::max(1, (int)s->cfg.steps_per_round);
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_request_tile(cupf_server* s, int64_t id, int32_t* tile_y,
                                                int32_t* z_chunk) {
  if (!s) return cupf_fail(CUPF_ERR_INVALID, "null server");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return cupf_fail(CUPF_ERR_INVALID, "unknown request");
  const Request* r = it->second.get();
  const bool placed = r->state != PENDING;
  if (tile_y) *tile_y = placed ? r->ty : 0;
  if (z_chunk) *z_chunk = placed ? r->zc : 0;
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_set_tile(cupf_server* s, int32_t tile_y) {
  if (!s) return cupf_fail(CUPF_ERR_INVALID, "null server");
  if (tile_y != 0 && !tile_height_built(tile_y))
    return cupf_fail(CUPF_ERR_INVALID, "tile_y must be 0, 4 or 8");
  s->cfg.tile_y = tile_y;
  s->tile_cache.clear();
  return CUPF_OK;
}

extern "C" cupf_status cupf_server_release(cupf_server* s, int64_t id) {
  if (!s) return cupf_fail(CUPF_ERR_INVALID, "null server");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return cupf_fail(CUPF_ERR_INVALID, "unknown request");
  if (it->second->state == RUNNING) return cupf_fail(CUPF_ERR_STATE, "request still running");
  if (it->second->state == PENDING) {
    auto q = std::find(s->queue.begin(), s->queue.end(), id);
    if (q != s->queue.end()) s->queue.erase(q);
  }
  Request* r = it->second.get();
  // a request that failed during admission may still have an upload queued
  if (r->state == FAILED) CK(cudaStreamSynchronize(s->stream));
  put_host(s, &r->hphi);
  put_host(s, &r->halpha);
  put_host(s, &r->hres);
  s->reqs.erase(it);
  return CUPF_OK;
}
