// cupf_capi.cu — C ABI of the B200 APT solver (include/cupf.h).
//
// Owns the device state of one simulation: two pair-plane buffers (ping-pong),
// their TMA tensor maps, coordinates / orientation tables, the argmax fields,
// the moving-domain archive and one CUDA stream.  Every call checks every CUDA
// return code and maps failures to a cupf_status with a per-thread message.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cupf.h"
#include "apt_aux.cuh"
#include "apt_nucl.cuh"
#include "capi_internal.h"
#include "apt_step.cuh"

using namespace cupf;

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

cupf_status cupf_fail(cupf_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}

#define fail cupf_fail

extern "C" const char* cupf_last_error(void) { return g_err.c_str(); }
extern "C" int cupf_abi_version(void) { return CUPF_ABI_VERSION; }
extern "C" size_t cupf_struct_size(int which) {
  return which == 0 ? sizeof(cupf_apt_params) : which == 1 ? sizeof(cupf_apt_inputs) : 0;
}

// ------------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// ------------------------------------------------------------------ handle
struct cupf_apt_handle {
  cupf_apt_params p;
  int device = 0;
  cupf_precision prec = CUPF_PREC_FP32;
  Grid g;
  int pair_bytes = 8;
  void* buf[2] = {nullptr, nullptr};
  CUtensorMap tmap[2];
  int cur = 0;  // buffer holding the current state
  int64_t steps_done = 0;
  bool initialised = false;
  cudaStream_t stream = nullptr;
  // device inputs
  float *x = nullptr, *y = nullptr, *z = nullptr, *sint = nullptr, *cost = nullptr;
  double* z64 = nullptr;             // z in FP64 (16-bit storage: FP64 time and heights)
  std::vector<double> z64_host;
  float* orient = nullptr;  // packed orientation table (pack_orientations)
  float *X_mac = nullptr, *Y_mac = nullptr, *Z_mac = nullptr, *t_mac = nullptr;
  float *psi_mac = nullptr, *T_3D = nullptr;
  bool has_T3D = false;
  std::vector<float> z_host;
  // argmax fields (reference layout, length)
  float* phi_m = nullptr;
  int* alpha_m = nullptr;
  int* err = nullptr;
  int* work = nullptr;  // persistent-launch work counter [next, done]
  int grid_cap = 0;     // resident CTAs of the step kernel (occupancy x SMs)
  // quiet-item flags of each buffer (StepArgs::quiet_in/out), sized for the
  // finest item grid (z chunks of one plane); all 0 = nothing known
  uint8_t* quiet[2] = {nullptr, nullptr};
  size_t quiet_cap = 0;
  bool skip_quiet = true;
  long long wait_limit = kWaitCycles;  // stage-wait bound of the step kernel (SM cycles)
  bool zc_user = false;  // z chunk fixed by the caller (set_tuning or CUPF_ZC)
  unsigned long long* active_cells = nullptr;
  unsigned long long* overflows = nullptr;  // merge overflows: [0] aliased, [1] dropped
  // read-back scratch (reference layout, num_pf * length), allocated on first use
  float* xfer_ph = nullptr;
  int* xfer_id = nullptr;
  // moving domain
  double* layer_sums = nullptr;
  int* alpha_full = nullptr;
  int fnz_f = 0;
  int* loss_area = nullptr;
  // reductions
  unsigned long long* counts = nullptr;
  long long* first = nullptr;
  double* qoi_part = nullptr;
  long long* jcand = nullptr;  // junction candidate cells
  long long jcand_cap = 0;
  unsigned long long* jcount = nullptr;
  unsigned char* jdistinct = nullptr;  // distinct values per interior cell
  // nucleation
  int* nucl_status = nullptr;
  int* nucl_count = nullptr;
  float* nucl_sphere = nullptr;
  int cnx = 0, cny = 0, cnz = 0, pts = 0;
  int counts_cap = 0;
  // launch shape
  int zc = 64;
  int ty = 8;  // column-tile height (cupf_apt_set_tile)
  int ntx = 0, nty = 0, nzc = 0;
  // events for timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

static const char* kOk = "";

static cupf_status upload(float** dst, const float* src, size_t n, cudaStream_t s) {
  if (n == 0) n = 1;
  CK(cudaMalloc((void**)dst, n * sizeof(float)));
  if (src)
    CK(cudaMemcpyAsync(*dst, src, n * sizeof(float), cudaMemcpyHostToDevice, s));
  else
    CK(cudaMemsetAsync(*dst, 0, n * sizeof(float), s));
  return CUPF_OK;
}

// Call f(S{}) with the storage format S of the handle.
template <class F>
static cupf_status with_storage(cupf_precision prec, F&& f) {
  switch (prec) {
    case CUPF_PREC_FP32: return f(PairF32{});
    case CUPF_PREC_BF16: return f(PairBF16{});
    case CUPF_PREC_FP16: return f(PairFP16{});
  }
  return fail(CUPF_ERR_UNSUPPORTED, "precision %d", (int)prec);
}

template <class S>
static typename S::T* B(void* p) {
  return static_cast<typename S::T*>(p);
}

// launch kernel<S> for the handle's storage format; buffers cast with B<S>(...)
#define LAUNCH_S(h, kernel, grid, block, ...)                                   \
  do {                                                                          \
    cupf_status st_ = with_storage((h)->prec, [&](auto tag) -> cupf_status {    \
      using S = decltype(tag);                                                  \
      kernel<S><<<(grid), (block), 0, (h)->stream>>>(__VA_ARGS__);              \
      return CUPF_OK;                                                           \
    });                                                                         \
    if (st_) return st_;                                                        \
  } while (0)

static cupf_status make_tmap(cupf_apt_handle* h, int b) {
  EncodeTiledFn enc = get_encode();
  if (!enc) return fail(CUPF_ERR_CUDA, "cuTensorMapEncodeTiled entry point not available");
  const Grid& g = h->g;
  return with_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    const cuuint64_t e = S::kBytes;
    cuuint64_t dims[4] = {(cuuint64_t)g.fnx, (cuuint64_t)g.fny, (cuuint64_t)g.fnz,
                          (cuuint64_t)g.np};
    cuuint64_t strides[3] = {(cuuint64_t)g.xp * e, (cuuint64_t)g.xp * g.fny * e,
                             (cuuint64_t)g.ss * e};
    cuuint32_t box[4] = {(cuuint32_t)S::kBW, (cuuint32_t)(h->ty + 2), 1u, (cuuint32_t)g.np};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(&h->tmap[b], S::kTmaType, 4, h->buf[b], dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return fail(CUPF_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return CUPF_OK;
  });
}

static void free_handle(cupf_apt_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  void* ptrs[] = {h->buf[0], h->buf[1], h->x, h->y, h->z, h->sint, h->cost, h->orient, h->X_mac, h->Y_mac,
                  h->Z_mac, h->t_mac, h->psi_mac, h->T_3D, h->phi_m, h->alpha_m, h->err, h->work,
                  h->xfer_ph, h->xfer_id, h->layer_sums, h->alpha_full, h->loss_area,
                  h->counts, h->first, h->qoi_part, h->nucl_status, h->nucl_count,
                  h->nucl_sphere, h->jcand, h->jcount, h->jdistinct, h->quiet[0], h->quiet[1],
                  h->active_cells, h->overflows, h->z64};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

// ------------------------------------------------------------------ step launch
template <int NP, class S, int TY>
static cupf_status launch_step_np(cupf_apt_handle* h, const StepArgs& a, const CUtensorMap& m) {
  static bool configured[64] = {};
  static int resident[64] = {};
  constexpr int NTHREADS = tile_threads<TY>();
  const int bytes = StepSmem<NP, S, TY>::kBytes;
  if (!configured[h->device & 63]) {
    CK(cudaFuncSetAttribute(apt_step_kernel<NP, S, TY>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int per_sm = 0, nsm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, apt_step_kernel<NP, S, TY>,
                                                     NTHREADS, bytes));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    resident[h->device & 63] = std::max(1, per_sm) * nsm;
    configured[h->device & 63] = true;
  }
  const int nitems = h->ntx * h->nty * h->nzc;
  const int nblk = std::min(nitems, h->grid_cap > 0 ? h->grid_cap : resident[h->device & 63]);
  apt_step_kernel<NP, S, TY><<<nblk, NTHREADS, bytes, h->stream>>>(m, a);
  CK(cudaGetLastError());
  return CUPF_OK;
}

static cupf_status launch_step(cupf_apt_handle* h, const StepArgs& a, const CUtensorMap& m) {
  return with_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    switch (h->g.np) {
#define CASE(N)                                                                 \
  case N:                                                                       \
    return h->ty == 4 ? launch_step_np<N, S, 4>(h, a, m) : launch_step_np<N, S, 8>(h, a, m);
      CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
#undef CASE
      default:
        return fail(CUPF_ERR_UNSUPPORTED, "num_pf=%d not built (1..8)", h->g.np);
    }
  });
}

static StepArgs step_args(cupf_apt_handle* h, float t, int use_iuc) {
  const cupf_apt_params& p = h->p;
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.fnx = p.fnx;
  a.fny = p.fny;
  a.fnz = p.fnz;
  a.xp = h->g.xp;
  a.slot_stride = h->g.ss;
  a.bcX = p.bcX;
  a.bcY = p.bcY;
  a.bcZ = p.bcZ;
  a.ntx = h->ntx;
  a.nty = h->nty;
  a.nzc = h->nzc;
  a.zc = h->zc;
  a.num_theta = p.num_theta;
  {
    const InvariantDivisor dv = invariant_divisor((uint32_t)p.num_theta);
    a.nt_magic = dv.m;
    a.nt_sh1 = dv.s1;
    a.nt_sh2 = dv.s2;
  }
  a.thermalType = p.thermalType;
  a.use_iuc = use_iuc;
  a.t = t;
  // 16-bit storage keeps time and heights in FP64; FP32 keeps the reference's
  // float forms (bit parity)
  a.fp64 = h->prec != CUPF_PREC_FP32;
  a.t64 = (double)(h->steps_done + 1) * (double)p.dt * (double)p.tau0;
  a.z64 = h->z64;
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
  a.Nx = p.Nx;
  a.Ny = p.Ny;
  a.Nz = p.Nz;
  a.x = h->x;
  a.y = h->y;
  a.z = h->z;
  a.sint = h->sint;
  a.cost = h->cost;
  a.orient = reinterpret_cast<const float4*>(h->orient);
  a.X_mac = h->X_mac;
  a.Y_mac = h->Y_mac;
  a.Z_mac = h->Z_mac;
  a.psi_mac = h->psi_mac;
  a.err = h->err;
  a.work = h->work;
  a.wait_limit = h->wait_limit;
  return a;
}

static void set_zc(cupf_apt_handle* h, int zc) {
  const int nz = h->p.fnz - 2;
  h->zc = zc < 1 ? 1 : (zc > nz ? nz : zc);
  h->ntx = (h->p.fnx - 2 + TX - 1) / TX;
  h->nty = (h->p.fny - 2 + h->ty - 1) / h->ty;
  h->nzc = (nz + h->zc - 1) / h->zc;
}

// Forget what the quiet-item flags say about both buffers: after anything but
// the step writes the slot buffers, or when the item grid changes.
static cupf_status invalidate_quiet(cupf_apt_handle* h) {
  for (int b = 0; b < 2; ++b)
    if (h->quiet[b]) CK(cudaMemsetAsync(h->quiet[b], 0, h->quiet_cap, h->stream));
  return CUPF_OK;
}

// Resident CTAs per SM the step kernel is compiled for (step_min_blocks).
static int resident_per_sm(const cupf_apt_handle* h) {
  int r = 2;
  with_storage(h->prec, [&](auto tag) -> cupf_status {
    using S = decltype(tag);
    switch (h->g.np) {
#define CASE(N)                                                                      \
  case N:                                                                            \
    r = h->ty == 4 ? step_min_blocks<N, S, 4>() : step_min_blocks<N, S, 8>();        \
    break;
      CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
#undef CASE
      default: break;
    }
    return CUPF_OK;
  });
  return r;
}

// Default z-chunk of a work item: the largest of 16, 8, 4, 2, 1 planes that
// still gives at least 2.5 work items per resident CTA, else 1.  Measured on
// the line case (B200, NUM_PF = 5 and 8): 16 is best from 128x128x256 up, while
// 96^3 wants 4 and 64^3 or 48^3 want 1-2 (2.5-3x faster than 8 there) -- with
// fewer items than CTAs most of the GPU idles, with many short items each pays
// the two extra planes of its TMA pipeline fill.
static int default_zc(cupf_apt_handle* h) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const long long tiles =
      (long long)((h->p.fnx - 2 + TX - 1) / TX) * ((h->p.fny - 2 + h->ty - 1) / h->ty);
  const int nz = h->p.fnz - 2;
  const long long want = (5LL * resident_per_sm(h) * nsm + 1) / 2;
  for (int zc = 16; zc > 1; zc /= 2)
    if (tiles * ((nz + zc - 1) / zc) >= want) return zc;
  return 1;
}

// z chunk for a state whose grain ids occupy nz_active interior planes (those
// within 10 planes of a plane holding an id: the tails the first steps grow):
// the largest of 16, 8, 4, 2 that gives at least 2 work items per resident CTA
// over those planes, else 1.  Quiet items cost next to nothing, so the items
// that count are the ones the step computes.  Measured on line cases (B200,
// NUM_PF = 8, FP32 and FP16, 64^3 to 256x256x512): within 6 % of the best chunk
// of 16..1 on every case, where sizing by all items was up to 18 % off.
static int zc_for_active(cupf_apt_handle* h, int nz_active) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const long long tiles =
      (long long)((h->p.fnx - 2 + TX - 1) / TX) * ((h->p.fny - 2 + h->ty - 1) / h->ty);
  const long long want = 2LL * resident_per_sm(h) * nsm;
  for (int zc = 16; zc > 1; zc /= 2)
    if (tiles * ((nz_active + zc - 1) / zc) >= want) return zc;
  return 1;
}

// Interior planes within 10 planes of a plane that holds an id (plane_any[k]
// for k = 0..fnz-1); all interior planes when none does.
static int active_planes(const std::vector<char>& plane_any, int fnz) {
  const int nz = fnz - 2, reach = 10;
  int n = 0, last = -1000000;
  std::vector<int> next(fnz + 1, 1000000);
  for (int k = fnz - 1; k >= 0; --k) next[k] = plane_any[k] ? k : next[k + 1];
  for (int k = 1; k <= nz; ++k) {
    if (plane_any[k]) last = k;
    if (k - last <= reach || next[k] - k <= reach) ++n;
  }
  return n > 0 ? n : nz;
}

static int grid_for(long long n, int block = 256) {
  long long b = (n + block - 1) / block;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

static cupf_status check_err_word(cupf_apt_handle* h) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (e != 0) return fail(CUPF_ERR_TIMEOUT, "step kernel reported error %d (TMA wait timed out)", e);
  return CUPF_OK;
}

// ------------------------------------------------------------------ API
extern "C" cupf_status cupf_apt_create(const cupf_apt_params* p, const cupf_apt_inputs* in,
                                       int device, cupf_precision precision,
                                       cupf_apt_handle** out) {
  if (!p || !in || !out) return fail(CUPF_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->fnx < 4 || p->fny < 4 || p->fnz < 4)
    return fail(CUPF_ERR_INVALID, "grid %dx%dx%d too small (each fn >= 4)", p->fnx, p->fny, p->fnz);
  if ((long long)p->fnx * p->fny * p->fnz > (1ll << 31) - 1)
    return fail(CUPF_ERR_INVALID, "grid has more than 2^31-1 points");
  if (p->num_pf < 1 || p->num_pf > 8)
    return fail(CUPF_ERR_UNSUPPORTED, "num_pf=%d not built (1..8)", p->num_pf);
  if (p->num_theta < 1) return fail(CUPF_ERR_INVALID, "num_theta must be >= 1");
  if (p->haloWidth != 1) return fail(CUPF_ERR_INVALID, "haloWidth must be 1");
  if (p->thermalType < 0 || p->thermalType > 5)
    return fail(CUPF_ERR_INVALID, "thermalType %d not in 0..5", p->thermalType);
  if (precision != CUPF_PREC_FP32 && precision != CUPF_PREC_BF16 && precision != CUPF_PREC_FP16)
    return fail(CUPF_ERR_UNSUPPORTED, "precision %d not built", (int)precision);
  if (precision != CUPF_PREC_FP32 && p->num_theta > 32767)
    return fail(CUPF_ERR_UNSUPPORTED, "16-bit storage keeps grain ids in int16 (num_theta <= 32767)");
  if (!in->x || !in->y || !in->z || !in->sint || !in->cost)
    return fail(CUPF_ERR_INVALID, "x, y, z, sint and cost are required");
  if (p->thermalType == 4 && (!in->X_mac || !in->Y_mac || !in->Z_mac || !in->psi_mac))
    return fail(CUPF_ERR_INVALID, "thermalType 4 needs X_mac, Y_mac, Z_mac and psi_mac");

  cupf_apt_handle* h = new cupf_apt_handle();
  h->p = *p;
  h->device = device;
  h->prec = precision;
  h->g.fnx = p->fnx;
  h->g.fny = p->fny;
  h->g.fnz = p->fnz;
  h->pair_bytes = precision == CUPF_PREC_FP32 ? 8 : 4;
  const int palign = precision == CUPF_PREC_FP32 ? PairF32::kPitchAlign : PairBF16::kPitchAlign;
  h->g.xp = (p->fnx + palign - 1) / palign * palign;
  h->g.np = p->num_pf;
  h->g.ss = (long long)h->g.xp * p->fny * p->fnz;
  cupf_status st = CUPF_OK;
#define TRY(x)                  \
  do {                          \
    st = (x);                   \
    if (st != CUPF_OK) {        \
      free_handle(h);           \
      return st;                \
    }                           \
  } while (0)
  auto cuda = [&](cudaError_t e, const char* what) -> cupf_status {
    if (e == cudaSuccess) return CUPF_OK;
    return fail(e == cudaErrorMemoryAllocation ? CUPF_ERR_OOM : CUPF_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
  };
  TRY(cuda(cudaSetDevice(device), "cudaSetDevice"));
  TRY(cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream"));
  TRY(cuda(cudaEventCreate(&h->ev0), "event"));
  TRY(cuda(cudaEventCreate(&h->ev1), "event"));
  const size_t bbytes = (size_t)h->g.ss * h->g.np * h->pair_bytes;
  for (int b = 0; b < 2; ++b) {
    TRY(cuda(cudaMalloc((void**)&h->buf[b], bbytes), "slot buffer"));
    TRY(cuda(cudaMemsetAsync(h->buf[b], 0xFF, bbytes, h->stream), "memset"));
  }
  const int nth = 2 * p->num_theta + 1;
  TRY(upload(&h->x, in->x, p->fnx, h->stream));
  TRY(upload(&h->y, in->y, p->fny, h->stream));
  TRY(upload(&h->z, in->z, p->fnz, h->stream));
  h->z_host.assign(in->z, in->z + p->fnz);
  h->z64_host.assign(in->z, in->z + p->fnz);
  TRY(cuda(cudaMalloc((void**)&h->z64, p->fnz * sizeof(double)), "z64"));
  TRY(cuda(cudaMemcpyAsync(h->z64, h->z64_host.data(), p->fnz * sizeof(double),
                           cudaMemcpyHostToDevice, h->stream), "z64 upload"));
  TRY(upload(&h->sint, in->sint, nth, h->stream));
  TRY(upload(&h->cost, in->cost, nth, h->stream));
  {
    std::vector<float> ot(4 * (size_t)(p->num_theta + 1));
    pack_orientations(in->sint, in->cost, p->num_theta, ot.data());
    TRY(upload(&h->orient, ot.data(), ot.size(), h->stream));
  }
  const size_t mNx = p->Nx > 0 ? p->Nx : 1, mNy = p->Ny > 0 ? p->Ny : 1;
  const size_t mNz = p->Nz > 0 ? p->Nz : 1, mNt = p->Nt > 0 ? p->Nt : 1;
  TRY(upload(&h->X_mac, in->X_mac, in->X_mac ? mNx : 2, h->stream));
  TRY(upload(&h->Y_mac, in->Y_mac, in->Y_mac ? mNy : 2, h->stream));
  TRY(upload(&h->Z_mac, in->Z_mac, in->Z_mac ? mNz : 2, h->stream));
  TRY(upload(&h->t_mac, in->t_mac, in->t_mac ? mNt : 2, h->stream));
  TRY(upload(&h->psi_mac, in->psi_mac, in->psi_mac ? mNx * mNy * mNz : 8, h->stream));
  TRY(upload(&h->T_3D, in->T_3D, in->T_3D ? mNx * mNy * mNz * mNt : 16, h->stream));
  h->has_T3D = in->T_3D != nullptr;
  const size_t L = (size_t)h->g.length();
  TRY(cuda(cudaMalloc((void**)&h->phi_m, L * sizeof(float)), "phi"));
  TRY(cuda(cudaMalloc((void**)&h->alpha_m, L * sizeof(int)), "alpha"));
  TRY(cuda(cudaMemsetAsync(h->phi_m, 0, L * sizeof(float), h->stream), "memset"));
  TRY(cuda(cudaMemsetAsync(h->alpha_m, 0, L * sizeof(int), h->stream), "memset"));
  TRY(cuda(cudaMalloc((void**)&h->err, sizeof(int)), "err"));
  TRY(cuda(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream), "memset"));
  TRY(cuda(cudaMalloc((void**)&h->work, 2 * sizeof(int)), "work"));
  TRY(cuda(cudaMemsetAsync(h->work, 0, 2 * sizeof(int), h->stream), "memset"));
  // flags for the most items any tile height gives (32x4 tiles, z chunks of 1)
  h->quiet_cap = (size_t)((p->fnx - 2 + TX - 1) / TX) * ((p->fny - 2 + 4 - 1) / 4) * (p->fnz - 2);
  for (int b = 0; b < 2; ++b) {
    TRY(cuda(cudaMalloc((void**)&h->quiet[b], h->quiet_cap), "quiet flags"));
    TRY(cuda(cudaMemsetAsync(h->quiet[b], 0, h->quiet_cap, h->stream), "memset"));
  }
  TRY(cuda(cudaMalloc((void**)&h->active_cells, sizeof(unsigned long long)), "counter"));
  TRY(cuda(cudaMemsetAsync(h->active_cells, 0, sizeof(unsigned long long), h->stream), "memset"));
  TRY(cuda(cudaMalloc((void**)&h->overflows, 2 * sizeof(unsigned long long)), "counter"));
  TRY(cuda(cudaMemsetAsync(h->overflows, 0, 2 * sizeof(unsigned long long), h->stream), "memset"));
  TRY(cuda(cudaMalloc((void**)&h->layer_sums, p->fnz * sizeof(double)), "layer sums"));
  for (int b = 0; b < 2; ++b) TRY(make_tmap(h, b));
  const char* zc_env = getenv("CUPF_ZC");
  h->zc_user = zc_env != nullptr;
  set_zc(h, zc_env ? atoi(zc_env) : default_zc(h));
  TRY(cuda(cudaStreamSynchronize(h->stream), "sync"));
#undef TRY
  *out = h;
  g_err = kOk;
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_destroy(cupf_apt_handle* h) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_handle(h);
  return CUPF_OK;
}

extern "C" void* cupf_apt_stream(cupf_apt_handle* h) { return h ? (void*)h->stream : nullptr; }

extern "C" cupf_status cupf_apt_set_tuning(cupf_apt_handle* h, int32_t z_chunk) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  if (z_chunk < 1) return fail(CUPF_ERR_INVALID, "z_chunk must be >= 1");
  CK(cudaSetDevice(h->device));
  set_zc(h, z_chunk);
  h->zc_user = true;
  return invalidate_quiet(h);
}

extern "C" cupf_status cupf_apt_set_tile(cupf_apt_handle* h, int32_t tile_y) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  if (!tile_height_built(tile_y)) return fail(CUPF_ERR_INVALID, "tile_y must be 8 or 4");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));  // no step in flight reads the old maps
  h->ty = tile_y;
  for (int b = 0; b < 2; ++b) {
    const cupf_status e = make_tmap(h, b);
    if (e) return e;
  }
  set_zc(h, h->zc);
  return invalidate_quiet(h);
}

extern "C" cupf_status cupf_apt_set_wait_limit(cupf_apt_handle* h, int64_t cycles) {
  if (!h || cycles < 0) return fail(CUPF_ERR_INVALID, "bad argument");
  h->wait_limit = cycles == 0 ? kWaitCycles : cycles;
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_set_skip_quiet(cupf_apt_handle* h, int32_t enable) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  CK(cudaSetDevice(h->device));
  h->skip_quiet = enable != 0;
  return invalidate_quiet(h);
}

extern "C" cupf_status cupf_apt_merge_overflows(cupf_apt_handle* h, uint64_t* counts) {
  if (!h || !counts) return fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  unsigned long long v[2] = {0, 0};
  CK(cudaMemcpyAsync(v, h->overflows, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemsetAsync(h->overflows, 0, sizeof(v), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  counts[0] = v[0];
  counts[1] = v[1];
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_active_cells(cupf_apt_handle* h, uint64_t* cells) {
  if (!h || !cells) return fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, h->active_cells, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemsetAsync(h->active_cells, 0, sizeof(v), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *cells = v;
  return CUPF_OK;
}

static cupf_status fill_halo(cupf_apt_handle* h, int b);

extern "C" cupf_status cupf_apt_init_from_argmax(cupf_apt_handle* h, const float* phi,
                                                 const int32_t* alpha) {
  if (!h || !phi || !alpha) return fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  const size_t L = (size_t)h->g.length();
  const int id_max = h->prec == CUPF_PREC_FP32 ? 0x7FFFFFFF : 32767;
  for (size_t i = 0; i < L; ++i)
    if ((double)phi[i] > LS && (alpha[i] < -1 || alpha[i] > id_max))
      return fail(CUPF_ERR_INVALID, "grain id %d at %zu outside [-1, %d]", alpha[i], i, id_max);
  if (!h->zc_user) {
    std::vector<char> plane_any(h->p.fnz, 0);
    for (int k = 1; k < h->p.fnz - 1; ++k)
      for (int j = 1; j < h->p.fny - 1 && !plane_any[k]; ++j)
        for (int i = 1; i < h->p.fnx - 1; ++i)
          if ((double)phi[(size_t)k * h->p.fnx * h->p.fny + (size_t)j * h->p.fnx + i] > LS) {
            plane_any[k] = 1;
            break;
          }
    set_zc(h, zc_for_active(h, active_planes(plane_any, h->p.fnz)));
  }
  CK(cudaMemcpyAsync(h->phi_m, phi, L * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->alpha_m, alpha, L * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  LAUNCH_S(h, init_kernel, grid_for(L), 256, B<S>(h->buf[0]), B<S>(h->buf[1]), h->phi_m,
           h->alpha_m, h->g);
  CK(cudaGetLastError());
  // the step reads x/y halo cells from the buffer it advances
  for (int b = 0; b < 2; ++b)
    if (cupf_status st = fill_halo(h, b)) return st;
  if (cupf_status st = invalidate_quiet(h)) return st;
  CK(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));  // a new state: no step has failed
  h->cur = 0;
  h->steps_done = 0;
  h->initialised = true;
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

static cupf_status ensure_xfer(cupf_apt_handle* h) {
  if (!h->xfer_ph) {
    const size_t n = (size_t)h->g.length() * h->g.np;
    CK(cudaMalloc((void**)&h->xfer_ph, n * sizeof(float)));
    CK(cudaMalloc((void**)&h->xfer_id, n * sizeof(int)));
  }
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_set_slots(cupf_apt_handle* h, const float* ph, const int32_t* ids,
                                          int64_t steps_done) {
  if (!h || !ph || !ids) return fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  const size_t L = (size_t)h->g.length();
  const size_t n = L * h->g.np;
  const int id_max = h->prec == CUPF_PREC_FP32 ? 0x7FFFFFFF : 32767;
  for (size_t i = 0; i < n; ++i)
    if (ids[i] < -1 || ids[i] > id_max)
      return fail(CUPF_ERR_INVALID, "grain id %d at %zu outside [-1, %d]", ids[i], i, id_max);
  if (!h->zc_user) {
    // reference layout: index = i + j*fnx + k*fnx*fny + slot*L
    std::vector<char> plane_any(h->p.fnz, 0);
    const int fnx = h->p.fnx, fny = h->p.fny;
    for (int p = 0; p < h->g.np; ++p)
      for (int k = 1; k < h->p.fnz - 1; ++k)
        for (int j = 1; j < fny - 1 && !plane_any[k]; ++j)
          for (int i = 1; i < fnx - 1; ++i)
            if (ids[p * L + (size_t)k * fnx * fny + (size_t)j * fnx + i] >= 0) {
              plane_any[k] = 1;
              break;
            }
    set_zc(h, zc_for_active(h, active_planes(plane_any, h->p.fnz)));
  }
  cupf_status st = ensure_xfer(h);
  if (st) return st;
  CK(cudaMemcpyAsync(h->xfer_ph, ph, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->xfer_id, ids, n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  LAUNCH_S(h, import_kernel, grid_for(n), 256, B<S>(h->buf[0]), h->xfer_ph, h->xfer_id, h->g);
  LAUNCH_S(h, import_kernel, grid_for(n), 256, B<S>(h->buf[1]), h->xfer_ph, h->xfer_id, h->g);
  CK(cudaGetLastError());
  for (int b = 0; b < 2; ++b)
    if ((st = fill_halo(h, b))) return st;
  if ((st = invalidate_quiet(h))) return st;
  CK(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));  // a new state: no step has failed
  h->cur = 0;
  h->steps_done = steps_done;
  h->initialised = true;
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

static cupf_status fill_halo(cupf_apt_handle* h, int b) {
  const Grid& g = h->g;
  const long long n = 2ll * g.fnx * g.fny + 2ll * g.fnx * (g.fnz - 2) + 2ll * (g.fny - 2) * (g.fnz - 2);
  LAUNCH_S(h, fill_halo_kernel, grid_for(n), 256, B<S>(h->buf[b]), g, h->p.bcX, h->p.bcY,
           h->p.bcZ);
  CK(cudaGetLastError());
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_get_slots(cupf_apt_handle* h, float* ph, int32_t* ids) {
  if (!h || !ph || !ids) return fail(CUPF_ERR_INVALID, "null argument");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  cupf_status st = ensure_xfer(h);
  if (st) return st;
  if ((st = fill_halo(h, h->cur))) return st;
  const size_t n = (size_t)h->g.length() * h->g.np;
  LAUNCH_S(h, export_kernel, grid_for(n), 256, B<S>(h->buf[h->cur]), h->xfer_ph, h->xfer_id,
           h->g);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ph, h->xfer_ph, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(ids, h->xfer_id, n * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_err_word(h);
}

extern "C" cupf_status cupf_apt_step(cupf_apt_handle* h, int32_t nsteps,
                                     int32_t use_initial_undercooling) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "step before init");
  if (nsteps < 0) return fail(CUPF_ERR_INVALID, "nsteps < 0");
  CK(cudaSetDevice(h->device));
  for (int n = 0; n < nsteps; ++n) {
    // t of step m (1-based): (float)m * dt * tau0, as (2*kt+1)*dt*tau0 in evolve
    const float t = (float)(h->steps_done + 1) * h->p.dt * h->p.tau0;
    StepArgs a = step_args(h, t, use_initial_undercooling);
    a.sr_key = (uint32_t)(h->steps_done + 1);
    a.in = h->buf[h->cur];
    a.out = h->buf[h->cur ^ 1];
    if (h->skip_quiet) {
      a.quiet_in = h->quiet[h->cur];
      a.quiet_out = h->quiet[h->cur ^ 1];
    }
    a.active_cells = h->active_cells;
    a.overflows = h->overflows;
    cupf_status st = launch_step(h, a, h->tmap[h->cur]);
    if (st) return st;
    h->cur ^= 1;
    h->steps_done += 1;
  }
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_steps_done(cupf_apt_handle* h, int64_t* steps) {
  if (!h || !steps) return fail(CUPF_ERR_INVALID, "null argument");
  *steps = h->steps_done;
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_collect(cupf_apt_handle* h, int32_t clear, float* phi_out,
                                        int32_t* alpha_out) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  const size_t L = (size_t)h->g.length();
  if (clear) {
    CK(cudaMemsetAsync(h->phi_m, 0, L * sizeof(float), h->stream));
    CK(cudaMemsetAsync(h->alpha_m, 0, L * sizeof(int), h->stream));
  }
  cupf_status st = fill_halo(h, h->cur);
  if (st) return st;
  LAUNCH_S(h, collect_kernel, grid_for(L), 256, B<S>(h->buf[h->cur]), h->phi_m, h->alpha_m, h->g);
  CK(cudaGetLastError());
  if (phi_out)
    CK(cudaMemcpyAsync(phi_out, h->phi_m, L * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (alpha_out)
    CK(cudaMemcpyAsync(alpha_out, h->alpha_m, L * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_err_word(h);
}

extern "C" cupf_status cupf_apt_junction_candidates(cupf_apt_handle* h, int64_t* cells,
                                                    int64_t cap, int64_t* count,
                                                    uint8_t* distinct) {
  if (!h || !count || cap < 0 || (cap > 0 && !cells)) return fail(CUPF_ERR_INVALID, "bad argument");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  const Grid& g = h->g;
  const long long ni = (long long)(g.fnx - 2) * (g.fny - 2) * (g.fnz - 2);
  const long long want = cap > 0 ? cap : 1;
  if (h->jcand_cap < want) {
    if (h->jcand) cudaFree(h->jcand);
    h->jcand = nullptr;
    h->jcand_cap = 0;
    CK(cudaMalloc((void**)&h->jcand, want * sizeof(long long)));
    h->jcand_cap = want;
  }
  if (!h->jcount) CK(cudaMalloc((void**)&h->jcount, sizeof(unsigned long long)));
  if (!h->jdistinct) CK(cudaMalloc((void**)&h->jdistinct, (size_t)ni));
  CK(cudaMemsetAsync(h->jcount, 0, sizeof(unsigned long long), h->stream));
  junction_candidates_kernel<<<grid_for(ni), 256, 0, h->stream>>>(
      h->alpha_m, g.fnx, g.fny, g.fnz, h->jcand, cap, h->jcount, h->jdistinct);
  CK(cudaGetLastError());
  unsigned long long n = 0;
  CK(cudaMemcpyAsync(&n, h->jcount, sizeof(n), cudaMemcpyDeviceToHost, h->stream));
  if (distinct)
    CK(cudaMemcpyAsync(distinct, h->jdistinct, (size_t)ni, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const long long got = std::min<long long>((long long)n, cap);
  if (got > 0) {
    CK(cudaMemcpyAsync(cells, h->jcand, got * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::sort(cells, cells + got);
  }
  *count = (int64_t)n;
  return CUPF_OK;
}

extern "C" cupf_status cupf_line_junction_candidates(int32_t device, int32_t fnx, int32_t fny,
                                                    const int32_t* layers, int32_t nlayers,
                                                    int64_t* cells, int64_t cap, int64_t* count) {
  if (!count || fnx < 3 || fny < 3 || nlayers < 0 || cap < 0 || (cap > 0 && !cells) ||
      (nlayers > 0 && !layers))
    return fail(CUPF_ERR_INVALID, "bad argument");
  *count = 0;
  if (nlayers == 0) return CUPF_OK;
  CK(cudaSetDevice(device));
  const cudaStream_t st = cudaStreamPerThread;
  const long long plane = (long long)fnx * fny;
  const long long ncell = (long long)(fnx - 2) * (fny - 2) * nlayers;
  const size_t lbytes = (size_t)plane * nlayers * sizeof(int32_t);
  const long long want = cap > 0 ? cap : 1;
  int32_t* d_layers = nullptr;
  long long* d_out = nullptr;
  unsigned long long* d_count = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&d_layers, lbytes, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_out, want * sizeof(long long), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_count, sizeof(unsigned long long), st);
  unsigned long long n = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_layers, layers, lbytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    line_junction_kernel<<<grid_for(ncell), 256, 0, st>>>(d_layers, nlayers, fnx, fny, d_out, cap,
                                                          d_count);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&n, d_count, sizeof(n), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  const long long got = std::min<long long>((long long)n, cap);
  if (e == cudaSuccess && got > 0) {
    e = cudaMemcpyAsync(cells, d_out, got * sizeof(long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (d_layers) cudaFreeAsync(d_layers, st);
  if (d_out) cudaFreeAsync(d_out, st);
  if (d_count) cudaFreeAsync(d_count, st);
  CK(e);
  CK(cudaStreamSynchronize(st));
  if (got > 0) std::sort(cells, cells + got);
  *count = (int64_t)n;
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_grain_volumes(cupf_apt_handle* h, int32_t num_grains,
                                              int64_t* counts) {
  if (!h || !counts || num_grains < 0) return fail(CUPF_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(h->device));
  if (h->counts_cap < num_grains + 1) {
    if (h->counts) cudaFree(h->counts);
    if (h->first) cudaFree(h->first);
    h->counts = nullptr;
    h->first = nullptr;
    CK(cudaMalloc((void**)&h->counts, (num_grains + 1) * sizeof(unsigned long long)));
    CK(cudaMalloc((void**)&h->first, (num_grains + 1) * sizeof(long long)));
    h->counts_cap = num_grains + 1;
  }
  CK(cudaMemsetAsync(h->counts, 0, (num_grains + 1) * sizeof(unsigned long long), h->stream));
  CK(cudaMemsetAsync(h->first, 0x7F, (num_grains + 1) * sizeof(long long), h->stream));
  const long long n = (long long)(h->p.fnx - 2) * (h->p.fny - 2) * (h->p.fnz - 2);
  volume_kernel<<<grid_for(n), 256, 0, h->stream>>>(h->alpha_m, h->p.fnx, h->p.fny, h->p.fnz,
                                                     num_grains, h->counts, h->first);
  CK(cudaGetLastError());
  std::vector<unsigned long long> c(num_grains + 1);
  CK(cudaMemcpyAsync(c.data(), h->counts, c.size() * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int i = 0; i <= num_grains; ++i) counts[i] = (int64_t)c[i];
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_qoi_sums(cupf_apt_handle* h, double* out) {
  if (!h || !out) return fail(CUPF_ERR_INVALID, "null argument");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  const int nb = 148 * 4;
  if (!h->qoi_part) CK(cudaMalloc((void**)&h->qoi_part, 2 * nb * sizeof(double)));
  cupf_status st = fill_halo(h, h->cur);
  if (st) return st;
  LAUNCH_S(h, qoi_sums_kernel, nb, 256, B<S>(h->buf[h->cur]), h->g, h->qoi_part);
  CK(cudaGetLastError());
  std::vector<double> part(2 * nb);
  CK(cudaMemcpyAsync(part.data(), h->qoi_part, part.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  double v = 0.0, a = 0.0;
  for (int b = 0; b < nb; ++b) {
    v += part[2 * b];
    a += part[2 * b + 1];
  }
  const double base = (double)(h->p.fnx - 2) * (h->p.fny - 2);
  out[0] = v;
  out[1] = a;
  out[2] = v / base;
  return check_err_word(h);
}

static NuclArgs nucl_args(cupf_apt_handle* h, int use_iuc) {
  const cupf_apt_params& p = h->p;
  NuclArgs a;
  memset(&a, 0, sizeof(a));
  a.fnx = p.fnx;
  a.fny = p.fny;
  a.fnz = p.fnz;
  a.xp = h->g.xp;
  a.slot_stride = h->g.ss;
  a.np = h->g.np;
  a.cnx = h->cnx;
  a.cny = h->cny;
  a.cnz = h->cnz;
  a.pts = h->pts;
  a.num_theta = p.num_theta;
  a.id_space = h->prec == CUPF_PREC_FP32 ? (1 << 30) : (32767 - p.num_theta);
  a.use_iuc = use_iuc;
  a.uc0 = p.underCoolingRate0;
  a.nmax0 = p.nuc_Nmax0;
  a.nmax = p.nuc_Nmax;
  a.mean = p.undcool_mean;
  a.std = p.undcool_std;
  a.rad = p.nuc_rad;
  a.dt2 = 2.0f * p.dt * p.tau0;
  a.t = (float)h->steps_done * p.dt * p.tau0;
  a.seed = (uint32_t)p.seed;
  a.step = (uint32_t)h->steps_done;
  a.T_3D = h->has_T3D ? h->T_3D : nullptr;
  a.X_mac = h->X_mac;
  a.Y_mac = h->Y_mac;
  a.Z_mac = h->Z_mac;
  a.t_mac = h->t_mac;
  a.x = h->x;
  a.y = h->y;
  a.z = h->z;
  a.Nx = p.Nx;
  a.Ny = p.Ny;
  a.Nz = p.Nz;
  a.Nt = p.Nt;
  a.sphere = h->nucl_sphere;
  a.status = h->nucl_status;
  a.count = h->nucl_count;
  a.quiet = h->quiet[h->cur];
  a.tw = TX;
  a.th = h->ty;
  a.zc = h->zc;
  a.ntx = h->ntx;
  a.nty = h->nty;
  return a;
}

extern "C" cupf_status cupf_apt_nucl_init(cupf_apt_handle* h) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "state not initialised");
  const cupf_apt_params& p = h->p;
  if (p.pts_cell < 0 || p.dx <= 0 || p.sqrt2 <= 0)
    return fail(CUPF_ERR_INVALID, "nucleation needs pts_cell >= 0, dx and sqrt2");
  if (h->prec != CUPF_PREC_FP32 && p.num_theta >= 32767)
    return fail(CUPF_ERR_UNSUPPORTED, "no id space left for nuclei in int16 storage");
  CK(cudaSetDevice(h->device));
  const int w = 2 * p.pts_cell + 1;
  h->pts = p.pts_cell;
  h->cnx = (p.fnx - 1 - 2) / w;
  h->cny = (p.fny - 1 - 2) / w;
  h->cnz = (p.fnz - 1 - 2) / w;
  const long long nc = (long long)h->cnx * h->cny * h->cnz;
  if (nc < 1) return fail(CUPF_ERR_INVALID, "grid smaller than one nucleation cell");
  if (!h->nucl_status) {
    CK(cudaMalloc((void**)&h->nucl_status, nc * sizeof(int)));
    CK(cudaMalloc((void**)&h->nucl_count, sizeof(int)));
    CK(cudaMalloc((void**)&h->nucl_sphere, (size_t)w * w * w * sizeof(float)));
  }
  // nucleus profile (add_nucl :515-528): tanh(dx*((1+pts)/2 - |offset|) / sqrt2)
  std::vector<float> sph((size_t)w * w * w);
  const float pf = (float)p.pts_cell;
  for (int k = -p.pts_cell; k <= p.pts_cell; ++k)
    for (int j = -p.pts_cell; j <= p.pts_cell; ++j)
      for (int i = -p.pts_cell; i <= p.pts_cell; ++i) {
        const float d = p.dx * ((1.0f + pf) / 2.0f - sqrtf((float)(i * i + j * j + k * k)));
        sph[((k + p.pts_cell) * w + (j + p.pts_cell)) * w + (i + p.pts_cell)] = tanhf(d / p.sqrt2);
      }
  CK(cudaMemcpyAsync(h->nucl_sphere, sph.data(), sph.size() * sizeof(float),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(h->nucl_count, 0, sizeof(int), h->stream));
  NuclArgs a = nucl_args(h, 0);
  LAUNCH_S(h, nucl_status_init_kernel, grid_for(nc), 256, B<S>(h->buf[h->cur]), a);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_nucl_reset(cupf_apt_handle* h) {
  if (!h || !h->nucl_status) return fail(CUPF_ERR_STATE, "nucleation not initialised");
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->nucl_status, 0,
                     (size_t)h->cnx * h->cny * h->cnz * sizeof(int), h->stream));
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_nucleate(cupf_apt_handle* h, int32_t use_initial_undercooling,
                                         int32_t* total) {
  if (!h || !h->nucl_status) return fail(CUPF_ERR_STATE, "nucleation not initialised");
  CK(cudaSetDevice(h->device));
  const long long nc = (long long)h->cnx * h->cny * h->cnz;
  NuclArgs a = nucl_args(h, use_initial_undercooling);
  LAUNCH_S(h, nucleate_kernel, grid_for(nc), 256, B<S>(h->buf[h->cur]), a);
  CK(cudaGetLastError());
  // nuclei change cells that source halo cells: refill the halo the step reads
  if (cupf_status st = fill_halo(h, h->cur)) return st;
  if (total) {
    CK(cudaMemcpyAsync(total, h->nucl_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_move_domain(cupf_apt_handle* h, int32_t* tip_front,
                                            int32_t tip_thres, int32_t* move_count,
                                            int32_t* moved) {
  if (!h || !tip_front || !move_count || !moved) return fail(CUPF_ERR_INVALID, "null argument");
  if (!h->initialised) return fail(CUPF_ERR_STATE, "state not initialised");
  CK(cudaSetDevice(h->device));
  const Grid& g = h->g;
  const cupf_apt_params& p = h->p;
  if (!h->alpha_full) {
    h->fnz_f = p.fnz * 4 + 8;  // archive capacity in layers; grown on demand below
    CK(cudaMalloc((void**)&h->alpha_full, (size_t)p.fnx * p.fny * h->fnz_f * sizeof(int)));
    CK(cudaMemsetAsync(h->alpha_full, 0, (size_t)p.fnx * p.fny * h->fnz_f * sizeof(int),
                       h->stream));
    CK(cudaMalloc((void**)&h->loss_area, p.num_theta * sizeof(int)));
    CK(cudaMemsetAsync(h->loss_area, 0, p.num_theta * sizeof(int), h->stream));
  }
  cupf_status st = fill_halo(h, h->cur);
  if (st) return st;
  LAUNCH_S(h, layer_sum_kernel, p.fnz, 256, B<S>(h->buf[h->cur]), h->layer_sums, g);
  CK(cudaGetLastError());
  std::vector<double> sums(p.fnz);
  CK(cudaMemcpyAsync(sums.data(), h->layer_sums, p.fnz * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // tip_mvf (PhaseField.cu:382-399): first layer whose mean is not above LS
  const float denom = (float)(p.num_pf * p.fnx * p.fny);
  while (((double)((float)sums[*tip_front] / denom) > LS) && (*tip_front < p.fnz - 1))
    (*tip_front)++;
  *moved = 0;
  const long long plane = (long long)p.fnx * p.fny;
  // Each layer moved: the argmax of the current buffer, its bottom interior layer
  // archived, then the interior shifted down one plane into the other buffer
  // (APTmove_frame), and copied back (APTcopy_frame: the interior only, so the
  // halo the next layer's argmax reads is the one from before the move).  Where
  // the thermal model updates every slot of every cell the step computes (types
  // 0, 1, 2, 5), the next step overwrites the other buffer wherever it is not
  // already empty, so instead of the copy back the halo cells go across and the
  // buffers swap (the other keeps the state before the move).  The cone and
  // paraboloid-table models (3, 4) leave slots unwritten past their fronts,
  // which must then hold the moved state: there the copy back stays.
  const int cur0 = h->cur;
  const bool swap = p.thermalType != 3 && p.thermalType != 4;
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
    const size_t L = (size_t)g.length();
    LAUNCH_S(h, collect_kernel, grid_for(L), 256, B<S>(h->buf[h->cur]), h->phi_m, h->alpha_m, g);
    archive_kernel<<<grid_for(plane), 256, 0, h->stream>>>(h->alpha_m, h->alpha_full, h->loss_area,
                                                           p.fnx, p.fny, *move_count, p.num_theta);
    const long long ni = (long long)(p.fnx - 2) * (p.fny - 2) * (p.fnz - 2) * p.num_pf;
    LAUNCH_S(h, shift_kernel, grid_for(ni), 256, B<S>(h->buf[h->cur]), B<S>(h->buf[h->cur ^ 1]), g);
    if (swap) {
      LAUNCH_S(h, copy_halo_kernel, grid_for(halo_cells(g)), 256, B<S>(h->buf[h->cur]),
               B<S>(h->buf[h->cur ^ 1]), g);
      h->cur ^= 1;
    } else {
      LAUNCH_S(h, copy_interior_kernel, grid_for(ni), 256, B<S>(h->buf[h->cur ^ 1]),
               B<S>(h->buf[h->cur]), g);
    }
    CK(cudaGetLastError());
    // z shift (APTmove_frame :365-369 then APTcopy_frame :401-402)
    std::vector<float>& z = h->z_host;
    const float ztop = 2.0f * z[p.fnz - 2] - z[p.fnz - 3];
    for (int k = 1; k < p.fnz - 2; ++k) z[k] = z[k + 1];
    z[p.fnz - 2] = ztop;
    CK(cudaMemcpyAsync(h->z, z.data(), p.fnz * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    // the same shift of the FP64 heights: the window offset accumulates in double
    std::vector<double>& z2 = h->z64_host;
    const double ztop2 = 2.0 * z2[p.fnz - 2] - z2[p.fnz - 3];
    for (int k = 1; k < p.fnz - 2; ++k) z2[k] = z2[k + 1];
    z2[p.fnz - 2] = ztop2;
    CK(cudaMemcpyAsync(h->z64, z2.data(), p.fnz * sizeof(double), cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *move_count += 1;
    *tip_front -= 1;
    *moved += 1;
  }
  if (*moved) {
    // quiet-item flags: the current buffer's are those of the state before the
    // move shifted by the layers moved.  The other buffer holds the moved state
    // too (copy back: the same flags), or the state before the move (swap, one
    // layer: its flags unchanged), or an intermediate state (swap, more layers:
    // flags cleared, nothing known).
    const int per = h->ntx * h->nty;
    const size_t nq = (size_t)per * h->nzc;
    const int tmp = h->cur == cur0 ? cur0 ^ 1 : h->cur;
    quiet_shift_kernel<<<grid_for((long long)nq), 256, 0, h->stream>>>(
        h->quiet[cur0], h->quiet[tmp], per, h->nzc, h->zc, p.fnz, *moved);
    if (tmp != h->cur)
      CK(cudaMemcpyAsync(h->quiet[h->cur], h->quiet[tmp], nq, cudaMemcpyDeviceToDevice, h->stream));
    if (swap && *moved > 1) CK(cudaMemsetAsync(h->quiet[h->cur ^ 1], 0, nq, h->stream));
    CK(cudaGetLastError());
  }
  // the current buffer's halo still holds the state before the move (and so does
  // the other's after a copy back)
  if ((st = fill_halo(h, h->cur))) return st;
  if (*moved && !swap && (st = fill_halo(h, h->cur ^ 1))) return st;
  CK(cudaStreamSynchronize(h->stream));
  return check_err_word(h);
}

extern "C" cupf_status cupf_apt_get_archive(cupf_apt_handle* h, int32_t fnz_f, int32_t* alpha_full,
                                            int32_t* loss_area) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  CK(cudaSetDevice(h->device));
  const long long plane = (long long)h->p.fnx * h->p.fny;
  if (alpha_full) {
    std::memset(alpha_full, 0, (size_t)plane * fnz_f * sizeof(int));
    if (h->alpha_full) {
      const int nl = fnz_f < h->fnz_f ? fnz_f : h->fnz_f;
      CK(cudaMemcpyAsync(alpha_full, h->alpha_full, (size_t)plane * nl * sizeof(int),
                         cudaMemcpyDeviceToHost, h->stream));
    }
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

extern "C" cupf_status cupf_apt_get_z(cupf_apt_handle* h, float* z) {
  if (!h || !z) return fail(CUPF_ERR_INVALID, "null argument");
  std::memcpy(z, h->z_host.data(), h->p.fnz * sizeof(float));
  return CUPF_OK;
}

extern "C" cupf_status cupf_apt_sync(cupf_apt_handle* h, int32_t timeout_ms) {
  if (!h) return fail(CUPF_ERR_INVALID, "null handle");
  CK(cudaSetDevice(h->device));
  if (timeout_ms <= 0) {
    CK(cudaStreamSynchronize(h->stream));
  } else {
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      cudaError_t e = cudaStreamQuery(h->stream);
      if (e == cudaSuccess) break;
      if (e != cudaErrorNotReady) CK(e);
      auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                    std::chrono::steady_clock::now() - t0)
                    .count();
      if (ms > timeout_ms) return fail(CUPF_ERR_TIMEOUT, "stream not idle after %d ms", timeout_ms);
      std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
  }
  return check_err_word(h);
}

extern "C" cupf_status cupf_apt_time_steps(cupf_apt_handle* h, int32_t nsteps, float* ms) {
  if (!h || !ms) return fail(CUPF_ERR_INVALID, "null argument");
  CK(cudaSetDevice(h->device));
  CK(cudaEventRecord(h->ev0, h->stream));
  cupf_status st = cupf_apt_step(h, nsteps, 0);
  if (st) return st;
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
  return check_err_word(h);
}
