// cupf_noalloc.cu — per-grain voxel counts of an argmax map without any
// device allocation.
//
// cupf_apt_grain_volumes keeps its reduction scratch (a count and a first
// occurrence per grain id) in device memory it allocates on first use.  Some
// callers cannot let a library allocate: simulation codes that hand all device
// memory to their own pool allocator at start-up (a cudaMalloc from inside a
// library then fails or fragments their pool), and long-running services whose
// device footprint must not grow after start-up.  cupf_grain_volumes_noalloc
// serves them: the caller passes the argmax map already on the device and a
// host array for the counts, and the scratch lives in the fixed-size device
// arrays below, which every GPU that loads this library holds until the
// process exits.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/cupf.h"
#include "apt_aux.cuh"
#include "capi_internal.h"

using namespace cupf;

// Scratch of the reduction: counts[g] and the first (k, j, i)-order index of
// grain g, for grain ids 0..CUPF_NOALLOC_MAX_GRAINS.
static __device__ __align__(256) unsigned long long g_noalloc_counts[CUPF_NOALLOC_MAX_GRAINS + 1];
static __device__ __align__(256) long long g_noalloc_first[CUPF_NOALLOC_MAX_GRAINS + 1];

namespace {
constexpr int kMaxDevices = 64;
struct ScratchAddr {
  bool ready = false;
  unsigned long long* counts = nullptr;
  long long* first = nullptr;
};
ScratchAddr g_addr[kMaxDevices];
std::mutex g_addr_mutex;

// Device address of the scratch arrays on the current device.  In host code the
// array names stand for host-side shadows, not device addresses, so the
// addresses are looked up once per device with cudaGetSymbolAddress.
cupf_status scratch_for_current_device(ScratchAddr** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return cupf_fail(CUPF_ERR_UNSUPPORTED, "device %d", dev);
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  ScratchAddr& a = g_addr[dev];
  if (!a.ready) {
    void* pc = nullptr;
    void* pf = nullptr;
    CK(cudaGetSymbolAddress(&pc, g_noalloc_counts));
    CK(cudaGetSymbolAddress(&pf, g_noalloc_first));
    a.counts = static_cast<unsigned long long*>(pc);
    a.first = static_cast<long long*>(pf);
    a.ready = true;
  }
  *out = &a;
  return CUPF_OK;
}
}  // namespace

extern "C" cupf_status cupf_grain_volumes_noalloc(const int32_t* alpha_dev, int32_t fnx,
                                                  int32_t fny, int32_t fnz, int32_t num_grains,
                                                  int64_t* counts, void* stream) {
  if (!alpha_dev || !counts) return cupf_fail(CUPF_ERR_INVALID, "null argument");
  if (fnx < 3 || fny < 3 || fnz < 3) return cupf_fail(CUPF_ERR_INVALID, "grid too small");
  if (num_grains < 0 || num_grains > CUPF_NOALLOC_MAX_GRAINS)
    return cupf_fail(CUPF_ERR_INVALID,
                     "num_grains %d outside 0..%d (the fixed scratch of the allocation-free "
                     "reduction holds %d grain ids; use cupf_apt_grain_volumes for more)",
                     num_grains, CUPF_NOALLOC_MAX_GRAINS, CUPF_NOALLOC_MAX_GRAINS);
  ScratchAddr* sc = nullptr;
  cupf_status st = scratch_for_current_device(&sc);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n = (size_t)num_grains + 1;
  // the arrays keep the previous call's contents: clear what must start fresh
  CK(cudaMemsetAsync(sc->counts, 0, n * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(sc->first, 0x7F, n * sizeof(long long), s));
  const long long ni = (long long)(fnx - 2) * (fny - 2) * (fnz - 2);
  long long nb = (ni + 255) / 256;
  if (nb > 148 * 16) nb = 148 * 16;
  if (nb < 1) nb = 1;
  volume_kernel<<<(int)nb, 256, 0, s>>>(alpha_dev, fnx, fny, fnz, num_grains, sc->counts, sc->first);
  CK(cudaGetLastError());
  static_assert(sizeof(unsigned long long) == sizeof(int64_t), "count width");
  CK(cudaMemcpyAsync(counts, sc->counts, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return CUPF_OK;
}
