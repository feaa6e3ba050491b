// capi_internal.h — error plumbing shared by the library's C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/cupf.h"

// Records a per-thread message (returned by cupf_last_error) and returns st.
cupf_status cupf_fail(cupf_status st, const char* fmt, ...);

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return cupf_fail(e_ == cudaErrorMemoryAllocation ? CUPF_ERR_OOM : CUPF_ERR_CUDA, \
                       "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),         \
                       __FILE__, __LINE__);                                            \
  } while (0)
