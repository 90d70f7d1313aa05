// Small CUDA helpers shared by the .cu translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "jsc_internal.h"

// Kernel launch counter, readable through jsc_launch_count().
extern "C" void jsc_count_launch(void);

#define JSC_CUDA_TRY(call)                                                  \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      jsc_set_error(JSC_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                    cudaGetErrorString(e_));                                \
      return JSC_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

#define JSC_LAUNCH_CHECK()                                                  \
  do {                                                                      \
    jsc_count_launch();                                                     \
    cudaError_t e_ = cudaGetLastError();                                    \
    if (e_ != cudaSuccess) {                                                \
      jsc_set_error(JSC_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,   \
                    cudaGetErrorString(e_));                                \
      return JSC_ERR_CUDA;                                                  \
    }                                                                       \
  } while (0)

// Device status word bits (set by kernels, read by the host after a run).
#define JSC_DEV_ERR_NLOS 1u
#define JSC_DEV_ERR_OBSERVER 2u
#define JSC_DEV_ERR_QUEUE 4u
#define JSC_DEV_ERR_WATCHDOG 8u

template <typename T>
static int jsc_dmalloc(T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    jsc_set_error(JSC_ERR_NOMEM, "cudaMalloc of %zu bytes: %s", n * sizeof(T),
                  cudaGetErrorString(e));
    *p = nullptr;
    return JSC_ERR_NOMEM;
  }
  return JSC_OK;
}
