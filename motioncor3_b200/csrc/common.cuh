// Shared device helpers and error plumbing for libmc3.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "fft_core.cuh"
#include "profile.h"

namespace mc3 {

// Status codes surfaced through the C ABI (include/mc3.h).
enum Status : int {
  kOk = 0,
  kEInval = 1,
  kENoMem = 2,
  kECuda = 3,
  kETimeout = 4,
  kEIo = 5,
  kEUnsupported = 6,
};

// Records the first CUDA error and returns it as a status code.
int cuda_status(cudaError_t e, const char* where);
int last_cuda_status(const char* where);

#define MC3_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return ::mc3::cuda_status(_e, #call); \
  } while (0)

#define MC3_CHECK_LAUNCH(where)                          \
  do {                                                   \
    cudaError_t _e = cudaGetLastError();                 \
    if (_e != cudaSuccess) return ::mc3::cuda_status(_e, where); \
  } while (0)

#define MC3_TRY(expr)                 \
  do {                                \
    int _s = (expr);                  \
    if (_s != ::mc3::kOk) return _s;  \
  } while (0)

inline __host__ __device__ int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Wrapped Fourier index along an axis of length n: (-n/2, n/2].
__host__ __device__ __forceinline__ int wrap_half(int y, int n) { return y > n / 2 ? y - n : y; }

}  // namespace mc3
