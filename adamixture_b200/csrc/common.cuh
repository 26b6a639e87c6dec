// Shared definitions for the adamixture_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/adamixture_b200.h"

#define ADX_CUDA_TRY(expr)                                    \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) { adx_set_cuda_error(_e); return ADX_ERR_CUDA; } \
  } while (0)

#define ADX_LAUNCH_CHECK()                                    \
  do {                                                        \
    cudaError_t _e = cudaGetLastError();                      \
    if (_e != cudaSuccess) { adx_set_cuda_error(_e); return ADX_ERR_CUDA; } \
  } while (0)

// Last CUDA error seen by the library (thread-local), readable through adx_last_error().
void adx_set_cuda_error(cudaError_t e);
void adx_set_message(const char* msg);

namespace adx {

constexpr double E_CLAMP = 1e-5;    // E-step reconstruction clamp
constexpr double LL_CLAMP = 1e-10;  // log-likelihood clamp
constexpr double DOMAIN = 1e-5;     // P/Q domain clamp after a step

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

__device__ __forceinline__ unsigned genotype(uint32_t byte, int s) { return (byte >> (2 * s)) & 3u; }

}  // namespace adx
