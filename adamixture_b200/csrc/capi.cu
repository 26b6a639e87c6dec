// Library-wide C ABI helpers: version, last-error message, device properties.
#include "common.cuh"

#include <stdio.h>
#include <string.h>

static thread_local char g_msg[512] = "";

void adx_set_message(const char* msg) {
  strncpy(g_msg, msg ? msg : "", sizeof(g_msg) - 1);
  g_msg[sizeof(g_msg) - 1] = 0;
}

void adx_set_cuda_error(cudaError_t e) {
  snprintf(g_msg, sizeof(g_msg), "CUDA error %d: %s", (int)e, cudaGetErrorString(e));
}

extern "C" const char* adx_version(void) { return "adamixture_b200 0.1.0 (sm_100a)"; }

extern "C" const char* adx_last_error(void) { return g_msg; }

namespace adx {

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cache[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

}  // namespace adx
