// Cross-validation on the packed genotypes (adamixture/src/cv.py:58-267): hiding a fold's
// held-out entries in a copy of the packed matrix, and the fold's binomial deviance score
//
//   dev(g, mu) = g log(g / mu) + (2 - g) log((2 - g) / (2 - mu)),
//   mu = clamp(2 P_j . Q_i, 1e-10, 2 - 1e-10)      (adamixture/src/utils_c/cython/br_qn.pyx:92-150)
//
// summed over the held-out entries. Folds come either as a list of flat indices j*N + i
// (the reference's shuffled-list rule, drawn on the host with its generator) or from the
// reference's deterministic hash of the flat index (cv.py:58-78), evaluated here per entry
// so no index list is built. From a list, hiding sets the entry's two bits to 3 with an
// atomic OR on the containing 32-bit word (entries of one byte may be hidden by different
// threads). The hash rule runs one thread per packed byte (SNPs 4r..4r+3 of sample i, rows
// over blocks, samples over threads): the flat index j*N + i is a multiply-add, the thread
// owns its byte (no atomics), and for 2..16 folds the fold count is a compile-time constant
// so the hash's modulo is a multiply-high sequence, not a 64-bit division.
// Deviance sums are float64 per-block partials added in a fixed order.
#include "common.cuh"

namespace adx {
namespace cv {

constexpr int TPB = 256;
// partials of a deviance sum: 40 per SM on 148 SMs, whole waves at 4, 5 (the deviance
// kernels hold 5) or 8 resident blocks per SM
constexpr int BLOCKS = 5920;

__device__ __forceinline__ uint64_t fold_hash(uint64_t flat, uint64_t seed) {
  uint64_t h = flat + seed + 0x9E3779B97F4A7C15ull;
  h ^= h >> 30;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 27;
  h *= 0x94D049BB133111EBull;
  h ^= h >> 31;
  return h;
}

// NF > 0: the fold count as a constant; NF == 0: n_folds at run time.
template <int NF>
__device__ __forceinline__ bool in_fold(uint64_t flat, uint64_t seed, uint64_t n_folds, uint64_t fold) {
  const uint64_t h = fold_hash(flat, seed);
  if constexpr (NF > 0) return h % (uint64_t)NF == fold;
  else return h % n_folds == fold;
}

__device__ __forceinline__ void hide(uint8_t* G, int64_t N, int64_t j, int64_t i) {
  const uint64_t addr = (uint64_t)((j >> 2) * N + i);
  unsigned int* word = reinterpret_cast<unsigned int*>(G + (addr & ~uint64_t(3)));
  atomicOr(word, 3u << (8u * (unsigned)(addr & 3u) + 2u * (unsigned)(j & 3)));
}

__device__ __forceinline__ unsigned geno(const uint8_t* G, int64_t N, int64_t j, int64_t i) {
  return (G[(j >> 2) * N + i] >> (2 * (j & 3))) & 3u;
}

__device__ __forceinline__ double deviance(const double* P, const double* Q, int K, int64_t j, int64_t i,
                                           unsigned g) {
  double mu = 0.0;
  for (int k = 0; k < K; ++k) mu += Q[i * K + k] * P[j * K + k];
  mu = 2.0 * mu;
  mu = mu < 1e-10 ? 1e-10 : (mu > 2.0 - 1e-10 ? 2.0 - 1e-10 : mu);
  const double gd = (double)g, rem = 2.0 - gd;
  double d = 0.0;
  if (gd > 0.0) d += gd * log(gd / mu);
  if (rem > 0.0) d += rem * log(rem / (2.0 - mu));
  return d;
}

__global__ void mask_list_kernel(uint8_t* G, int64_t M, int64_t N, const int64_t* __restrict__ idx, int64_t n,
                                 int* err) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = idx[e];
    if (f < 0 || f >= M * N) { atomicExch(err, 1); continue; }
    hide(G, N, f / N, f % N);
  }
}

// Every (j, i) with g != 3 in the unmasked G0 and the fold's hash; hidden in G.
template <int NF>
__global__ void mask_hash_kernel(uint8_t* G, const uint8_t* __restrict__ G0, int64_t M, int64_t N, uint64_t seed,
                                 uint64_t n_folds, uint64_t fold) {
  const int64_t rows = (M + 3) >> 2;
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const int ns = (int)min((int64_t)4, M - 4 * r);
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
      const int64_t b = r * N + i;
      const unsigned byte = G0[b];
      const uint64_t f0 = (uint64_t)(4 * r) * (uint64_t)N + (uint64_t)i;
      unsigned mask = 0u;
      for (int s = 0; s < ns; ++s)
        if (((byte >> (2 * s)) & 3u) != 3u && in_fold<NF>(f0 + (uint64_t)s * (uint64_t)N, seed, n_folds, fold))
          mask |= 3u << (2 * s);
      if (mask) G[b] = (uint8_t)(G[b] | mask);
    }
  }
}

__device__ __forceinline__ void block_sum_to(double v, double* part) {
  __shared__ double red[TPB / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < TPB / 32; ++w) s += red[w];
    part[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(TPB) dev_list_kernel(const uint8_t* __restrict__ G0, int64_t M, int64_t N, int K,
                                                       const double* __restrict__ P, const double* __restrict__ Q,
                                                       const int64_t* __restrict__ idx, int64_t n, double* part) {
  double acc = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * TPB + threadIdx.x; e < n; e += (int64_t)gridDim.x * TPB) {
    const int64_t f = idx[e];
    if (f < 0 || f >= M * N) continue;
    const int64_t j = f / N, i = f - j * N;
    const unsigned g = geno(G0, N, j, i);
    if (g != 3u) acc += deviance(P, Q, K, j, i, g);
  }
  block_sum_to(acc, part);
}

template <int NF>
__global__ void __launch_bounds__(TPB) dev_hash_kernel(const uint8_t* __restrict__ G0, int64_t M, int64_t N, int K,
                                                       const double* __restrict__ P, const double* __restrict__ Q,
                                                       uint64_t seed, uint64_t n_folds, uint64_t fold, double* part) {
  double acc = 0.0;
  const int64_t rows = (M + 3) >> 2;
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const int ns = (int)min((int64_t)4, M - 4 * r);
    for (int64_t i = threadIdx.x; i < N; i += TPB) {
      const unsigned byte = G0[r * N + i];
      const uint64_t f0 = (uint64_t)(4 * r) * (uint64_t)N + (uint64_t)i;
      for (int s = 0; s < ns; ++s) {
        const unsigned g = (byte >> (2 * s)) & 3u;
        if (g != 3u && in_fold<NF>(f0 + (uint64_t)s * (uint64_t)N, seed, n_folds, fold))
          acc += deviance(P, Q, K, 4 * r + s, i, g);
      }
    }
  }
  block_sum_to(acc, part);
}

__global__ void sum_kernel(const double* part, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += part[b];
    *out = s;
  }
}

}  // namespace cv
}  // namespace adx

using namespace adx;

static bool cv_args_ok(const void* G, int64_t M, int64_t N) { return G && M > 0 && N > 0; }

// Fold counts 2..16 as compile-time constants, anything else at run time.
#define ADX_CV_FOLD_SWITCH(nf, MACRO)                                                      \
  switch (nf) {                                                                            \
    case 2: MACRO(2); break;   case 3: MACRO(3); break;   case 4: MACRO(4); break;         \
    case 5: MACRO(5); break;   case 6: MACRO(6); break;   case 7: MACRO(7); break;         \
    case 8: MACRO(8); break;   case 9: MACRO(9); break;   case 10: MACRO(10); break;       \
    case 11: MACRO(11); break; case 12: MACRO(12); break; case 13: MACRO(13); break;       \
    case 14: MACRO(14); break; case 15: MACRO(15); break; case 16: MACRO(16); break;       \
    default: MACRO(0); break;                                                              \
  }

// The masked copy is written by 32-bit atomics: it must start on a 4-byte boundary and its
// allocation (g_bytes) must cover the packed matrix rounded up to whole words.
static bool mask_buffer_ok(const void* G, int64_t M, int64_t N, size_t g_bytes) {
  const size_t need = (size_t)((M + 3) / 4) * (size_t)N;
  return !(((uintptr_t)G) & 3u) && g_bytes % 4 == 0 && g_bytes >= need;
}

extern "C" int adx_cv_workspace_bytes(size_t* bytes) {
  if (!bytes) return ADX_ERR_ARG;
  *bytes = (size_t)cv::BLOCKS * sizeof(double) + sizeof(int) + 252;
  return ADX_OK;
}

extern "C" int adx_cv_mask_list(uint8_t* G, size_t g_bytes, int64_t M, int64_t N, const int64_t* idx, int64_t n,
                                void* workspace, size_t workspace_bytes, void* stream) {
  size_t need = 0;
  adx_cv_workspace_bytes(&need);
  if (!cv_args_ok(G, M, N) || (n > 0 && !idx) || n < 0 || !mask_buffer_ok(G, M, N, g_bytes)) {
    adx_set_message("adx_cv_mask_list: bad argument (G: 4-byte aligned, g_bytes a multiple of 4 covering it)");
    return ADX_ERR_ARG;
  }
  if (!workspace || workspace_bytes < need) { adx_set_message("adx_cv_mask_list: workspace too small"); return ADX_ERR_WORKSPACE; }
  if (n == 0) return ADX_OK;
  cudaStream_t st = as_stream(stream);
  int* err = reinterpret_cast<int*>(static_cast<uint8_t*>(workspace) + cv::BLOCKS * sizeof(double));
  ADX_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  const int64_t blocks = ceil_div(n, 256) < 4096 ? ceil_div(n, 256) : 4096;
  cv::mask_list_kernel<<<(unsigned)blocks, 256, 0, st>>>(G, M, N, idx, n, err);
  ADX_LAUNCH_CHECK();
  int h_err = 0;
  ADX_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  ADX_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_err) { adx_set_message("adx_cv_mask_list: flat index out of range"); return ADX_ERR_ARG; }
  return ADX_OK;
}

extern "C" int adx_cv_mask_hash(uint8_t* G, size_t g_bytes, const uint8_t* G0, int64_t M, int64_t N, uint64_t seed,
                                int n_folds, int fold, void* stream) {
  if (!cv_args_ok(G, M, N) || !G0 || n_folds < 1 || fold < 0 || fold >= n_folds || !mask_buffer_ok(G, M, N, g_bytes)) {
    adx_set_message("adx_cv_mask_hash: bad argument (G: 4-byte aligned, g_bytes a multiple of 4 covering it)");
    return ADX_ERR_ARG;
  }
  const int64_t blocks = (int64_t)sm_count() * 8;
  cudaStream_t st = as_stream(stream);
#define ADX_MASK(NF) cv::mask_hash_kernel<NF><<<(unsigned)blocks, 256, 0, st>>>(G, G0, M, N, seed, (uint64_t)n_folds, (uint64_t)fold)
  ADX_CV_FOLD_SWITCH(n_folds, ADX_MASK)
#undef ADX_MASK
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_cv_deviance_list(const uint8_t* G0, int64_t M, int64_t N, int K, const double* P, const double* Q,
                                    const int64_t* idx, int64_t n, double* out, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  size_t need = 0;
  adx_cv_workspace_bytes(&need);
  if (!cv_args_ok(G0, M, N) || !P || !Q || !out || K < 1 || K > ADX_MAX_K || n < 0 || (n > 0 && !idx)) {
    adx_set_message("adx_cv_deviance_list: bad argument");
    return ADX_ERR_ARG;
  }
  if (!workspace || workspace_bytes < need) { adx_set_message("adx_cv_deviance_list: workspace too small"); return ADX_ERR_WORKSPACE; }
  cudaStream_t st = as_stream(stream);
  double* part = static_cast<double*>(workspace);
  cv::dev_list_kernel<<<cv::BLOCKS, cv::TPB, 0, st>>>(G0, M, N, K, P, Q, idx, n, part);
  ADX_LAUNCH_CHECK();
  cv::sum_kernel<<<1, 32, 0, st>>>(part, cv::BLOCKS, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_cv_deviance_hash(const uint8_t* G0, int64_t M, int64_t N, int K, const double* P, const double* Q,
                                    uint64_t seed, int n_folds, int fold, double* out, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  size_t need = 0;
  adx_cv_workspace_bytes(&need);
  if (!cv_args_ok(G0, M, N) || !P || !Q || !out || K < 1 || K > ADX_MAX_K || n_folds < 1 || fold < 0 ||
      fold >= n_folds) {
    adx_set_message("adx_cv_deviance_hash: bad argument");
    return ADX_ERR_ARG;
  }
  if (!workspace || workspace_bytes < need) { adx_set_message("adx_cv_deviance_hash: workspace too small"); return ADX_ERR_WORKSPACE; }
  cudaStream_t st = as_stream(stream);
  double* part = static_cast<double*>(workspace);
#define ADX_DEV(NF) cv::dev_hash_kernel<NF><<<cv::BLOCKS, cv::TPB, 0, st>>>(G0, M, N, K, P, Q, seed, (uint64_t)n_folds, (uint64_t)fold, part)
  ADX_CV_FOLD_SWITCH(n_folds, ADX_DEV)
#undef ADX_DEV
  ADX_LAUNCH_CHECK();
  cv::sum_kernel<<<1, 32, 0, st>>>(part, cv::BLOCKS, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

