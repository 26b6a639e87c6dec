// The warm-start network: 33 -> 256 -> 256 -> K (K <= 16), GELU hidden layers, softmax
// output with a residual prior (logits = f(x) + prior, prior = log of the ALS memberships,
// so an untrained network reproduces the ALS start). Weights are BF16 (the fp32 master
// copies live with the optimiser), activations and accumulation FP32.
//
// Training and inference run on these kernels: a tiled GEMM (C = opA(A) opB(B), fp32 A,
// fp32 or BF16 B, arbitrary strides, so one kernel serves the forward X W', and the
// backward dY W and dY' X), bias + GELU (exact erf form) forward and backward, the fused
// softmax / cross-entropy against soft targets, column sums for the bias gradients, and
// Adam on the fp32 masters writing the BF16 copies. The network is small (about 77k
// weights; a 100k-sample forward is about 15 GFLOP), so plain CUDA-core tiles are used
// rather than tensor-core MMAs: at these widths the MMA set-up would dominate.
#include <cuda_bf16.h>

#include "common.cuh"

namespace adx {
namespace mlp {

constexpr int D_IN = 33;
constexpr int H = 256;
constexpr int KMAX = 16;

__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// C[m][n] (+)= sum_k A[m*am + k*ak] * B[k*bk + n*bn]; 64 x 64 tiles, 256 threads, 4 x 4 each.
template <typename TB>
__global__ void __launch_bounds__(256) gemm_kernel(int64_t M, int N, int K, const float* __restrict__ A,
                                                   int64_t am, int64_t ak, const TB* __restrict__ B, int64_t bk,
                                                   int64_t bn, float* __restrict__ C, int64_t ldc, int accumulate) {
  __shared__ float As[16][64 + 1];
  __shared__ float Bs[16][64 + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t m0 = (int64_t)blockIdx.y * 64;
  const int n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int kk = e / 64, r = e % 64;
      const int64_t m = m0 + r;
      const int k = k0 + kk;
      As[kk][r] = (m < M && k < K) ? A[m * am + (int64_t)k * ak] : 0.0f;
      const int n = n0 + r;
      Bs[kk][r] = (n < N && k < K) ? ld(B + (int64_t)k * bk + (int64_t)n * bn) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float* c = C + m * ldc + n;
      *c = accumulate ? *c + acc[i][j] : acc[i][j];
    }
  }
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// pre += b (in place); post = gelu(pre)
__global__ void bias_gelu_kernel(float* pre, const float* __restrict__ b, float* post, int64_t rows, int O) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * O) return;
  const float v = pre[e] + b[e % O];
  pre[e] = v;
  post[e] = gelu(v);
}

// d_pre = d_post * gelu'(pre) (in place over d_post)
__global__ void gelu_bwd_kernel(float* d, const float* __restrict__ pre, int64_t n) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) d[e] *= gelu_grad(pre[e]);
}

// logits z = z + b3 + prior (b3, prior optional); p = softmax(z); with targets:
// dz = (p - t) / B and the per-block partial of -sum t log p.
__global__ void softmax_kernel(float* z, const float* __restrict__ b, const float* __restrict__ prior,
                               const float* __restrict__ target, int64_t rows, int K, float* p, float* dz,
                               float* loss_part) {
  __shared__ float red[256];
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (r < rows) {
    float v[KMAX];
    float mx = -INFINITY;
    for (int k = 0; k < K; ++k) {
      v[k] = z[r * K + k] + (b ? b[k] : 0.0f) + (prior ? prior[r * K + k] : 0.0f);
      z[r * K + k] = v[k];
      mx = fmaxf(mx, v[k]);
    }
    float s = 0.0f;
    for (int k = 0; k < K; ++k) {
      v[k] = expf(v[k] - mx);
      s += v[k];
    }
    const float inv = 1.0f / s, ls = logf(s);
    for (int k = 0; k < K; ++k) {
      const float pk = v[k] * inv;
      p[r * K + k] = pk;
      if (target) {
        const float t = target[r * K + k];
        dz[r * K + k] = (pk - t) / (float)rows;
        // log p_k = (z_k - mx) - log s
        if (t > 0.0f) l -= t * (z[r * K + k] - mx - ls);
      }
    }
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss_part) loss_part[blockIdx.x] = red[0];
}

// db[o] = sum_r dY[r][o], in row order
__global__ void colsum_kernel(const float* __restrict__ dY, int64_t rows, int O, float* db) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= O) return;
  float s = 0.0f;
  for (int64_t r = 0; r < rows; ++r) s += dY[r * O + o];
  db[o] = s;
}

__global__ void sum_kernel(const float* part, int n, float* out, float scale) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += part[i];
    *out = s * scale;
  }
}

__global__ void adam_kernel(float* w, __nv_bfloat16* wb, const float* __restrict__ g, float* m, float* v, int64_t n,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gr = g[e];
  const float mm = b1 * m[e] + (1.0f - b1) * gr;
  const float vv = b2 * v[e] + (1.0f - b2) * gr * gr;
  m[e] = mm;
  v[e] = vv;
  const float nw = w[e] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  w[e] = nw;
  if (wb) wb[e] = __float2bfloat16_rn(nw);
}

struct Ws {
  float *h1p, *h1, *h2p, *h2, *z, *p, *d1, *d2, *dz, *loss_part;
  static size_t bytes(int64_t B, int K) {
    const int64_t rb = (B + 255) / 256;
    return (size_t)(B * (6 * (int64_t)H + 3 * K) + rb + 64) * sizeof(float);
  }
  Ws(void* base, int64_t B, int K) {
    float* f = static_cast<float*>(base);
    h1p = f; f += B * H;
    h1 = f; f += B * H;
    h2p = f; f += B * H;
    h2 = f; f += B * H;
    d1 = f; f += B * H;
    d2 = f; f += B * H;
    z = f; f += B * K;
    p = f; f += B * K;
    dz = f; f += B * K;
    loss_part = f;
  }
};

template <typename TB>
static void gemm(cudaStream_t st, int64_t M, int N, int K, const float* A, int64_t am, int64_t ak, const TB* B,
                 int64_t bk, int64_t bn, float* C, int64_t ldc, int accumulate) {
  const dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64));
  gemm_kernel<TB><<<grid, 256, 0, st>>>(M, N, K, A, am, ak, B, bk, bn, C, ldc, accumulate);
}

}  // namespace mlp
}  // namespace adx

using namespace adx;
using bf16 = __nv_bfloat16;

extern "C" int adx_mlp_workspace_bytes(int64_t B, int K, size_t* bytes) {
  if (!bytes || B <= 0 || K < 1 || K > mlp::KMAX) {
    adx_set_message("adx_mlp_workspace_bytes: bad argument");
    return ADX_ERR_ARG;
  }
  *bytes = mlp::Ws::bytes(B, K);
  return ADX_OK;
}

static bool mlp_args_ok(int64_t B, int K, const void* X, const void* W1, const void* W2, const void* W3) {
  return B > 0 && K >= 1 && K <= mlp::KMAX && X && W1 && W2 && W3;
}

// Q_out [B][K] = softmax(f(X) + prior); activations kept in the workspace for a backward.
extern "C" int adx_mlp_forward(const float* X, const float* prior, const uint16_t* W1, const float* b1,
                               const uint16_t* W2, const float* b2, const uint16_t* W3, const float* b3, int64_t B,
                               int K, float* Q_out, void* workspace, size_t workspace_bytes, void* stream) {
  if (!mlp_args_ok(B, K, X, W1, W2, W3) || !b1 || !b2 || !b3) {
    adx_set_message("adx_mlp_forward: bad argument");
    return ADX_ERR_ARG;
  }
  if (!workspace || workspace_bytes < mlp::Ws::bytes(B, K)) {
    adx_set_message("adx_mlp_forward: workspace too small");
    return ADX_ERR_WORKSPACE;
  }
  using namespace mlp;
  cudaStream_t st = as_stream(stream);
  Ws w(workspace, B, K);
  const bf16* w1 = reinterpret_cast<const bf16*>(W1);
  const bf16* w2 = reinterpret_cast<const bf16*>(W2);
  const bf16* w3 = reinterpret_cast<const bf16*>(W3);
  const unsigned eb = (unsigned)ceil_div(B * H, 256);
  gemm<bf16>(st, B, H, D_IN, X, D_IN, 1, w1, 1, D_IN, w.h1p, H, 0);
  bias_gelu_kernel<<<eb, 256, 0, st>>>(w.h1p, b1, w.h1, B, H);
  gemm<bf16>(st, B, H, H, w.h1, H, 1, w2, 1, H, w.h2p, H, 0);
  bias_gelu_kernel<<<eb, 256, 0, st>>>(w.h2p, b2, w.h2, B, H);
  gemm<bf16>(st, B, K, H, w.h2, H, 1, w3, 1, H, w.z, K, 0);
  softmax_kernel<<<(unsigned)ceil_div(B, 256), 256, 0, st>>>(w.z, b3, prior, nullptr, B, K, w.p, nullptr, nullptr);
  ADX_LAUNCH_CHECK();
  if (Q_out) ADX_CUDA_TRY(cudaMemcpyAsync(Q_out, w.p, (size_t)B * K * sizeof(float), cudaMemcpyDeviceToDevice, st));
  return ADX_OK;
}

// Cross-entropy of the last forward's softmax against soft targets T [B][K] (mean over
// rows, written to *loss) and the gradients of every weight and bias (fp32).
extern "C" int adx_mlp_backward(const float* X, const float* T, const uint16_t* W2, const uint16_t* W3, int64_t B,
                                int K, float* dW1, float* db1, float* dW2, float* db2, float* dW3, float* db3,
                                float* loss, void* workspace, size_t workspace_bytes, void* stream) {
  if (!mlp_args_ok(B, K, X, X, W2, W3) || !T || !dW1 || !db1 || !dW2 || !db2 || !dW3 || !db3 || !loss) {
    adx_set_message("adx_mlp_backward: bad argument");
    return ADX_ERR_ARG;
  }
  if (!workspace || workspace_bytes < mlp::Ws::bytes(B, K)) {
    adx_set_message("adx_mlp_backward: workspace too small");
    return ADX_ERR_WORKSPACE;
  }
  using namespace mlp;
  cudaStream_t st = as_stream(stream);
  Ws w(workspace, B, K);
  const bf16* w2 = reinterpret_cast<const bf16*>(W2);
  const bf16* w3 = reinterpret_cast<const bf16*>(W3);
  const unsigned rb = (unsigned)ceil_div(B, 256);
  // dz = (p - t) / B and the loss from the stored logits (they already hold b3 + prior)
  softmax_kernel<<<rb, 256, 0, st>>>(w.z, nullptr, nullptr, T, B, K, w.p, w.dz, w.loss_part);
  sum_kernel<<<1, 32, 0, st>>>(w.loss_part, (int)rb, loss, 1.0f / (float)B);
  // layer 3: dW3 = dz' h2, db3 = colsum dz, d2 = dz W3
  gemm<float>(st, K, H, B, w.dz, 1, K, w.h2, H, 1, dW3, H, 0);
  colsum_kernel<<<1, 32, 0, st>>>(w.dz, B, K, db3);
  gemm<bf16>(st, B, H, K, w.dz, K, 1, w3, H, 1, w.d2, H, 0);
  gelu_bwd_kernel<<<(unsigned)ceil_div(B * H, 256), 256, 0, st>>>(w.d2, w.h2p, B * H);
  // layer 2
  gemm<float>(st, H, H, B, w.d2, 1, H, w.h1, H, 1, dW2, H, 0);
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(w.d2, B, H, db2);
  gemm<bf16>(st, B, H, H, w.d2, H, 1, w2, H, 1, w.d1, H, 0);
  gelu_bwd_kernel<<<(unsigned)ceil_div(B * H, 256), 256, 0, st>>>(w.d1, w.h1p, B * H);
  // layer 1
  gemm<float>(st, H, D_IN, B, w.d1, 1, H, X, D_IN, 1, dW1, D_IN, 0);
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(w.d1, B, H, db1);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

// Adam step on an fp32 master tensor (optionally refreshing its BF16 copy); t >= 1.
extern "C" int adx_mlp_adam(float* w, uint16_t* w_bf16, const float* g, float* m, float* v, int64_t n, float lr,
                            float beta1, float beta2, float eps, int t, void* stream) {
  if (!w || !g || !m || !v || n <= 0 || t < 1) {
    adx_set_message("adx_mlp_adam: bad argument");
    return ADX_ERR_ARG;
  }
  const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
  mlp::adam_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, as_stream(stream)>>>(
      w, reinterpret_cast<bf16*>(w_bf16), g, m, v, n, lr, beta1, beta2, eps, c1, c2);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}
