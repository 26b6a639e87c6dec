// The warm-start network: 33 -> 256 -> 256 -> K (K <= 16), GELU hidden layers, softmax
// output with a residual prior (logits = f(x) + prior, prior = log of the ALS memberships,
// so an untrained network reproduces the ALS start). Weights are BF16 (the fp32 master
// copies live with the optimiser), activations fp32, products on the tensor cores.
//
// Training and inference run on these kernels: a BF16 tensor-core GEMM (mma.sync m16n8k16,
// FP32 accumulation; C = A B with arbitrary strides, fp32 A and fp32 or BF16 B rounded to
// BF16 as they are staged, so one kernel serves the forward X W', the backward dY W and the
// weight gradients dY' X, the last split over the batch with partial products summed in a
// fixed order), bias + GELU (exact erf form) forward and backward, the fused softmax /
// cross-entropy against soft targets, column sums for the bias gradients, and Adam on the
// fp32 masters writing the BF16 copies.
#include <cuda_bf16.h>

#include "common.cuh"

namespace adx {
namespace mlp {

constexpr int D_IN = 33;
constexpr int H = 256;
constexpr int KMAX = 16;

__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// ---------------------------------------------------------------- BF16 tensor-core GEMM
//
// C[m][n] (+)= sum_k A(m, k) B(k, n), A(m, k) = A[m*am + k*ak] (fp32), B(k, n) = B[k*bk + n*bn]
// (fp32 or BF16); both are rounded to BF16 as they are staged in shared memory and the
// products accumulate in FP32 (mma.sync.m16n8k16 .bf16, fragments: A rows g and g+8,
// columns 2t, 2t+1 (+8); B rows 2t, 2t+1 (+8), column g; C rows g, g+8, columns 2t, 2t+1;
// g = lane / 4, t = lane % 4). CTA tile 128 x 64 over 8 warps of 32 x 32 (2 x 4 MMA tiles),
// k in steps of 32. Shared tiles are stored [row][k] (B transposed) with a row stride of 40
// BF16 (20 words), so each fragment's 32-bit loads hit 32 different banks. With
// gridDim.z > 1 the k range is split and CTA z writes its product to part[z] (M x N fp32);
// gemm_reduce_kernel adds the splits in order.
constexpr int GT_M = 128, GT_N = 64, GT_K = 32, GT_S = 40;

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <typename TB>
__global__ void __launch_bounds__(256) gemm_mma_kernel(int64_t M, int N, int64_t K, int64_t kchunk,
                                                       const float* __restrict__ A, int64_t am, int64_t ak,
                                                       const TB* __restrict__ B, int64_t bk, int64_t bn,
                                                       float* __restrict__ C, int64_t ldc, int accumulate,
                                                       float* __restrict__ part) {
  __shared__ __align__(16) __nv_bfloat16 As[GT_M * GT_S];
  __shared__ __align__(16) __nv_bfloat16 Bs[GT_N * GT_S];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;   // the warp's 32 x 32 block
  const int64_t m0 = (int64_t)blockIdx.y * GT_M;
  const int n0 = blockIdx.x * GT_N;
  const int64_t k_lo = (int64_t)blockIdx.z * kchunk;
  const int64_t k_hi = min(K, k_lo + kchunk);
  float acc[2][4][4] = {};
  for (int64_t k0 = k_lo; k0 < k_hi; k0 += GT_K) {
    // stage A (128 x 32) and B^T (64 x 32) as BF16; the index order follows the operand's
    // contiguous dimension so that consecutive threads read consecutive addresses
    for (int e = threadIdx.x; e < GT_M * GT_K; e += 256) {
      const int r = am == 1 ? (e % GT_M) : (e / GT_K), kk = am == 1 ? (e / GT_M) : (e % GT_K);
      const int64_t m = m0 + r, k = k0 + kk;
      As[r * GT_S + kk] = __float2bfloat16_rn((m < M && k < k_hi) ? A[m * am + k * ak] : 0.0f);
    }
    for (int e = threadIdx.x; e < GT_N * GT_K; e += 256) {
      const int c = bn == 1 ? (e % GT_N) : (e / GT_K), kk = bn == 1 ? (e / GT_N) : (e % GT_K);
      const int n = n0 + c;
      const int64_t k = k0 + kk;
      float v = 0.0f;
      if (n < N && k < k_hi) v = ld(B + k * bk + (int64_t)n * bn);
      Bs[c * GT_S + kk] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    const uint32_t* Aw = reinterpret_cast<const uint32_t*>(As);
    const uint32_t* Bw = reinterpret_cast<const uint32_t*>(Bs);
#pragma unroll
    for (int ks = 0; ks < GT_K; ks += 16) {
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + 16 * i + g;
        a[i][0] = Aw[(r * GT_S + ks + 2 * t) >> 1];
        a[i][1] = Aw[((r + 8) * GT_S + ks + 2 * t) >> 1];
        a[i][2] = Aw[(r * GT_S + ks + 8 + 2 * t) >> 1];
        a[i][3] = Aw[((r + 8) * GT_S + ks + 8 + 2 * t) >> 1];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + 8 * j + g;
        b[j][0] = Bw[(c * GT_S + ks + 2 * t) >> 1];
        b[j][1] = Bw[(c * GT_S + ks + 8 + 2 * t) >> 1];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i][0], a[i][1], a[i][2], a[i][3], b[j][0], b[j][1]);
    }
    __syncthreads();
  }
  float* out = part ? part + (int64_t)blockIdx.z * M * N : C;
  const int64_t ldo = part ? N : ldc;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t m = m0 + wm + 16 * i + g + 8 * (e >> 1);
        const int n = n0 + wn + 8 * j + 2 * t + (e & 1);
        if (m >= M || n >= N) continue;
        float* c = out + m * ldo + n;
        *c = (accumulate && !part) ? *c + acc[i][j][e] : acc[i][j][e];
      }
}

// C[m][n] (+)= sum over splits z in order of part[z][m][n]
__global__ void gemm_reduce_kernel(const float* __restrict__ part, int splits, int64_t M, int N, float* C,
                                   int64_t ldc, int accumulate) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * N) return;
  float s = 0.0f;
  for (int z = 0; z < splits; ++z) s += part[(int64_t)z * M * N + e];
  const int64_t m = e / N, n = e % N;
  C[m * ldc + n] = accumulate ? C[m * ldc + n] + s : s;
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

// Splits of the weight-gradient GEMMs' batch axis: about 4 CTAs per SM over the 2 x 4
// (or fewer) output tiles, each split at least 256 rows.
constexpr int MAX_SPLITS = 64;

struct Ws {
  float *h1p, *h1, *h2p, *h2, *z, *p, *d1, *d2, *dz, *loss_part, *part;
  static size_t bytes(int64_t B, int K) {
    const int64_t rb = (B + 255) / 256;
    return (size_t)(B * (6 * (int64_t)H + 3 * K) + rb + 64 + (int64_t)MAX_SPLITS * H * H) * sizeof(float);
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
    loss_part = f; f += (B + 255) / 256 + 64;
    part = f;
  }
};

// C = A B (+ C) on the tensor cores; a long k axis (the batch, for weight gradients) is
// split over up to MAX_SPLITS CTAs per output tile and reduced in order through `part`.
template <typename TB>
static void gemm(cudaStream_t st, int64_t M, int N, int64_t K, const float* A, int64_t am, int64_t ak, const TB* B,
                 int64_t bk, int64_t bn, float* C, int64_t ldc, int accumulate, float* part = nullptr) {
  const int64_t tiles = ((M + GT_M - 1) / GT_M) * ((N + GT_N - 1) / GT_N);
  int splits = 1;
  if (part && tiles < 148) {
    const int64_t want = (148 * 4 + tiles - 1) / tiles;
    const int64_t cap = (K + 255) / 256;
    int64_t sp = want < cap ? want : cap;
    sp = sp < MAX_SPLITS ? sp : MAX_SPLITS;
    splits = (int)sp;
    splits = splits < 1 ? 1 : splits;
  }
  int64_t kchunk = (K + splits - 1) / splits;
  kchunk = (kchunk + GT_K - 1) / GT_K * GT_K;
  splits = (int)((K + kchunk - 1) / kchunk);
  const dim3 grid((unsigned)((N + GT_N - 1) / GT_N), (unsigned)((M + GT_M - 1) / GT_M), (unsigned)splits);
  gemm_mma_kernel<TB><<<grid, 256, 0, st>>>(M, N, K, kchunk, A, am, ak, B, bk, bn, C, ldc, accumulate,
                                            splits > 1 ? part : nullptr);
  if (splits > 1)
    gemm_reduce_kernel<<<(unsigned)((M * N + 255) / 256), 256, 0, st>>>(part, splits, M, N, C, ldc, accumulate);
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
  gemm<float>(st, K, H, B, w.dz, 1, K, w.h2, H, 1, dW3, H, 0, w.part);
  colsum_kernel<<<1, 32, 0, st>>>(w.dz, B, K, db3);
  gemm<bf16>(st, B, H, K, w.dz, K, 1, w3, H, 1, w.d2, H, 0);
  gelu_bwd_kernel<<<(unsigned)ceil_div(B * H, 256), 256, 0, st>>>(w.d2, w.h2p, B * H);
  // layer 2
  gemm<float>(st, H, H, B, w.d2, 1, H, w.h1, H, 1, dW2, H, 0, w.part);
  colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(w.d2, B, H, db2);
  gemm<bf16>(st, B, H, H, w.d2, H, 1, w2, H, 1, w.d1, H, 0);
  gelu_bwd_kernel<<<(unsigned)ceil_div(B * H, 256), 256, 0, st>>>(w.d1, w.h1p, B * H);
  // layer 1
  gemm<float>(st, H, D_IN, B, w.d1, 1, H, X, D_IN, 1, dW1, D_IN, 0, w.part);
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
