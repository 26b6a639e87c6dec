// Products of the centred genotype matrix with skinny float32 factors, for the shifted
// randomized SVD initialisation (adamixture/model/svd_gpu.py:40-154):
//
//   rows:  Y[M][L] = Xc . B      (B [N][L])      svd_gpu.py:106, 138 (proj = X @ orth)
//   cols:  Z[N][L] (+)= Xc' . Y  (Y [M][L])      svd_gpu.py:86, 107 (accum += X.T @ proj)
//
// Xc[j][i] = g_ji - 2 f_j, 0 where missing (adamixture/src/utils_c/cuda/pack2bit.cu:46-77).
// The reference decodes each 8192-SNP chunk into a float32 [chunk][N] matrix and hands it
// to cuBLAS; here each CTA decodes 32-SNP x 128-sample tiles of the packed matrix into
// shared memory and contracts them on the spot, so the only HBM traffic is the packed
// genotypes (0.25 B per entry) and the factors.
//
// Both kernels: 256 threads = 64 groups of OP "own" indices (SNPs for rows, samples for
// cols; OP = 8 while L <= 32, else 4) x 4 groups of C = LP/4 factor columns; each thread
// keeps an OP x C float32 tile of the output in registers and walks the contracted axis in
// chunks staged in shared memory (factor rows of the chunk, decoded genotype block of 32 KB).
// A thread's own indices are OP/4 runs of 4 spaced 256 apart, so each 16-byte load of the
// decoded block covers 512 contiguous bytes across the warp (no bank conflicts); shared
// loads per FMA are about 1/C + 1/OP. L <= 80 (LP = L rounded up to 4). Partial sums of the
// cols product over SNP ranges go to a workspace and are added in a fixed order, so
// results do not depend on scheduling.
#include "common.cuh"

namespace adx {
namespace rsvd {

constexpr int TPB = 256;
constexpr int OG = 64;        // own groups
constexpr int CG = 4;         // column groups
constexpr int CH = 32;        // granularity of the cols product's SNP ranges
constexpr int LMAX = 80;
constexpr int XS_FLOATS = 8192;  // decoded block: 32 KB

// own indices per thread for C columns per thread
__host__ __device__ constexpr int own_per_thread(int C) { return C <= 8 ? 8 : 4; }

__device__ __forceinline__ float centred(uint32_t byte, int s, float two_f) {
  const uint32_t g = (byte >> (2 * s)) & 3u;
  return g == 3u ? 0.0f : (float)g - two_f;
}

// own index of (thread group og, run v, slot q)
__device__ __forceinline__ int own_of(int og, int v, int q) { return v * (OG * 4) + og * 4 + q; }

// Y[j][:] = sum_i Xc[j][i] B[i][:] for the OWN SNPs of this CTA.
template <int C>  // columns per thread = LP / 4
__global__ void __launch_bounds__(TPB) rows_kernel(const uint8_t* __restrict__ G, int64_t M, int64_t N,
                                                   const float* __restrict__ f, const float* __restrict__ B,
                                                   int L, float* __restrict__ Y) {
  constexpr int LP = C * CG, OP = own_per_thread(C), OWN = OG * OP, CHK = XS_FLOATS / OWN;
  __shared__ __align__(16) float xs[CHK][OWN];   // [sample][snp]
  __shared__ __align__(16) float bs[CHK][LP];
  __shared__ float tf[OWN];
  const int tid = threadIdx.x, og = tid & (OG - 1), cg = tid / OG;
  const int64_t j0 = (int64_t)blockIdx.x * OWN;
  for (int t = tid; t < OWN; t += TPB) {
    const int64_t j = j0 + t;
    tf[t] = j < M ? 2.0f * f[j] : 0.0f;
  }
  float acc[OP][C];
#pragma unroll
  for (int a = 0; a < OP; ++a)
#pragma unroll
    for (int c = 0; c < C; ++c) acc[a][c] = 0.0f;
  const int64_t rows = (M + 3) >> 2;
  for (int64_t i0 = 0; i0 < N; i0 += CHK) {
    __syncthreads();
    for (int e = tid; e < CHK * LP; e += TPB) {
      const int s = e / LP, l = e - s * LP;
      const int64_t i = i0 + s;
      bs[s][l] = (i < N && l < L) ? B[i * L + l] : 0.0f;
    }
    // OWN/4 packed rows x CHK samples: one byte gives 4 SNPs of one sample
    for (int e = tid; e < (OWN / 4) * CHK; e += TPB) {
      const int pr = e / CHK, s = e - pr * CHK;
      const int64_t row = (j0 >> 2) + pr, i = i0 + s;
      const uint32_t byte = (row < rows && i < N) ? (uint32_t)G[row * N + i] : 0xFFu;
#pragma unroll
      for (int q = 0; q < 4; ++q) xs[s][pr * 4 + q] = centred(byte, q, tf[pr * 4 + q]);
    }
    __syncthreads();
    const int smax = (int)min((int64_t)CHK, N - i0);
    for (int s = 0; s < smax; ++s) {
      float x[OP];
#pragma unroll
      for (int v = 0; v < OP / 4; ++v) {
        const float4 x4 = *reinterpret_cast<const float4*>(&xs[s][own_of(og, v, 0)]);
        x[4 * v] = x4.x; x[4 * v + 1] = x4.y; x[4 * v + 2] = x4.z; x[4 * v + 3] = x4.w;
      }
      float b[C];
#pragma unroll
      for (int c = 0; c < C; ++c) b[c] = bs[s][cg * C + c];
#pragma unroll
      for (int a = 0; a < OP; ++a)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[a][c] = fmaf(x[a], b[c], acc[a][c]);
    }
  }
#pragma unroll
  for (int a = 0; a < OP; ++a) {
    const int64_t j = j0 + own_of(og, a >> 2, a & 3);
    if (j >= M) continue;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const int l = cg * C + c;
      if (l < L) Y[j * L + l] = acc[a][c];
    }
  }
}

// Partial Z over one SNP range for the OWN samples of this CTA: part[split][i][:].
template <int C>
__global__ void __launch_bounds__(TPB) cols_kernel(const uint8_t* __restrict__ G, int64_t M, int64_t N,
                                                   const float* __restrict__ f, const float* __restrict__ Yf,
                                                   int L, int64_t snps_per_split, float* __restrict__ part) {
  constexpr int LP = C * CG, OP = own_per_thread(C), OWN = OG * OP, CHK = XS_FLOATS / OWN;
  static_assert(CHK % 4 == 0 && CH % CHK == 0, "SNP chunks are whole packed rows inside a range");
  __shared__ __align__(16) float xs[CHK][OWN];   // [snp][sample]
  __shared__ __align__(16) float ys[CHK][LP];
  __shared__ float tf[CHK];
  const int tid = threadIdx.x, og = tid & (OG - 1), cg = tid / OG;
  const int64_t n_tiles = (N + OWN - 1) / OWN;
  const int64_t tile = blockIdx.x % n_tiles;
  const int split = (int)(blockIdx.x / n_tiles);
  const int64_t i0 = tile * OWN;
  const int64_t js = (int64_t)split * snps_per_split;
  const int64_t je = min(M, js + snps_per_split);
  float acc[OP][C];
#pragma unroll
  for (int a = 0; a < OP; ++a)
#pragma unroll
    for (int c = 0; c < C; ++c) acc[a][c] = 0.0f;
  for (int64_t j0 = js; j0 < je; j0 += CHK) {
    __syncthreads();
    for (int e = tid; e < CHK * LP; e += TPB) {
      const int s = e / LP, l = e - s * LP;
      const int64_t j = j0 + s;
      ys[s][l] = (j < je && l < L) ? Yf[j * L + l] : 0.0f;
    }
    if (tid < CHK) {
      const int64_t j = j0 + tid;
      tf[tid] = j < je ? 2.0f * f[j] : 0.0f;
    }
    __syncthreads();
    // CHK SNPs (CHK/4 packed rows; js is a multiple of 4) x OWN samples
    for (int e = tid; e < (CHK / 4) * OWN; e += TPB) {
      const int pr = e / OWN, s = e - pr * OWN;
      const int64_t row = (j0 >> 2) + pr, i = i0 + s;
      const uint32_t byte = (j0 + pr * 4 < je && i < N) ? (uint32_t)G[row * N + i] : 0xFFu;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const bool in = j0 + pr * 4 + q < je;
        xs[pr * 4 + q][s] = in ? centred(byte, q, tf[pr * 4 + q]) : 0.0f;
      }
    }
    __syncthreads();
    const int jmax = (int)min((int64_t)CHK, je - j0);
    for (int s = 0; s < jmax; ++s) {
      float x[OP];
#pragma unroll
      for (int v = 0; v < OP / 4; ++v) {
        const float4 x4 = *reinterpret_cast<const float4*>(&xs[s][own_of(og, v, 0)]);
        x[4 * v] = x4.x; x[4 * v + 1] = x4.y; x[4 * v + 2] = x4.z; x[4 * v + 3] = x4.w;
      }
      float y[C];
#pragma unroll
      for (int c = 0; c < C; ++c) y[c] = ys[s][cg * C + c];
#pragma unroll
      for (int a = 0; a < OP; ++a)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[a][c] = fmaf(x[a], y[c], acc[a][c]);
    }
  }
  float* out = part + (int64_t)split * N * L;
#pragma unroll
  for (int a = 0; a < OP; ++a) {
    const int64_t i = i0 + own_of(og, a >> 2, a & 3);
    if (i >= N) continue;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const int l = cg * C + c;
      if (l < L) out[i * L + l] = acc[a][c];
    }
  }
}

// Z (+)= sum over splits of part, in split order.
__global__ void reduce_kernel(const float* __restrict__ part, int n_split, int64_t n, int accumulate,
                              float* __restrict__ Z) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float v = accumulate ? Z[e] : 0.0f;
  for (int s = 0; s < n_split; ++s) v += part[(int64_t)s * n + e];
  Z[e] = v;
}

struct ColsPlan {
  int n_split;
  int64_t snps_per_split;
  size_t bytes;
};

static ColsPlan cols_plan(int64_t M, int64_t N, int L) {
  ColsPlan p{};
  const int C = (L + CG - 1) / CG;
  const int64_t tiles = ceil_div(N, (int64_t)OG * own_per_thread(C));
  // enough CTAs for about 4 per SM; SNP ranges are whole chunks
  int64_t split = ceil_div((int64_t)sm_count() * 4, tiles);
  const int64_t chunks = ceil_div(M, CH);
  split = split < 1 ? 1 : (split > chunks ? chunks : split);
  p.snps_per_split = ceil_div(chunks, split) * CH;
  p.n_split = (int)ceil_div(M, p.snps_per_split);
  p.bytes = (size_t)p.n_split * (size_t)N * (size_t)L * sizeof(float);
  return p;
}

}  // namespace rsvd
}  // namespace adx

using namespace adx;

#define ADX_LP_SWITCH(L, X)                                                              \
  switch ((L + 3) / 4) {                                                                 \
    case 1: X(1) break;   case 2: X(2) break;   case 3: X(3) break;   case 4: X(4) break;   \
    case 5: X(5) break;   case 6: X(6) break;   case 7: X(7) break;   case 8: X(8) break;   \
    case 9: X(9) break;   case 10: X(10) break; case 11: X(11) break; case 12: X(12) break; \
    case 13: X(13) break; case 14: X(14) break; case 15: X(15) break; case 16: X(16) break; \
    case 17: X(17) break; case 18: X(18) break; case 19: X(19) break; default: X(20) break; \
  }

extern "C" int adx_rsvd_workspace_bytes(int64_t M, int64_t N, int L, size_t* bytes) {
  if (!bytes || M <= 0 || N <= 0 || L < 1 || L > rsvd::LMAX) {
    adx_set_message("adx_rsvd_workspace_bytes: bad argument");
    return ADX_ERR_ARG;
  }
  *bytes = rsvd::cols_plan(M, N, L).bytes;
  return ADX_OK;
}

extern "C" int adx_rsvd_rows(const uint8_t* G, int64_t M, int64_t N, const float* f, const float* B, int L,
                             float* Y, void* stream) {
  if (!G || !f || !B || !Y || M <= 0 || N <= 0 || L < 1 || L > rsvd::LMAX) {
    adx_set_message("adx_rsvd_rows: bad argument");
    return ADX_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  const int64_t own = (int64_t)rsvd::OG * rsvd::own_per_thread((L + rsvd::CG - 1) / rsvd::CG);
  const unsigned blocks = (unsigned)ceil_div(M, own);
#define LAUNCH(C) rsvd::rows_kernel<C><<<blocks, rsvd::TPB, 0, st>>>(G, M, N, f, B, L, Y);
  ADX_LP_SWITCH(L, LAUNCH)
#undef LAUNCH
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_rsvd_cols(const uint8_t* G, int64_t M, int64_t N, const float* f, const float* Y, int L,
                             int accumulate, float* Z, void* workspace, size_t workspace_bytes, void* stream) {
  if (!G || !f || !Y || !Z || M <= 0 || N <= 0 || L < 1 || L > rsvd::LMAX) {
    adx_set_message("adx_rsvd_cols: bad argument");
    return ADX_ERR_ARG;
  }
  const rsvd::ColsPlan p = rsvd::cols_plan(M, N, L);
  if (!workspace || workspace_bytes < p.bytes) {
    adx_set_message("adx_rsvd_cols: workspace too small");
    return ADX_ERR_WORKSPACE;
  }
  cudaStream_t st = as_stream(stream);
  float* part = static_cast<float*>(workspace);
  const int64_t own = (int64_t)rsvd::OG * rsvd::own_per_thread((L + rsvd::CG - 1) / rsvd::CG);
  const unsigned blocks = (unsigned)(ceil_div(N, own) * p.n_split);
#define LAUNCH(C) rsvd::cols_kernel<C><<<blocks, rsvd::TPB, 0, st>>>(G, M, N, f, Y, L, p.snps_per_split, part);
  ADX_LP_SWITCH(L, LAUNCH)
#undef LAUNCH
  ADX_LAUNCH_CHECK();
  const int64_t n = N * (int64_t)L;
  rsvd::reduce_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(part, p.n_split, n, accumulate, Z);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}
