// Packed-genotype layout kernels: decode, centring, per-SNP frequencies, per-sample counts,
// PLINK BED ingestion (decode + flip) and the synthetic cohort sampler.
//
// Packed layout: G[ceil(M/4)][N] uint8, byte (j>>2)*N + i holds SNP j of sample i in bits
// 2*(j&3) (adamixture/src/utils_c/cython/snp_reader.pyx:76-120). Consecutive samples are
// consecutive bytes, so every kernel here reads rows of G with consecutive threads on
// consecutive samples (coalesced), 16 bytes per thread where the row alignment allows.
#include "common.cuh"

namespace adx {

// ---------------------------------------------------------------- decode (pack2bit.cu:15-77)

__global__ void unpack_u8_kernel(const uint8_t* __restrict__ G, int64_t N, int64_t M_total,
                                 int64_t m_start, int64_t count, int64_t byte_offset,
                                 uint8_t* __restrict__ out) {
  const int64_t total = count * N;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t lm = idx / N, i = idx - lm * N;
    const int64_t j = m_start + lm;
    uint8_t v = 3;
    if (j < M_total && (j >> 2) >= byte_offset)
      v = (uint8_t)genotype(G[((j >> 2) - byte_offset) * N + i], (int)(j & 3));
    out[idx] = v;
  }
}

__global__ void unpack_center_kernel(const uint8_t* __restrict__ G, int64_t N, int64_t M_total,
                                     int64_t m_start, int64_t count, int64_t byte_offset,
                                     const float* __restrict__ f, float* __restrict__ out) {
  const int64_t total = count * N;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t lm = idx / N, i = idx - lm * N;
    const int64_t j = m_start + lm;
    float v = 0.0f;
    if (j < M_total && (j >> 2) >= byte_offset) {
      const unsigned g = genotype(G[((j >> 2) - byte_offset) * N + i], (int)(j & 3));
      v = g == 3u ? 0.0f : ((float)g - 2.0f * f[j]);
    }
    out[idx] = v;
  }
}

// ---------------------------------------------------------------- per-SNP frequencies

// One warp per packed row (4 SNPs): sums and observed counts of the 4 SNPs over all samples.
__global__ void allele_freq_kernel(const uint8_t* __restrict__ G, int64_t M, int64_t N,
                                   float* __restrict__ f) {
  const int64_t rows = (M + 3) >> 2;
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    unsigned long long sum[4] = {0, 0, 0, 0}, cnt[4] = {0, 0, 0, 0};
    const uint8_t* row = G + r * N;
    for (int64_t i = lane; i < N; i += 32) {
      const uint32_t b = row[i];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const unsigned g = genotype(b, s);
        if (g != 3u) { sum[s] += g; cnt[s] += 1; }
      }
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) {
        sum[s] += __shfl_xor_sync(0xffffffffu, sum[s], o);
        cnt[s] += __shfl_xor_sync(0xffffffffu, cnt[s], o);
      }
    }
    if (lane < 4) {
      const int64_t j = r * 4 + lane;
      if (j < M) {
        // utils.py:826-829: f = sum / (2 * count) where count > 0, else 0 (float32 math)
        const float s = (float)sum[lane], c = (float)cnt[lane];
        f[j] = cnt[lane] ? s / (2.0f * c) : 0.0f;
      }
    }
  }
}

// ---------------------------------------------------------------- per-sample counts

// q_bat_i = 2 * #observed SNPs of sample i. A byte holds 4 SNPs; a 2-bit field is missing
// iff both bits are set, so #missing = popc(b & (b >> 1) & 0x55). Padding fields of the last
// row are 0 (observed) and are excluded. Blocks on grid.y cover disjoint row ranges and add
// their integer counts into q_bat with float64 atomics: integer-valued doubles below 2^53
// add exactly, so the result does not depend on the order.
__global__ void sample_counts_kernel(const uint8_t* __restrict__ G, int64_t M, int64_t N,
                                     int64_t rows_per_part, double* __restrict__ q_bat) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t rows = (M + 3) >> 2;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_part;
  const int64_t r1 = min(rows, r0 + rows_per_part);
  if (r0 >= r1) return;
  unsigned long long miss = 0;
  for (int64_t r = r0; r < r1; ++r) {
    const uint32_t b = G[r * N + i];
    miss += __popc(b & (b >> 1) & 0x55u);
  }
  int64_t snps = min(M, r1 * 4) - r0 * 4;
  atomicAdd(q_bat + i, 2.0 * (double)(snps - (int64_t)miss));
}

// Heterozygous genotype (g = 1, bits 01) count per sample, same partition and exact
// integer-valued float64 atomics as sample_counts_kernel; padding bits are 00 (g = 0).
__global__ void het_counts_kernel(const uint8_t* __restrict__ G, int64_t M, int64_t N,
                                  int64_t rows_per_part, double* __restrict__ het) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int64_t rows = (M + 3) >> 2;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_part;
  const int64_t r1 = min(rows, r0 + rows_per_part);
  if (r0 >= r1) return;
  unsigned long long h = 0;
  for (int64_t r = r0; r < r1; ++r) {
    const uint32_t b = G[r * N + i];
    h += __popc(b & ~(b >> 1) & 0x55u);
  }
  atomicAdd(het + i, (double)h);
}

// ---------------------------------------------------------------- synthetic sampler

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 27;
  z *= 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z;
}

template <int KMAX>
__global__ void simulate_kernel(const uint32_t* __restrict__ Pq, const uint32_t* __restrict__ Qq,
                                int64_t M, int64_t N, int K, uint64_t key1, uint64_t key2,
                                uint32_t miss_q, uint8_t* __restrict__ G) {
  // one thread per sample, grid-stride over packed rows (blockIdx.y)
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  uint32_t q[KMAX];
#pragma unroll
  for (int k = 0; k < KMAX; ++k) q[k] = k < K ? Qq[i * K + k] : 0u;
  const int64_t rows = (M + 3) >> 2;
  for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
    uint32_t byte = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int64_t j = r * 4 + s;
      if (j >= M) break;
      uint64_t hq = 0;
#pragma unroll
      for (int k = 0; k < KMAX; ++k)
        if (k < K) hq += (uint64_t)__ldg(Pq + j * K + k) * q[k];
      const uint64_t c = ((uint64_t)j * (uint64_t)N + (uint64_t)i) * 0x9E3779B97F4A7C15ull;
      const uint64_t z1 = splitmix64(c + key1);
      const uint64_t z2 = splitmix64(c + key2);
      uint32_t g = (uint32_t)((z1 & 0xFFFFFFFFull) < hq) + (uint32_t)((z1 >> 32) < hq);
      if ((uint32_t)(z2 & 0xFFFFFFFFull) < miss_q) g = 3u;
      byte |= g << (2 * s);
    }
    G[r * N + i] = (uint8_t)byte;
  }
}

// ---------------------------------------------------------------- PLINK BED -> packed

// One thread per output byte (packed row r, sample i): the 4 SNPs' 2-bit BED codes of
// sample i decode through LUT [2,3,1,0] (snp_reader.pyx:53-58). Also accumulates the sum
// of dosages and the observed count per block for the flip decision.
__global__ void bed_decode_kernel(const uint8_t* __restrict__ bed, int64_t M, int64_t N,
                                  uint8_t* __restrict__ G, unsigned long long* __restrict__ acc) {
  __shared__ unsigned long long sh[2];
  if (threadIdx.x < 2) sh[threadIdx.x] = 0;
  __syncthreads();
  const int64_t nb = (N + 3) >> 2;
  const int64_t rows = (M + 3) >> 2;
  const int64_t total = rows * N;
  unsigned long long s = 0, c = 0;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / N, i = idx - r * N;
    uint32_t out = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t j = r * 4 + k;
      if (j >= M) break;
      const uint32_t code = (bed[j * nb + (i >> 2)] >> (2 * (i & 3))) & 3u;
      const uint32_t g = (0x1Eu >> (2 * code)) & 3u;  // LUT {2,3,1,0} packed as 0b00011110
      if (g != 3u) { s += g; c += 2; }
      out |= g << (2 * k);
    }
    G[idx] = (uint8_t)out;
  }
  atomicAdd(&sh[0], s);  // integer sums: exact, order-independent
  atomicAdd(&sh[1], c);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(&acc[0], sh[0]);
    atomicAdd(&acc[1], sh[1]);
  }
}

// 0<->2 swap of every field when sum/count >= 0.5 (snp_reader.pyx:254-303); padding fields
// of the last row stay 0.
__global__ void bed_flip_kernel(const unsigned long long* __restrict__ acc, int64_t M, int64_t N,
                                uint8_t* __restrict__ G, int* __restrict__ flipped) {
  const unsigned long long s = acc[0], c = acc[1];
  const bool flip = c != 0 && (double)s / (double)c >= 0.5;
  const int64_t rows = (M + 3) >> 2;
  const int64_t total = rows * N;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid == 0 && flipped) *flipped = flip ? 1 : 0;
  if (!flip) return;
  const int rem = (int)(M & 3);
  const uint32_t last_mask = rem ? ((1u << (2 * rem)) - 1u) : 0xFFu;
  for (int64_t idx = gid; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = G[idx];
    // per field: 0->2, 1->1, 2->0, 3->3  ==  v ^ (2 if v is 0 or 2)
    const uint32_t even = ~b & 0x55u;  // fields whose low bit is 0: values 0 and 2
    uint32_t out = b ^ (even << 1);
    if (idx / N == rows - 1) out &= last_mask;
    G[idx] = (uint8_t)out;
  }
}

}  // namespace adx

using namespace adx;

static unsigned grid_for(int64_t work, int threads) {
  const int64_t b = ceil_div(work, threads);
  const int64_t cap = (int64_t)sm_count() * 32;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

extern "C" int adx_unpack_u8(const uint8_t* G, int64_t rows, int64_t N, int64_t M_total,
                             int64_t m_start, int64_t count, int64_t byte_offset, uint8_t* out,
                             void* stream) {
  if (N <= 0 || M_total < 0 || m_start < 0 || count < 0 || byte_offset < 0 || !G || (!out && count)) {
    adx_set_message("adx_unpack_u8: bad arguments");
    return ADX_ERR_ARG;
  }
  count = count < M_total - m_start ? count : M_total - m_start;
  if (count <= 0) return ADX_OK;
  const int64_t last_row = ((m_start + count - 1) >> 2) - byte_offset;
  if (last_row >= rows) { adx_set_message("adx_unpack_u8: chunk beyond the packed rows given"); return ADX_ERR_ARG; }
  unpack_u8_kernel<<<grid_for(count * N, 256), 256, 0, as_stream(stream)>>>(G, N, M_total, m_start, count, byte_offset, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_unpack_center_f32(const uint8_t* G, int64_t rows, int64_t N, int64_t M_total,
                                     int64_t m_start, int64_t count, int64_t byte_offset,
                                     const float* f, float* out, void* stream) {
  if (N <= 0 || M_total < 0 || m_start < 0 || count < 0 || byte_offset < 0 || !G || !f || (!out && count)) {
    adx_set_message("adx_unpack_center_f32: bad arguments");
    return ADX_ERR_ARG;
  }
  count = count < M_total - m_start ? count : M_total - m_start;
  if (count <= 0) return ADX_OK;
  const int64_t last_row = ((m_start + count - 1) >> 2) - byte_offset;
  if (last_row >= rows) { adx_set_message("adx_unpack_center_f32: chunk beyond the packed rows given"); return ADX_ERR_ARG; }
  unpack_center_kernel<<<grid_for(count * N, 256), 256, 0, as_stream(stream)>>>(G, N, M_total, m_start, count, byte_offset, f, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_allele_frequency(const uint8_t* G, int64_t M, int64_t N, float* f, void* stream) {
  if (M <= 0 || N <= 0 || !G || !f) { adx_set_message("adx_allele_frequency: bad arguments"); return ADX_ERR_ARG; }
  const int64_t rows = (M + 3) >> 2;
  allele_freq_kernel<<<grid_for(rows * 32, 256), 256, 0, as_stream(stream)>>>(G, M, N, f);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_sample_counts(const uint8_t* G, int64_t M, int64_t N, double* q_bat, void* stream) {
  if (M <= 0 || N <= 0 || !G || !q_bat) { adx_set_message("adx_sample_counts: bad arguments"); return ADX_ERR_ARG; }
  const int64_t rows = (M + 3) >> 2;
  const int threads = 256;
  const int64_t xblocks = ceil_div(N, threads);
  int64_t parts = ceil_div((int64_t)sm_count() * 8, xblocks);
  parts = parts < 1 ? 1 : (parts > rows ? rows : parts);
  parts = parts > 65535 ? 65535 : parts;
  const int64_t rpp = ceil_div(rows, parts);
  parts = ceil_div(rows, rpp);
  cudaStream_t st = as_stream(stream);
  ADX_CUDA_TRY(cudaMemsetAsync(q_bat, 0, (size_t)N * sizeof(double), st));
  sample_counts_kernel<<<dim3((unsigned)xblocks, (unsigned)parts), threads, 0, st>>>(G, M, N, rpp, q_bat);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_sample_het_counts(const uint8_t* G, int64_t M, int64_t N, double* het, void* stream) {
  if (M <= 0 || N <= 0 || !G || !het) { adx_set_message("adx_sample_het_counts: bad arguments"); return ADX_ERR_ARG; }
  const int64_t rows = (M + 3) >> 2;
  const int threads = 256;
  const int64_t xblocks = ceil_div(N, threads);
  int64_t parts = ceil_div((int64_t)sm_count() * 8, xblocks);
  parts = parts < 1 ? 1 : (parts > rows ? rows : parts);
  parts = parts > 65535 ? 65535 : parts;
  const int64_t rpp = ceil_div(rows, parts);
  parts = ceil_div(rows, rpp);
  cudaStream_t st = as_stream(stream);
  ADX_CUDA_TRY(cudaMemsetAsync(het, 0, (size_t)N * sizeof(double), st));
  het_counts_kernel<<<dim3((unsigned)xblocks, (unsigned)parts), threads, 0, st>>>(G, M, N, rpp, het);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_simulate_packed(const uint32_t* Pq, const uint32_t* Qq, int64_t M, int64_t N,
                                   int K, uint64_t key1, uint64_t key2, uint32_t miss_q, uint8_t* G,
                                   void* stream) {
  if (M <= 0 || N <= 0 || K < 1 || K > ADX_MAX_K || !Pq || !Qq || !G) {
    adx_set_message("adx_simulate_packed: bad arguments");
    return ADX_ERR_ARG;
  }
  const int threads = 128;
  const int64_t rows = (M + 3) >> 2;
  const unsigned gx = (unsigned)ceil_div(N, threads);
  int64_t gy = ceil_div((int64_t)sm_count() * 16, gx);
  gy = gy < 1 ? 1 : (gy > rows ? rows : gy);
  gy = gy > 65535 ? 65535 : gy;
  const dim3 grid(gx, (unsigned)gy);
  cudaStream_t st = as_stream(stream);
#define SIM(KM) simulate_kernel<KM><<<grid, threads, 0, st>>>(Pq, Qq, M, N, K, key1, key2, miss_q, G)
  if (K <= 4) SIM(4);
  else if (K <= 8) SIM(8);
  else if (K <= 16) SIM(16);
  else if (K <= 32) SIM(32);
  else SIM(64);
#undef SIM
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_bed_workspace_bytes(int64_t M, int64_t N, size_t* bytes) {
  if (M <= 0 || N <= 0 || !bytes) { adx_set_message("adx_bed_workspace_bytes: bad arguments"); return ADX_ERR_ARG; }
  *bytes = 2 * sizeof(unsigned long long);
  return ADX_OK;
}

extern "C" int adx_bed_to_packed(const uint8_t* bed, int64_t M, int64_t N, uint8_t* G, int* flipped,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  if (M <= 0 || N <= 0 || !bed || !G || !workspace) { adx_set_message("adx_bed_to_packed: bad arguments"); return ADX_ERR_ARG; }
  if (workspace_bytes < 2 * sizeof(unsigned long long)) { adx_set_message("adx_bed_to_packed: workspace too small"); return ADX_ERR_WORKSPACE; }
  cudaStream_t st = as_stream(stream);
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(workspace);
  ADX_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), st));
  const int64_t total = ((M + 3) >> 2) * N;
  bed_decode_kernel<<<grid_for(total, 256), 256, 0, st>>>(bed, M, N, G, acc);
  ADX_LAUNCH_CHECK();
  bed_flip_kernel<<<grid_for(total, 256), 256, 0, st>>>(acc, M, N, G, flipped);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}
