// Gradient and Hessian passes of the original ADMIXTURE (BR-QN) algorithm in float64,
// straight from the packed genotypes:
//
//   Q side (per sample i):  Xtz_q[i] = sum_j a_ji P_j + b_ji (1 - P_j)
//                           XtX_q[i] = sum_j (a_ji / h_ji) P_j P_j' + (b_ji / (1-h_ji)) (1-P_j)(1-P_j)'
//   P side (per SNP j):     Xtz_p[j] = sum_i (a_ji - b_ji) Q_i
//                           XtX_p[j] = sum_i (a_ji / h_ji + b_ji / (1-h_ji)) Q_i Q_i'
//
// with h = clamp(P_j . Q_i, 1e-10, 1 - 1e-10), a = g / h, b = (2 - g) / (1 - h), missing
// entries skipped. adamixture/model/br_qn_gpu.py:67-214 (the reference materialises the
// coefficient matrices per 8192-SNP chunk and contracts them with einsum); the per-entry
// arithmetic follows adamixture/src/utils_c/cython/sqp.pyx:258-328.
//
// One kernel serves both sides: a CTA owns a tile of 32 "rows" (samples for Q, SNPs for
// P) and a block of up to 128 (k <= l) pairs of the symmetric K x K Hessian, and reduces
// over a range of the other axis in chunks of 32. Per chunk the CTA computes h and the
// coefficients of the 32 x 32 entries once into shared memory, then each thread (row r =
// lane, pair slot = warp) accumulates 16 pairs in registers. Ranges of the reduced axis
// are split across CTAs when the row tiles alone do not fill the GPU; their sums meet in
// float64 atomics on the zeroed outputs.
#include "common.cuh"

namespace adx {
namespace gh {

constexpr int TR = 32;       // rows per tile
constexpr int CJ = 32;       // reduced-axis entries per chunk
constexpr int SLOTS = 8;     // warps
constexpr int PER_T = 16;    // pairs per thread
constexpr int PAIRS = SLOTS * PER_T;  // pairs per CTA
constexpr int TPB = 32 * SLOTS;

struct Args {
  const uint8_t* G;
  const double* P;   // [M][K]
  const double* Q;   // [N][K]
  int64_t M, N;
  int K;
  double* XtX;       // [rows][K][K]
  double* Xtz;       // [rows][K]
  int n_pblk;        // pair blocks
  int n_split;       // splits of the reduced axis
  int64_t chunks_per_split;
};

template <bool QSIDE>
__global__ void __launch_bounds__(TPB) grad_hess_kernel(Args a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int K = a.K;
  double* own = reinterpret_cast<double*>(smem);          // [TR][K]  rows' factors
  double* fac = own + TR * K;                             // [CJ][K]  reduced-axis factors
  double* c1 = fac + CJ * K;                              // [CJ][TR] coefficient planes
  double* c2 = c1 + CJ * TR;
  double* d1 = c2 + CJ * TR;
  double* d2 = d1 + CJ * TR;
  uint8_t* pk = reinterpret_cast<uint8_t*>(d2 + CJ * TR); // pair table (k, l)
  uint8_t* pl = pk + PAIRS;

  const int tid = threadIdx.x, lane = tid & 31, slot = tid >> 5;
  const int64_t n_rows = QSIDE ? a.N : a.M;
  const int64_t n_red = QSIDE ? a.M : a.N;
  const double* ownF = QSIDE ? a.Q : a.P;
  const double* redF = QSIDE ? a.P : a.Q;

  int64_t b = blockIdx.x;
  const int pblk = (int)(b % a.n_pblk); b /= a.n_pblk;
  const int split = (int)(b % a.n_split); b /= a.n_split;
  const int64_t row0 = b * TR;
  const int n_pairs = K * (K + 1) / 2;

  // pair table: pairs pblk*PAIRS + t in row-major order of the upper triangle
  for (int t = tid; t < PAIRS; t += TPB) {
    int p = pblk * PAIRS + t, k = 0;
    if (p < n_pairs) {
      while (p >= K - k) { p -= K - k; ++k; }
      pk[t] = (uint8_t)k;
      pl[t] = (uint8_t)(k + p);
    } else {
      pk[t] = 0xFF;
      pl[t] = 0xFF;
    }
  }
  for (int e = tid; e < TR * K; e += TPB) {
    const int r = e / K, k = e - r * K;
    const int64_t row = row0 + r;
    own[e] = row < n_rows ? ownF[row * K + k] : 0.0;
  }

  double acc[PER_T], xz[8];
#pragma unroll
  for (int q = 0; q < PER_T; ++q) acc[q] = 0.0;
#pragma unroll
  for (int m = 0; m < 8; ++m) xz[m] = 0.0;

  const int64_t n_chunks = (n_red + CJ - 1) / CJ;
  const int64_t ch0 = (int64_t)split * a.chunks_per_split;
  const int64_t ch1 = min(n_chunks, ch0 + a.chunks_per_split);
  for (int64_t ch = ch0; ch < ch1; ++ch) {
    const int64_t red0 = ch * CJ;
    __syncthreads();  // previous chunk's readers are done
    for (int e = tid; e < CJ * K; e += TPB) {
      const int c = e / K, k = e - c * K;
      const int64_t j = red0 + c;
      fac[e] = j < n_red ? redF[j * K + k] : 0.0;
    }
    __syncthreads();
    // coefficients of the TR x CJ entries; lanes walk the sample axis of G
    for (int e = tid; e < TR * CJ; e += TPB) {
      int r, c;
      if (QSIDE) { c = e / TR; r = e - c * TR; } else { r = e / CJ; c = e - r * CJ; }
      const int64_t row = row0 + r, red = red0 + c;
      double v1 = 0.0, v2 = 0.0, w1 = 0.0, w2 = 0.0;
      if (row < n_rows && red < n_red) {
        const int64_t snp = QSIDE ? red : row, smp = QSIDE ? row : red;
        const unsigned g = genotype(a.G[(snp >> 2) * a.N + smp], (int)(snp & 3));
        if (g != 3u) {
          double h = 0.0;
          for (int k = 0; k < K; ++k) h += own[r * K + k] * fac[c * K + k];
          h = fmax(fmin(h, 1.0 - 1e-10), 1e-10);
          const double gd = (double)g;
          v1 = gd / h;
          v2 = (2.0 - gd) / (1.0 - h);
          w1 = v1 / h;
          w2 = v2 / (1.0 - h);
        }
      }
      c1[c * TR + r] = v1;
      c2[c * TR + r] = v2;
      d1[c * TR + r] = w1;
      d2[c * TR + r] = w2;
    }
    __syncthreads();
    const int cmax = (int)min((int64_t)CJ, n_red - red0);
    for (int c = 0; c < cmax; ++c) {
      const double* f = fac + c * K;
      const double e1 = d1[c * TR + lane], e2 = d2[c * TR + lane];
#pragma unroll
      for (int q = 0; q < PER_T; ++q) {
        const int t = slot + SLOTS * q;
        const int k = pk[t];
        if (k == 0xFF) continue;
        const int l = pl[t];
        if (QSIDE) {
          acc[q] += e1 * f[k] * f[l] + e2 * (1.0 - f[k]) * (1.0 - f[l]);
        } else {
          acc[q] += (e1 + e2) * f[k] * f[l];
        }
      }
      if (pblk == 0) {
        const double z1 = c1[c * TR + lane], z2 = c2[c * TR + lane];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const int k = slot + SLOTS * m;
          if (k < K) xz[m] += QSIDE ? (z1 * f[k] + z2 * (1.0 - f[k])) : ((z1 - z2) * f[k]);
        }
      }
    }
  }

  const int64_t row = row0 + lane;
  if (row >= n_rows) return;
  double* H = a.XtX + row * K * K;
#pragma unroll
  for (int q = 0; q < PER_T; ++q) {
    const int t = slot + SLOTS * q;
    const int k = pk[t];
    if (k == 0xFF) continue;
    const int l = pl[t];
    atomicAdd(H + k * K + l, acc[q]);
    if (l != k) atomicAdd(H + l * K + k, acc[q]);
  }
  if (pblk == 0) {
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int k = slot + SLOTS * m;
      if (k < K) atomicAdd(a.Xtz + row * K + k, xz[m]);
    }
  }
}

}  // namespace gh
}  // namespace adx

using namespace adx;

template <bool QSIDE>
static int grad_hess(const uint8_t* G, int64_t M, int64_t N, int K, const double* P, const double* Q,
                     double* XtX, double* Xtz, void* stream, const char* name) {
  if (!G || !P || !Q || !XtX || !Xtz || M <= 0 || N <= 0 || K < 1 || K > ADX_MAX_K) {
    adx_set_message(name);
    return ADX_ERR_ARG;
  }
  cudaStream_t st = as_stream(stream);
  const int64_t n_rows = QSIDE ? N : M, n_red = QSIDE ? M : N;
  ADX_CUDA_TRY(cudaMemsetAsync(XtX, 0, (size_t)n_rows * K * K * sizeof(double), st));
  ADX_CUDA_TRY(cudaMemsetAsync(Xtz, 0, (size_t)n_rows * K * sizeof(double), st));
  gh::Args a{G, P, Q, M, N, K, XtX, Xtz, 0, 0, 0};
  const int n_pairs = K * (K + 1) / 2;
  a.n_pblk = (n_pairs + gh::PAIRS - 1) / gh::PAIRS;
  const int64_t tiles = ceil_div(n_rows, gh::TR);
  const int64_t n_chunks = ceil_div(n_red, gh::CJ);
  // about 8 CTAs per SM in all
  int64_t split = ceil_div((int64_t)sm_count() * 8, tiles * a.n_pblk);
  split = split < 1 ? 1 : (split > n_chunks ? n_chunks : split);
  a.chunks_per_split = ceil_div(n_chunks, split);
  a.n_split = (int)ceil_div(n_chunks, a.chunks_per_split);
  const size_t smem = (size_t)(gh::TR + gh::CJ) * K * sizeof(double) + 4 * gh::CJ * gh::TR * sizeof(double) +
                      2 * gh::PAIRS;
  ADX_CUDA_TRY(cudaFuncSetAttribute(gh::grad_hess_kernel<QSIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t blocks = tiles * a.n_pblk * a.n_split;
  gh::grad_hess_kernel<QSIDE><<<(unsigned)blocks, gh::TPB, smem, st>>>(a);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_grad_hess_q(const uint8_t* G, int64_t M, int64_t N, int K, const double* P, const double* Q,
                               double* XtX_q, double* Xtz_q, void* stream) {
  return grad_hess<true>(G, M, N, K, P, Q, XtX_q, Xtz_q, stream, "adx_grad_hess_q: bad argument");
}

extern "C" int adx_grad_hess_p(const uint8_t* G, int64_t M, int64_t N, int K, const double* P, const double* Q,
                               double* XtX_p, double* Xtz_p, void* stream) {
  return grad_hess<false>(G, M, N, K, P, Q, XtX_p, Xtz_p, stream, "adx_grad_hess_p: bad argument");
}
