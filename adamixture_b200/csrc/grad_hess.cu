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
// Each pass is a GEMM with a fused prologue. The Hessian of a row (sample for Q, SNP for P)
// is a weighted sum over the other axis of per-entry pair products -- P_jk P_jl (and the
// complement's) for the Q side, Q_ik Q_il for the P side -- and those products do not depend
// on the row. A CTA owns 64 rows and 64 (k <= l) pairs of the symmetric K x K Hessian and
// walks a range of the other axis in chunks of 32: per chunk it stages the factor rows,
// forms the 32 x 64 pair products and the 64 x 32 coefficients (h, then a/h and b/(1-h))
// once in shared memory, and the product runs on the float64 tensor-core MMA
// (mma.sync m16n8k4 .f64: 512 FMAs per warp instruction, operands from registers): each
// warp owns 32 rows x 16 pairs as 2 x 2 MMA tiles, loading its fragments from shared
// memory whose rows are padded by 4 doubles so a fragment load is conflict-free. Every
// chunk enters the MMAs whole: entries past the reduced axis have zero coefficients. The
// gradient rides along in the CTAs of the first pair
// block. Ranges of the reduced axis are split across CTAs when the row tiles alone do not
// fill the GPU; their sums meet in float64 atomics on the zeroed outputs.
#include "common.cuh"

namespace adx {
namespace gh {

constexpr int TR = 64;       // rows per tile
constexpr int TP = 64;       // pairs per tile
constexpr int CJ = 32;       // reduced-axis entries per chunk
constexpr int TPB = 256;     // 8 warps: 2 row blocks of 32 x 4 pair blocks of 16
constexpr int CSTR = TR + 4; // padded row stride of the coefficient tiles (doubles)
constexpr int PSTR = TP + 4; // padded row stride of the pair-product tiles (doubles)

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

// d (4 doubles: rows g, g, g+8, g+8; columns 2t, 2t+1, 2t, 2t+1 of a 16 x 8 tile) +=
// A (16 x 4: a0 row g, a1 row g+8, column t) . B (4 x 8: b0 row t, column g), float64
// tensor-core MMA; g = lane / 4, t = lane % 4.
__device__ __forceinline__ void mma_f64(double (&d)[4], double a0, double a1, double b0) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a0), "d"(a1), "d"(b0));
}

// shared-memory layout (doubles unless noted)
struct Smem {
  double *own, *fac, *coef, *zc, *pp;
  uint8_t *pk, *pl;
  static __host__ size_t bytes(int K, int nt) {
    return sizeof(double) * ((size_t)(TR + CJ) * K + (size_t)nt * CJ * 2 * CSTR + (size_t)nt * CJ * PSTR) + 2 * TP;
  }
  __device__ Smem(uint8_t* base, int K, int nt) {
    double* d = reinterpret_cast<double*>(base);
    own = d; d += TR * K;            // [TR][K] factors of the tile's rows
    fac = d; d += CJ * K;            // [CJ][K] factors of the chunk's reduced entries
    coef = d; d += nt * CJ * CSTR;   // [nt][CJ][CSTR] Hessian coefficients
    zc = d; d += nt * CJ * CSTR;     // [nt][CJ][CSTR] gradient coefficients
    pp = d; d += nt * CJ * PSTR;     // [nt][CJ][PSTR] pair products
    pk = reinterpret_cast<uint8_t*>(d);
    pl = pk + TP;
  }
};

// KM: an upper bound of K known at compile time (4, 6, 8, 10, 12, 16, or 64 for the rest),
// which sizes the gradient's MMA tiles (64 rows x ceil(KM / 8) column tiles of 8, spread
// over the 8 warps) and, for KM <= 16, the factor row kept in registers.
template <bool QSIDE, int KM>
__global__ void __launch_bounds__(TPB) grad_hess_kernel(Args a) {
  constexpr int NTG = (KM + 7) / 8;          // gradient column tiles
  constexpr int GT = (4 * NTG + 7) / 8;      // gradient tiles per warp
  constexpr int NT = QSIDE ? 2 : 1;   // coefficient terms
  extern __shared__ __align__(16) uint8_t smem[];
  const int K = a.K;
  Smem s(smem, K, NT);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int fg = lane >> 2, ft = lane & 3;   // MMA fragment group and thread in group
  const int wr = warp & 1, wp = warp >> 1;   // the warp's row block (32) and pair block (16)
  const int64_t n_rows = QSIDE ? a.N : a.M;
  const int64_t n_red = QSIDE ? a.M : a.N;
  const double* ownF = QSIDE ? a.Q : a.P;
  const double* redF = QSIDE ? a.P : a.Q;

  int64_t b = blockIdx.x;
  const int pblk = (int)(b % a.n_pblk); b /= a.n_pblk;
  const int split = (int)(b % a.n_split); b /= a.n_split;
  const int64_t row0 = b * TR;
  const int n_pairs = K * (K + 1) / 2;
  const bool do_grad = pblk == 0;

  // pair table: pairs pblk*TP + t in row-major order of the upper triangle
  for (int t = tid; t < TP; t += TPB) {
    int p = pblk * TP + t, k = 0;
    if (p < n_pairs) {
      while (p >= K - k) { p -= K - k; ++k; }
      s.pk[t] = (uint8_t)k;
      s.pl[t] = (uint8_t)(k + p);
    } else {
      s.pk[t] = 0xFF;
      s.pl[t] = 0xFF;
    }
  }
  for (int e = tid; e < TR * K; e += TPB) {
    const int r = e / K, k = e - r * K;
    const int64_t row = row0 + r;
    s.own[e] = row < n_rows ? ownF[row * K + k] : 0.0;
  }

  double acc[2][2][4];   // [row tile][pair tile][fragment]
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
  // gradient: 4 row tiles x NTG column tiles of 16 x 8; warp w owns tiles w, w + 8, ...
  double gacc[GT][4];
#pragma unroll
  for (int q = 0; q < GT; ++q)
#pragma unroll
    for (int v = 0; v < 4; ++v) gacc[q][v] = 0.0;

  const int64_t n_chunks = (n_red + CJ - 1) / CJ;
  const int64_t ch0 = (int64_t)split * a.chunks_per_split;
  const int64_t ch1 = min(n_chunks, ch0 + a.chunks_per_split);
  for (int64_t ch = ch0; ch < ch1; ++ch) {
    const int64_t red0 = ch * CJ;
    __syncthreads();  // the previous chunk's readers are done
    {
      // the chunk's factor rows are contiguous: a flat copy, zeros past the reduced axis
      const int64_t base = red0 * K, end = n_red * K;
      for (int e = tid; e < CJ * K; e += TPB) s.fac[e] = base + e < end ? redF[base + e] : 0.0;
    }
    __syncthreads();
    // pair products of the chunk's entries (shared by every row); TPB is a multiple of
    // TP, so a thread's entries all have pair t = tid % TP
    {
      static_assert(TPB % TP == 0, "one pair per thread");
      const int t = tid & (TP - 1);
      const int k = s.pk[t], l = s.pl[t];
      for (int c = tid / TP; c < CJ; c += TPB / TP) {
        double v0 = 0.0, v1 = 0.0;
        if (k != 0xFF) {
          const double fk = s.fac[c * K + k], fl = s.fac[c * K + l];
          v0 = fk * fl;
          if (QSIDE) v1 = (1.0 - fk) * (1.0 - fl);
        }
        s.pp[c * PSTR + t] = v0;
        if (QSIDE) s.pp[CJ * PSTR + c * PSTR + t] = v1;
      }
    }
    // coefficients of the TR x CJ entries; lanes walk the sample axis of G. A thread's
    // entries share one factor row -- its row (tid & 63) on the Q side, its reduced entry
    // (tid & 31) on the P side -- held in registers for K <= 16
    double fix[KM <= 16 ? KM : 1];
    if constexpr (KM <= 16) {
      const double* src = QSIDE ? s.own + (tid & (TR - 1)) * K : s.fac + (tid & (CJ - 1)) * K;
#pragma unroll
      for (int k = 0; k < KM; ++k) fix[k] = k < K ? src[k] : 0.0;
    }
    // A thread's 8 entries run along the SNP axis -- Q side: chunk entries 8 (tid >> 6) + n
    // of row tid & 63; P side: rows 8 (tid >> 5) + n of chunk entry tid & 31 -- so they come
    // from two packed genotype bytes (SNPs snp0 .. snp0 + 7 of one sample).
    const int fixed = QSIDE ? (tid & (TR - 1)) : (tid & (CJ - 1));
    const int first = QSIDE ? 8 * (tid >> 6) : 8 * (tid >> 5);
    const int64_t smp = (QSIDE ? row0 : red0) + fixed;
    const int64_t snp0 = (QSIDE ? red0 : row0) + first;   // a multiple of 8
    uint32_t gbytes = 0xFFFFu;                              // all missing outside the matrix
    if (smp < a.N) {
      if (snp0 < a.M) gbytes = (gbytes & 0xFF00u) | (uint32_t)a.G[(snp0 >> 2) * a.N + smp];
      if (snp0 + 4 < a.M) gbytes = (gbytes & 0x00FFu) | ((uint32_t)a.G[((snp0 >> 2) + 1) * a.N + smp] << 8);
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const int r = QSIDE ? fixed : first + n;
      const int c = QSIDE ? first + n : fixed;
      const int64_t row = row0 + r, red = red0 + c;
      double w1 = 0.0, w2 = 0.0, z1 = 0.0, z2 = 0.0;
      if (row < n_rows && red < n_red) {
        const unsigned g = (gbytes >> (2 * n)) & 3u;   // SNP snp0 + n
        if (g != 3u) {
          double h = 0.0;
          if constexpr (KM <= 16) {
            const double* var = QSIDE ? s.fac + c * K : s.own + r * K;
            if (KM % 2 == 0 && K == KM) {
              // K even: the row starts 16-byte aligned, read it two doubles at a time
#pragma unroll
              for (int k = 0; k < KM; k += 2) {
                const double2 v2 = *reinterpret_cast<const double2*>(var + k);
                h += QSIDE ? fix[k] * v2.x : v2.x * fix[k];
                h += QSIDE ? fix[k + 1] * v2.y : v2.y * fix[k + 1];
              }
            } else {
#pragma unroll
              for (int k = 0; k < KM; ++k)
                if (k < K) h += QSIDE ? fix[k] * var[k] : var[k] * fix[k];
            }
          } else {
            for (int k = 0; k < K; ++k) h += s.own[r * K + k] * s.fac[c * K + k];
          }
          h = fmax(fmin(h, 1.0 - 1e-10), 1e-10);
          const double gd = (double)g, om = 1.0 - h;
          // 1/h and 1/(1-h) from one reciprocal of x = h(1-h) in [1e-10, 0.25]: the hardware
          // approximation refined by two Newton-Raphson steps r <- r (2 - x r), each of which
          // squares the relative error (within a unit or two of the last place after both)
          const double x = h * om;
          double rr;
          asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(rr) : "d"(x));
          rr = fma(rr, fma(-x, rr, 1.0), rr);
          rr = fma(rr, fma(-x, rr, 1.0), rr);
          const double ih = om * rr, iom = h * rr;
          z1 = gd * ih;
          z2 = (2.0 - gd) * iom;
          w1 = z1 * ih;
          w2 = z2 * iom;
        }
      }
      if (QSIDE) {
        s.coef[c * CSTR + r] = w1;
        s.coef[CJ * CSTR + c * CSTR + r] = w2;
        s.zc[c * CSTR + r] = z1;
        s.zc[CJ * CSTR + c * CSTR + r] = z2;
      } else {
        s.coef[c * CSTR + r] = w1 + w2;
        s.zc[c * CSTR + r] = z1 - z2;
      }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      // A (rows x chunk entries) = coef^T, B (chunk entries x pairs) = pp: fragment
      // element (row fg [+8], entry ft) of A, (entry ft, pair fg) of B
      const double* cf = s.coef + t * CJ * CSTR + wr * 32 + fg;
      const double* pr = s.pp + t * CJ * PSTR + wp * 16 + fg;
#pragma unroll
      for (int c0 = 0; c0 < CJ; c0 += 4) {
        const double* ca = cf + (c0 + ft) * CSTR;
        const double* pb = pr + (c0 + ft) * PSTR;
        const double a00 = ca[0], a01 = ca[8], a10 = ca[16], a11 = ca[24];
        const double b0 = pb[0], b1 = pb[8];
        mma_f64(acc[0][0], a00, a01, b0);
        mma_f64(acc[0][1], a00, a01, b1);
        mma_f64(acc[1][0], a10, a11, b0);
        mma_f64(acc[1][1], a10, a11, b1);
      }
    }
    if (do_grad) {
      // Xtz += z1' fac (+ z2' (1 - fac) on the Q side): A = z (rows x chunk entries),
      // B = the chunk's factor rows, columns k >= K fed zeros
#pragma unroll
      for (int q = 0; q < GT; ++q) {
        const int tix = warp + 8 * q;
        if (tix >= 4 * NTG) break;   // warp-uniform
        const int mt = tix & 3, k = (tix >> 2) * 8 + fg;
        const bool kin = k < K;
        const double* z = s.zc + mt * 16 + fg;
#pragma unroll
        for (int c0 = 0; c0 < CJ; c0 += 4) {
          const int c = c0 + ft;
          const double f = kin ? s.fac[c * K + k] : 0.0;
          mma_f64(gacc[q], z[c * CSTR], z[c * CSTR + 8], f);
          if (QSIDE) mma_f64(gacc[q], z[(CJ + c) * CSTR], z[(CJ + c) * CSTR + 8], kin ? 1.0 - f : 0.0);
        }
      }
    }
  }

  // scatter: both halves of the symmetric Hessian; accumulator v of tile (i, j) is row
  // fg (+8 for v >= 2), pair 2 ft + (v & 1) of the tile
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int64_t row = row0 + wr * 32 + i * 16 + fg + (v >> 1) * 8;
      if (row >= n_rows) continue;
      double* H = a.XtX + row * K * K;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int t = wp * 16 + j * 8 + 2 * ft + (v & 1);
        const int k = s.pk[t];
        if (k == 0xFF) continue;
        const int l = s.pl[t];
        atomicAdd(H + k * K + l, acc[i][j][v]);
        if (l != k) atomicAdd(H + l * K + k, acc[i][j][v]);
      }
    }
  if (do_grad) {
#pragma unroll
    for (int q = 0; q < GT; ++q) {
      const int tix = warp + 8 * q;
      if (tix >= 4 * NTG) break;
      const int mt = tix & 3, nt = tix >> 2;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int64_t row = row0 + mt * 16 + fg + (v >> 1) * 8;
        const int k = nt * 8 + 2 * ft + (v & 1);
        if (row < n_rows && k < K) atomicAdd(a.Xtz + row * K + k, gacc[q][v]);
      }
    }
  }
}

}  // namespace gh
}  // namespace adx

using namespace adx;

template <bool QSIDE, int KM>
static int grad_hess_launch(const gh::Args& a, size_t smem, int64_t blocks, cudaStream_t st) {
  ADX_CUDA_TRY(cudaFuncSetAttribute(gh::grad_hess_kernel<QSIDE, KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gh::grad_hess_kernel<QSIDE, KM><<<(unsigned)blocks, gh::TPB, smem, st>>>(a);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

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
  a.n_pblk = (n_pairs + gh::TP - 1) / gh::TP;
  const int64_t tiles = ceil_div(n_rows, gh::TR);
  const int64_t n_chunks = ceil_div(n_red, gh::CJ);
  // about 8 CTAs per SM in all
  int64_t split = ceil_div((int64_t)sm_count() * 8, tiles * a.n_pblk);
  split = split < 1 ? 1 : (split > n_chunks ? n_chunks : split);
  a.chunks_per_split = ceil_div(n_chunks, split);
  a.n_split = (int)ceil_div(n_chunks, a.chunks_per_split);
  const size_t smem = gh::Smem::bytes(K, QSIDE ? 2 : 1);
  const int64_t blocks = tiles * a.n_pblk * a.n_split;
  if (K <= 4) return grad_hess_launch<QSIDE, 4>(a, smem, blocks, st);
  if (K <= 6) return grad_hess_launch<QSIDE, 6>(a, smem, blocks, st);
  if (K <= 8) return grad_hess_launch<QSIDE, 8>(a, smem, blocks, st);
  if (K <= 10) return grad_hess_launch<QSIDE, 10>(a, smem, blocks, st);
  if (K <= 12) return grad_hess_launch<QSIDE, 12>(a, smem, blocks, st);
  if (K <= 16) return grad_hess_launch<QSIDE, 16>(a, smem, blocks, st);
  return grad_hess_launch<QSIDE, 64>(a, smem, blocks, st);
}

extern "C" int adx_grad_hess_q(const uint8_t* G, int64_t M, int64_t N, int K, const double* P, const double* Q,
                               double* XtX_q, double* Xtz_q, void* stream) {
  return grad_hess<true>(G, M, N, K, P, Q, XtX_q, Xtz_q, stream, "adx_grad_hess_q: bad argument");
}

extern "C" int adx_grad_hess_p(const uint8_t* G, int64_t M, int64_t N, int K, const double* P, const double* Q,
                               double* XtX_p, double* Xtz_p, void* stream) {
  return grad_hess<false>(G, M, N, K, P, Q, XtX_p, Xtz_p, stream, "adx_grad_hess_p: bad argument");
}
