// Batched per-row K x K solvers in float64, one warp per row:
//
// * bounded least squares by block principal pivoting (the ALS initialisation's P and Q
//   updates), adamixture/src/utils_c/cuda/bvls_kernel.cu:11-164 (its unconstrained start
//   solved by the same elimination, as adamixture/src/utils_c/cython/bvls.pyx:130-227 does);
// * the SQP step of the original ADMIXTURE algorithm: the sweep-operator active-set QP on
//   the (K+2)-square simplex tableau of a Q row or the (K+1)-square box tableau of a P row,
//   then the simplex / box projection with pseudocount 1e-5,
//   adamixture/src/utils_c/cuda/sqp_kernel.cu:6-311.
//
// A row's working set (augmented system or tableau, vectors, flags) lives in the warp's
// slice of shared memory; the lanes split every inner loop (rows of an elimination step,
// columns of a sweep), so each element sees the same operations in the same order as the
// one-thread-per-row reference, and the control decisions (pivot row, active set, step
// length) are warp-uniform.
#include "common.cuh"

namespace adx {
namespace solve {

constexpr double SINGULAR_TOL = 1e-12;
constexpr double PIVOT_TOL = 1e-8;
constexpr int BPP_MAX_ITER = 50;
constexpr int QP_MAX_ITER = 1000;

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------- BVLS

// Per-warp scratch of a BVLS row (KM >= K).
template <int KM>
struct BvlsScratch {
  double aug[KM * (KM + 1)];
  double x[KM], b[KM], bs[KM];
  int F[KM], U[KM], map[KM];
};

// Gauss-Jordan elimination with partial pivoting on the free subset (F[i] == 1) of
// A x = bs; writes x[map[i]] for the free variables. Returns false (x untouched) when a
// pivot falls below SINGULAR_TOL. bvls_kernel.cu:11-72.
template <int KM>
__device__ bool solve_subset(const double* A, int K, BvlsScratch<KM>& s, int lane) {
  // free indices in increasing order
  int n = 0;
  for (int base = 0; base < K; base += 32) {
    const int i = base + lane;
    const bool f = i < K && s.F[i] == 1;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (f) s.map[n + __popc(m & ((1u << lane) - 1u))] = i;
    n += __popc(m);
  }
  __syncwarp();
  if (n == 0) return true;
  const int w = n + 1;
  for (int e = lane; e < n * w; e += 32) {
    const int i = e / w, j = e - i * w;
    s.aug[e] = j < n ? A[s.map[i] * K + s.map[j]] : s.bs[s.map[i]];
  }
  __syncwarp();
  for (int i = 0; i < n; ++i) {
    // pivot: the first row of maximal |aug[k][i]|, k >= i
    double best = -1.0;
    int brow = n;
    for (int k = i + lane; k < n; k += 32) {
      const double v = fabs(s.aug[k * w + i]);
      if (v > best) { best = v; brow = k; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, o);
      const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
      if (ov > best || (ov == best && orow < brow)) { best = ov; brow = orow; }
    }
    if (best < SINGULAR_TOL) return false;
    if (brow != i) {
      for (int j = i + lane; j <= n; j += 32) {
        const double t = s.aug[i * w + j];
        s.aug[i * w + j] = s.aug[brow * w + j];
        s.aug[brow * w + j] = t;
      }
      __syncwarp();
    }
    const double pivot = s.aug[i * w + i];
    __syncwarp();
    for (int j = i + lane; j <= n; j += 32) s.aug[i * w + j] /= pivot;
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
      if (k == i) continue;
      const double t = s.aug[k * w + i];
      for (int j = i; j <= n; ++j) s.aug[k * w + j] -= t * s.aug[i * w + j];
    }
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) s.x[s.map[i]] = s.aug[i * w + n];
  __syncwarp();
  return true;
}

// One warp per row of B: X[row] = argmin over lower <= x <= upper of 1/2 x'Ax - b'x by
// block principal pivoting from the unconstrained solution. bvls_kernel.cu:75-164.
template <int KM>
__global__ void bvls_kernel(const double* __restrict__ A, const double* __restrict__ B, int64_t M, int K,
                            double lower, double upper, double* __restrict__ X, int wpb) {
  extern __shared__ __align__(16) uint8_t smem[];
  double* As = reinterpret_cast<double*>(smem);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BvlsScratch<KM>& s = reinterpret_cast<BvlsScratch<KM>*>(smem + ((size_t)KM * KM * sizeof(double)))[warp];
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) As[e] = A[e];
  __syncthreads();
  for (int64_t row = (int64_t)blockIdx.x * wpb + warp; row < M; row += (int64_t)gridDim.x * wpb) {
    const double* b = B + row * K;
    for (int i = lane; i < K; i += 32) {
      s.b[i] = b[i];
      s.bs[i] = b[i];
      s.F[i] = 1;
      s.U[i] = 0;
      s.x[i] = 0.0;
    }
    __syncwarp();
    if (solve_subset<KM>(As, K, s, lane)) {
      bool changed = false;
      for (int i = lane; i < K; i += 32) {
        if (s.x[i] < lower - PIVOT_TOL) { s.F[i] = 0; s.U[i] = 0; changed = true; }
        else if (s.x[i] > upper + PIVOT_TOL) { s.F[i] = 0; s.U[i] = 1; changed = true; }
      }
      changed = __any_sync(0xffffffffu, changed);
      __syncwarp();
      for (int it = 1; changed && it < BPP_MAX_ITER; ++it) {
        for (int i = lane; i < K; i += 32) {
          if (s.F[i] == 1) {
            double v = s.b[i];
            for (int j = 0; j < K; ++j)
              if (s.F[j] == 0) v -= As[i * K + j] * (s.U[j] == 1 ? upper : lower);
            s.bs[i] = v;
          }
        }
        __syncwarp();
        if (!solve_subset<KM>(As, K, s, lane)) break;
        for (int i = lane; i < K; i += 32)
          if (s.F[i] == 0) s.x[i] = s.U[i] == 1 ? upper : lower;
        __syncwarp();
        bool ch = false;
        for (int i = lane; i < K; i += 32) {
          double y = -s.b[i];
          for (int j = 0; j < K; ++j) y += As[i * K + j] * s.x[j];
          if (s.F[i] == 1) {
            if (s.x[i] < lower - PIVOT_TOL) { s.F[i] = 0; s.U[i] = 0; ch = true; }
            else if (s.x[i] > upper + PIVOT_TOL) { s.F[i] = 0; s.U[i] = 1; ch = true; }
          } else if (s.U[i] == 0 && y < -PIVOT_TOL) {
            s.F[i] = 1; s.U[i] = 0; ch = true;
          } else if (s.U[i] == 1 && y > PIVOT_TOL) {
            s.F[i] = 1; s.U[i] = 0; ch = true;
          }
        }
        changed = __any_sync(0xffffffffu, ch);
        __syncwarp();
      }
    }
    for (int i = lane; i < K; i += 32) X[row * K + i] = s.x[i];
    __syncwarp();
  }
}

// ---------------------------------------------------------------- SQP

template <int KM>
struct SqpScratch {
  double tab[(KM + 2) * (KM + 2)];
  double tmp[KM + 2];
  double delta[KM], par[KM], out[KM];
  int swept[KM];
};

// Sweep operator on pivot k of the sz x sz tableau. sqp_kernel.cu:6-26.
template <int KM>
__device__ void sweep(SqpScratch<KM>& s, int sz, int k, bool inverse, int lane) {
  const double piv = s.tab[k * sz + k];
  if (piv == 0.0) return;
  const double p = 1.0 / piv;
  for (int i = lane; i < sz; i += 32) s.tmp[i] = s.tab[i * sz + k];
  __syncwarp();
  for (int i = lane; i < sz; i += 32) {
    s.tab[i * sz + k] = 0.0;
    s.tab[k * sz + i] = 0.0;
  }
  if (lane == 0) s.tmp[k] = inverse ? 1.0 : -1.0;
  __syncwarp();
  for (int i = 0; i < sz; ++i) {
    const double pv = p * s.tmp[i];
    for (int j = lane; j < sz; j += 32) s.tab[j * sz + i] -= pv * s.tmp[j];
  }
  __syncwarp();
}

// Active-set QP on the swept tableau: p parameters, c equality constraints. Returns the
// iteration count, or 0 when it gives up (delta stays as far as it got). sqp_kernel.cu:28-123.
template <int KM>
__device__ int quadratic_program(SqpScratch<KM>& s, int p, int c, int lane) {
  const int sz = p + c + 1;
  const double small = 1e-5, tol = 1e-8;
  for (int i = lane; i < p; i += 32) s.delta[i] = 0.0;
  __syncwarp();
  // s.out holds the diagonal as it was before any sweep (d in the reference); each pivot
  // is checked against it while earlier sweeps change the current diagonal
  for (int i = 0; i < p; ++i) {
    const double d = s.out[i];
    if (d <= 0.0 || s.tab[i * sz + i] < d * tol) return 0;
    sweep<KM>(s, sz, i, false, lane);
  }
  for (int i = lane; i < p; i += 32) s.swept[i] = 1;
  __syncwarp();
  for (int i = p; i < p + c; ++i) {
    if (s.tab[i * sz + i] >= 0.0) return 0;
    sweep<KM>(s, sz, i, false, lane);
  }
  for (int iteration = 1; iteration <= QP_MAX_ITER; ++iteration) {
    double a = 1.0;
    for (int i = lane; i < p; i += 32) {
      if (s.swept[i]) {
        const double ui = s.tab[i * sz + (sz - 1)];
        const double ai = (ui > 0.0 ? 1.0 : 0.0) - s.par[i] - s.delta[i];
        if (fabs(ui) > 1e-10) a = fmin(a, ai / ui);
      }
    }
    a = warp_min(a);
    for (int i = lane; i < p; i += 32) {
      if (s.swept[i]) {
        const double ui = s.tab[i * sz + (sz - 1)];
        s.delta[i] = s.delta[i] + a * ui;
        const double nu = (1.0 - a) * ui;
        s.tab[i * sz + (sz - 1)] = nu;
        s.tab[(sz - 1) * sz + i] = nu;
      }
    }
    __syncwarp();
    // the first swept parameter that reached a bound leaves the model
    int pick = p;
    for (int base = 0; base < p && pick == p; base += 32) {
      const int i = base + lane;
      bool hit = false;
      if (i < p) {
        const double v = s.par[i] + s.delta[i];
        const bool critical = (0.0 >= v - small) || (1.0 <= v + small);
        hit = s.swept[i] && fabs(s.tab[i * sz + i]) > 1e-10 && critical;
      }
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (m) pick = base + __ffs(m) - 1;
    }
    if (pick < p) {
      sweep<KM>(s, sz, pick, true, lane);
      if (lane == 0) s.swept[pick] = 0;
      __syncwarp();
      continue;
    }
    // the first unswept parameter whose multiplier points into the interior re-enters
    for (int base = 0; base < p && pick == p; base += 32) {
      const int i = base + lane;
      bool hit = false;
      if (i < p) {
        const double ui = s.tab[i * sz + (sz - 1)];
        const double v = s.par[i] + s.delta[i];
        const bool violation = (ui > 0.0 && 0.0 >= v - small) || (ui < 0.0 && 1.0 <= v + small);
        hit = !s.swept[i] && violation;
      }
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (m) pick = base + __ffs(m) - 1;
    }
    if (pick < p) {
      sweep<KM>(s, sz, pick, false, lane);
      if (lane == 0) s.swept[pick] = 1;
      __syncwarp();
      continue;
    }
    return iteration;
  }
  return 0;
}

// Projection of a Q row onto {x >= pc, sum x = 1}. sqp_kernel.cu:125-166 (lane 0).
__device__ void project_simplex_row(double* b, int n, double pc) {
  const double tau = 1.0 - n * pc;
  int idx[ADX_MAX_K];
  for (int i = 0; i < n; ++i) {
    b[i] -= pc;
    idx[i] = i;
  }
  for (int i = 1; i < n; ++i) {
    const int key = idx[i];
    const double kv = b[key];
    int j = i - 1;
    while (j >= 0 && b[idx[j]] < kv) {
      idx[j + 1] = idx[j];
      --j;
    }
    idx[j + 1] = key;
  }
  double tsum = 0.0, tmax = 0.0;
  bool bget = false;
  for (int i = 0; i < n - 1; ++i) {
    tsum += b[idx[i]];
    tmax = (tsum - tau) / (i + 1);
    if (tmax >= b[idx[i + 1]]) { bget = true; break; }
  }
  if (!bget) tmax = (tsum + b[idx[n - 1]] - tau) / n;
  for (int i = 0; i < n; ++i) {
    const double v = b[i] - tmax;
    b[i] = (v < 0.0 ? 0.0 : v) + pc;
  }
}

// One warp per row. SIMPLEX: Q rows (tableau K+2, with the shift mu from v_kk);
// otherwise P rows (tableau K+1). `g` is the gradient as the reference's caller passes it
// (negated), so the tableau's last row/column holds -g. sqp_kernel.cu:177-311.
template <int KM, bool SIMPLEX>
__global__ void sqp_kernel(const double* __restrict__ H, const double* __restrict__ g,
                           const double* __restrict__ X, const double* __restrict__ v_kk, int64_t rows,
                           int K, double* __restrict__ Xn, int wpb) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  SqpScratch<KM>& s = reinterpret_cast<SqpScratch<KM>*>(smem)[warp];
  const int sz = SIMPLEX ? K + 2 : K + 1;
  for (int64_t row = (int64_t)blockIdx.x * wpb + warp; row < rows; row += (int64_t)gridDim.x * wpb) {
    const double* Hr = H + row * K * K;
    const double* gr = g + row * K;
    const double* xr = X + row * K;
    double mu = 0.0;
    if (SIMPLEX) {
      // mu = 2 max(0, (|t|_1 - 2 |t_0|) / K), t = v_kk (H v_kk[:,0]); sums in index order
      for (int i = lane; i < K; i += 32) {
        double t = 0.0;
        for (int j = 0; j < K; ++j) t += Hr[i * K + j] * v_kk[j * K];
        s.tmp[i] = t;
      }
      __syncwarp();
      for (int i = lane; i < K; i += 32) {
        double t2 = 0.0;
        for (int j = 0; j < K; ++j) t2 += v_kk[i * K + j] * s.tmp[j];
        s.out[i] = t2;
      }
      __syncwarp();
      if (lane == 0) {
        double norm1 = 0.0;
        for (int i = 0; i < K; ++i) norm1 += fabs(s.out[i]);
        double m = 2.0 * ((norm1 - 2.0 * fabs(s.out[0])) / K);
        s.tmp[0] = m < 0.0 ? 0.0 : m;
      }
      __syncwarp();
      mu = s.tmp[0];
      __syncwarp();
    }
    for (int e = lane; e < sz * sz; e += 32) {
      const int i = e / sz, j = e - i * sz;
      double v = 0.0;
      if (i < K && j < K) v = Hr[i * K + j] + mu;
      else if (i < K && j == sz - 1) v = -gr[i];
      else if (j < K && i == sz - 1) v = -gr[j];
      else if (SIMPLEX && ((i < K && j == K) || (j < K && i == K))) v = 1.0;
      s.tab[e] = v;
    }
    for (int i = lane; i < K; i += 32) s.par[i] = xr[i];
    __syncwarp();
    if (SIMPLEX && lane == 0) {
      double sx = 0.0;
      for (int i = 0; i < K; ++i) sx += xr[i];
      s.tab[K * sz + (K + 1)] = 1.0 - sx;
      s.tab[(K + 1) * sz + K] = 1.0 - sx;
    }
    // the QP checks each pivot against the diagonal as it was before any sweep
    for (int i = lane; i < K; i += 32) s.out[i] = s.tab[i * sz + i];
    __syncwarp();
    quadratic_program<KM>(s, K, SIMPLEX ? 1 : 0, lane);
    __syncwarp();
    for (int i = lane; i < K; i += 32) s.out[i] = s.par[i] + s.delta[i];
    __syncwarp();
    if (SIMPLEX) {
      if (lane == 0) project_simplex_row(s.out, K, 1e-5);
    } else {
      for (int i = lane; i < K; i += 32) s.out[i] = fmin(fmax(s.out[i], 1e-5), 1.0 - 1e-5);
    }
    __syncwarp();
    for (int i = lane; i < K; i += 32) Xn[row * K + i] = s.out[i];
    __syncwarp();
  }
}

template <typename S>
static int warps_per_block(size_t fixed) {
  // keep a block's shared memory within 96 KiB, at most 8 warps
  int w = (int)((96 * 1024 - fixed) / sizeof(S));
  return w < 1 ? 1 : (w > 8 ? 8 : w);
}

}  // namespace solve

#define ADX_KM_SWITCH(K, X) \
  if ((K) <= 8) { X(8) } else if ((K) <= 16) { X(16) } else if ((K) <= 32) { X(32) } else { X(64) }

static int grid_for(int64_t rows, int wpb) {
  const int64_t need = ceil_div(rows, wpb);
  const int64_t cap = (int64_t)sm_count() * 16;
  return (int)(need < cap ? (need < 1 ? 1 : need) : cap);
}

}  // namespace adx

using namespace adx;

extern "C" int adx_bvls(const double* A, const double* B, int64_t M, int K, double lower, double upper,
                        double* X, void* stream) {
  if (!A || !B || !X || M < 0 || K < 1 || K > ADX_MAX_K) {
    adx_set_message("adx_bvls: bad argument");
    return ADX_ERR_ARG;
  }
  if (M == 0) return ADX_OK;
  cudaStream_t st = as_stream(stream);
#define LAUNCH(KM)                                                                                      \
  {                                                                                                     \
    const size_t fixed = (size_t)KM * KM * sizeof(double);                                              \
    const int wpb = solve::warps_per_block<solve::BvlsScratch<KM>>(fixed);                              \
    const size_t smem = fixed + (size_t)wpb * sizeof(solve::BvlsScratch<KM>);                           \
    ADX_CUDA_TRY(cudaFuncSetAttribute(solve::bvls_kernel<KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    solve::bvls_kernel<KM><<<grid_for(M, wpb), 32 * wpb, smem, st>>>(A, B, M, K, lower, upper, X, wpb); \
  }
  ADX_KM_SWITCH(K, LAUNCH)
#undef LAUNCH
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

template <bool SIMPLEX>
static int launch_sqp(const double* H, const double* g, const double* X, const double* v_kk, int64_t rows,
                      int K, double* Xn, void* stream) {
  cudaStream_t st = as_stream(stream);
#define LAUNCH(KM)                                                                                      \
  {                                                                                                     \
    const int wpb = solve::warps_per_block<solve::SqpScratch<KM>>(0);                                   \
    const size_t smem = (size_t)wpb * sizeof(solve::SqpScratch<KM>);                                    \
    ADX_CUDA_TRY(cudaFuncSetAttribute(solve::sqp_kernel<KM, SIMPLEX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    solve::sqp_kernel<KM, SIMPLEX><<<grid_for(rows, wpb), 32 * wpb, smem, st>>>(H, g, X, v_kk, rows, K, Xn, wpb); \
  }
  ADX_KM_SWITCH(K, LAUNCH)
#undef LAUNCH
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_sqp_q(const double* XtX, const double* Xtz, const double* Q, const double* v_kk, int64_t N,
                         int K, double* Q_next, void* stream) {
  if (!XtX || !Xtz || !Q || !v_kk || !Q_next || N < 0 || K < 1 || K > ADX_MAX_K) {
    adx_set_message("adx_sqp_q: bad argument");
    return ADX_ERR_ARG;
  }
  if (N == 0) return ADX_OK;
  return launch_sqp<true>(XtX, Xtz, Q, v_kk, N, K, Q_next, stream);
}

extern "C" int adx_sqp_p(const double* XtX, const double* Xtz, const double* P, int64_t M, int K,
                         double* P_next, void* stream) {
  if (!XtX || !Xtz || !P || !P_next || M < 0 || K < 1 || K > ADX_MAX_K) {
    adx_set_message("adx_sqp_p: bad argument");
    return ADX_ERR_ARG;
  }
  if (M == 0) return ADX_OK;
  return launch_sqp<false>(XtX, Xtz, P, nullptr, M, K, P_next, stream);
}

// ---------------------------------------------------------------- projections

namespace adx {
namespace solve {

// Thread per row: Q rows onto {q >= 1e-5, sum q = 1} (sqp.pyx:112-146), P rows clamped to
// [1e-5, 1 - 1e-5] (sqp.pyx:148-151).
__global__ void project_simplex_kernel(double* __restrict__ X, int64_t rows, int K) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  double b[ADX_MAX_K];
  for (int k = 0; k < K; ++k) b[k] = X[r * K + k];
  project_simplex_row(b, K, 1e-5);
  for (int k = 0; k < K; ++k) X[r * K + k] = b[k];
}

__global__ void project_box_kernel(double* __restrict__ X, int64_t n) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) X[e] = fmin(fmax(X[e], 1e-5), 1.0 - 1e-5);
}

}  // namespace solve
}  // namespace adx

extern "C" int adx_project_simplex(double* Q, int64_t N, int K, void* stream) {
  if (!Q || N < 0 || K < 1 || K > ADX_MAX_K) {
    adx_set_message("adx_project_simplex: bad argument");
    return ADX_ERR_ARG;
  }
  if (N == 0) return ADX_OK;
  solve::project_simplex_kernel<<<(unsigned)ceil_div(N, 128), 128, 0, as_stream(stream)>>>(Q, N, K);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_project_box(double* P, int64_t M, int K, void* stream) {
  if (!P || M < 0 || K < 1 || K > ADX_MAX_K) {
    adx_set_message("adx_project_box: bad argument");
    return ADX_ERR_ARG;
  }
  const int64_t n = M * K;
  if (n == 0) return ADX_OK;
  solve::project_box_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, as_stream(stream)>>>(P, n);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}
