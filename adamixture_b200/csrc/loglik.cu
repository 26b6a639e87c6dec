// Binomial log-likelihood of (P, Q) over the packed genotypes, float64 sum
// (adamixture/model/em_adam_gpu.py:226-279):
//   L = sum over observed (j,i) of g log h + (2-g) log(1-h),  h = clamp(P_j.Q_i, 1e-10, 1-1e-10).
//
// Instead of two float64 logarithms per entry, each thread multiplies the per-entry factor
//   f = h^g (1-h)^(2-g)  (1 when missing)
// into a float64 running product per sample slot and moves the binary exponent into an
// integer every packed quad (4 entries: f >= 1e-20, so the product never leaves the normal
// range). log(prod) + e*ln2 once per thread gives the same sum as the per-entry logs to
// float64 rounding (each multiply adds <= 2^-53 relative error, i.e. <= 1.1e-16 absolute in
// the log). h is formed in float64 (ADX_F64) or float32 (ADX_F32) from P and Q of that type;
// with a float32 h the factor is formed in float32 too (the running product stays float64).
// The float32 path holds P scaled by 2^31 (exact: a power of two), so h, 1-h and f come out
// scaled by 2^31, 2^31 and 2^62 with the same roundings; a factor then lies in
// [2^62 1e-20, 2^62] = [0.046, 4.6e18] and the product of two of them in [2.1e-3, 2.1e37], a
// normal float32. The two factors of an entry pair are multiplied in float32 (one more
// rounding, 2^-24 relative) and the pair goes into the float64 product with one conversion
// and one multiply; the 2^248 of every packed quad is taken off the exponent at the end.
// Per-block float64 partials are summed by a one-block kernel in block order: deterministic.
#include "common.cuh"

#include <math.h>
#include <stdio.h>

#include <mutex>

namespace adx {

constexpr int LL_TPB = 256;
// 12 per SM on 148 SMs: whole waves at 1, 2, 3, 4 or 6 resident blocks per SM (the instances
// hold 1 to 4); fixed, so the summation order does not depend on the GPU
constexpr int LL_BLOCKS = 1776;
constexpr float LL_SCALE = 2147483648.0f;  // 2^31: float32 P is held x LL_SCALE
constexpr int LL_QUAD_EXP = 248;          // a quad's four factors carry (2^62)^4

template <typename R, int KMAX>
struct LlCfg {
  static constexpr int SPT = (sizeof(R) == 4) ? (KMAX <= 16 ? 4 : (KMAX <= 32 ? 2 : 1))
                                              : (KMAX <= 16 ? 2 : 1);
  static constexpr int CH = 32;
};

// Split x = m * 2^e with m in [0.5, 1): returns m, adds e to *e.
__device__ __forceinline__ double renorm(double x, int& e) {
  int hi = __double2hiint(x);
  const int lo = __double2loint(x);
  const int ex = ((hi >> 20) & 0x7FF) - 1022;
  e += ex;
  hi = (hi & 0x800FFFFF) | (1022 << 20);
  return __hiloint2double(hi, lo);
}

// Packed float32 pair: d = a * b + c per lane (fma.rn per lane, as the scalar FMA).
__device__ __forceinline__ unsigned long long fma_f32x2(unsigned long long a, unsigned long long b,
                                                        unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack_f32x2(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// vec: the host checked that N is a multiple of SPT and G is SPT-byte aligned, so a
// thread's SPT bytes of a packed row are one aligned load.
template <typename R, int KMAX>
__global__ void __launch_bounds__(LL_TPB, KMAX <= 12 ? 3 : 1)
loglik_kernel(const uint8_t* __restrict__ G, const R* __restrict__ P, const R* __restrict__ Q,
              int64_t M, int64_t N, int K, int64_t n_stile, int n_split, int n_mblk, int64_t mb,
              int vec, double* __restrict__ partial) {
  using C = LlCfg<R, KMAX>;
  constexpr int SPT = C::SPT, CH = C::CH;
  // float32 h of two samples at once with packed FMAs: P is kept duplicated {p, p}
  constexpr bool PAIRS = sizeof(R) == 4 && SPT % 2 == 0;
  __shared__ __align__(16) unsigned char ps_raw[CH * KMAX * (PAIRS ? 8 : sizeof(R))];
  R(*Ps)[KMAX] = reinterpret_cast<R(*)[KMAX]>(ps_raw);
  unsigned long long(*Ps2)[KMAX] = reinterpret_cast<unsigned long long(*)[KMAX]>(ps_raw);
  __shared__ double wsum[LL_TPB / 32];
  const int mblk = blockIdx.x % n_mblk;
  const int split = blockIdx.x / n_mblk;
  const int64_t j0 = (int64_t)mblk * mb;
  const int64_t j1 = min(M, j0 + mb);
  const int64_t W = (int64_t)LL_TPB * SPT;
  double acc = 0.0;
  for (int64_t st = split; st < n_stile; st += n_split) {
    const int64_t i0 = st * W + (int64_t)threadIdx.x * SPT;
    const bool vload = vec && i0 < N;
    // the thread's SPT bytes of packed row `row` (byte u = sample i0 + u; 0xFF, all
    // missing, past N)
    auto load_word = [&](int64_t row) -> uint32_t {
      const uint8_t* src = G + row * N + i0;
      if (vload) {
        if constexpr (SPT == 4) return __ldg(reinterpret_cast<const unsigned int*>(src));
        else if constexpr (SPT == 2) return (uint32_t)__ldg(reinterpret_cast<const unsigned short*>(src));
        else return (uint32_t)__ldg(src);
      }
      uint32_t w = 0;
#pragma unroll
      for (int u = 0; u < SPT; ++u) w |= (i0 + u < N ? (uint32_t)__ldg(src + u) : 0xFFu) << (8 * u);
      return w;
    };
    R q[PAIRS ? 1 : SPT][KMAX];                               // scalar path
    unsigned long long qp[PAIRS ? SPT / 2 : 1][KMAX];         // packed path: {q_u, q_u+1}
    double prod[SPT];
    int ex[SPT];
    int quads = 0;  // packed quads folded into prod (float32 path: 2^248 each to take off)
    auto qval = [&](int u, int k) -> R { return (i0 + u < N && k < K) ? Q[(i0 + u) * K + k] : (R)0; };
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
      prod[u] = 1.0;
      ex[u] = 0;
    }
    if constexpr (PAIRS) {
#pragma unroll
      for (int v = 0; v < SPT / 2; ++v)
#pragma unroll
        for (int k = 0; k < KMAX; ++k) qp[v][k] = pack_f32x2((float)qval(2 * v, k), (float)qval(2 * v + 1, k));
    } else {
#pragma unroll
      for (int u = 0; u < SPT; ++u)
#pragma unroll
        for (int k = 0; k < KMAX; ++k) q[u][k] = qval(u, k);
    }
    for (int64_t c0 = j0; c0 < j1; c0 += CH) {
      const int cn = (int)min((int64_t)CH, j1 - c0);
      __syncthreads();
      for (int e = threadIdx.x; e < CH * KMAX; e += LL_TPB) {
        const int jl = e / KMAX, k = e % KMAX;
        R v = (jl < cn && k < K) ? P[(c0 + jl) * K + k] : (R)0;
        if constexpr (sizeof(R) == 4) v *= LL_SCALE;
        if constexpr (PAIRS) Ps2[jl][k] = pack_f32x2((float)v, (float)v);
        else Ps[jl][k] = v;
      }
      __syncthreads();
      uint32_t word = load_word(c0 >> 2);
      for (int qd = 0; qd < cn; qd += 4) {
        const uint32_t cur = word;
        if (qd + 4 < cn) word = load_word((c0 + qd + 4) >> 2);  // next quad, ahead of the math
        // no early exit for a ragged chunk end (only the last chunk, when M % 4 != 0): the
        // entries past it count as missing (factor 1), so the four SNPs' dot products are
        // independent and interleave (Ps rows past cn are zeros, inside the CH-row tile)
        float fpair[SPT];  // float32 path: the scaled factor of the pair's first entry
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const int jl = qd + s;
          const bool live = jl < cn;
          R h[SPT];
          if constexpr (PAIRS) {
#pragma unroll
            for (int v = 0; v < SPT / 2; ++v) {
              unsigned long long a2 = 0ull;
#pragma unroll
              for (int k = 0; k < KMAX; ++k) a2 = fma_f32x2(Ps2[jl][k], qp[v][k], a2);
              float lo, hi;
              unpack_f32x2(a2, lo, hi);
              h[2 * v] = lo;
              h[2 * v + 1] = hi;
            }
          } else {
#pragma unroll
            for (int u = 0; u < SPT; ++u) {
              h[u] = 0;
#pragma unroll
              for (int k = 0; k < KMAX; ++k) h[u] += Ps[jl][k] * q[u][k];
            }
          }
#pragma unroll
          for (int u = 0; u < SPT; ++u) {
            const unsigned g = live ? genotype(cur >> (8 * u), s) : 3u;
            if constexpr (sizeof(R) == 4) {
              // float32 h: the factor in float32 as well (its rounding, 6e-8 relative, is below
              // that of h itself); the clamp h in [1e-10, 1-1e-10] is applied to h and to 1-h,
              // since 1-1e-10 is not a float32 value. All three are x2^31 (h, 1-h) and x2^62 (f).
              // f = x * y from the genotype's two bits: g=0 om*om, g=1 om*hf, g=2 hf*hf, missing
              // 2^31*2^31 (the scaled 1), the same products as a four-way select, with two
              // selects and one multiply
              const float hf = fmaxf(h[u], (float)LL_CLAMP * LL_SCALE);
              const float om = fmaxf(LL_SCALE - h[u], (float)LL_CLAMP * LL_SCALE);
              const bool miss = g == 3u, gz = g == 0u;
              const float hf3 = miss ? LL_SCALE : hf;
              const float f = ((g & 2u) ? hf3 : om) * (gz ? om : hf3);
              if (s & 1) prod[u] *= (double)(fpair[u] * f);
              else fpair[u] = f;
            } else {
              const double hd = fmin(fmax((double)h[u], LL_CLAMP), 1.0 - LL_CLAMP);
              const double om = 1.0 - hd;
              const bool miss = g == 3u, gz = g == 0u;
              const double hd3 = miss ? 1.0 : hd;
              prod[u] *= ((g & 2u) ? hd3 : om) * (gz ? om : hd3);  // the float32 form's two selects
            }
          }
        }
#pragma unroll
        for (int u = 0; u < SPT; ++u) prod[u] = renorm(prod[u], ex[u]);
        ++quads;
      }
    }
    const double off = sizeof(R) == 4 ? (double)LL_QUAD_EXP * (double)quads : 0.0;
#pragma unroll
    for (int u = 0; u < SPT; ++u) acc += log(prod[u]) + ((double)ex[u] - off) * 0.69314718055994530942;
  }
  // block reduction in fixed order
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < LL_TPB / 32; ++w) s += wsum[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int n, double* __restrict__ out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w >= 1; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

int pick_kmax(int K);

struct LlPlan {
  int kmax, spt;
  int64_t n_stile;
  int n_split, n_mblk;
  int64_t mb;
};

template <typename R, int KMAX>
static int spt_of() { return LlCfg<R, KMAX>::SPT; }

#define ADX_LL_KMAX_SWITCH(kmax, MACRO)                                                \
  switch (kmax) {                                                                      \
    case 2: MACRO(2); break;   case 3: MACRO(3); break;   case 4: MACRO(4); break;     \
    case 6: MACRO(6); break;   case 8: MACRO(8); break;   case 10: MACRO(10); break;   \
    case 12: MACRO(12); break; case 16: MACRO(16); break; case 24: MACRO(24); break;   \
    case 32: MACRO(32); break; case 48: MACRO(48); break; case 64: MACRO(64); break;   \
    default: break;                                                                    \
  }

// Whether a thread's SPT bytes of a packed row can be one aligned load: N a multiple of
// SPT (so every row starts SPT-aligned relative to G) and G itself SPT-byte aligned.
static int ll_vec_loads(const uint8_t* G, int64_t N, int spt) {
  return (N % spt == 0) && (reinterpret_cast<uintptr_t>(G) % (uintptr_t)spt == 0) ? 1 : 0;
}

static int ll_plan(int64_t M, int64_t N, int K, int prec, LlPlan& pl) {
  if (M <= 0 || N <= 0 || K < 1 || K > ADX_MAX_K) return ADX_ERR_ARG;
  if (prec != ADX_F64 && prec != ADX_F32 && prec != ADX_BF16 && prec != ADX_F16) return ADX_ERR_UNSUPPORTED;
  pl.kmax = pick_kmax(K);
  int spt = 1;
#define S64(KM) spt = spt_of<double, KM>()
#define S32(KM) spt = spt_of<float, KM>()
  if (prec == ADX_F64) { ADX_LL_KMAX_SWITCH(pl.kmax, S64) } else { ADX_LL_KMAX_SWITCH(pl.kmax, S32) }
#undef S64
#undef S32
  pl.spt = spt;
  pl.n_stile = ceil_div(N, (int64_t)LL_TPB * spt);
  int64_t n_split = pl.n_stile < 8 ? pl.n_stile : 8;
  // at most LL_BLOCKS blocks (rounding the SNP blocks up to 32 rows only lowers the count),
  // so the grid never spills a few blocks into one more wave
  int64_t n_mblk = LL_BLOCKS / n_split;
  const int64_t max_mblk = ceil_div(M, 32);
  n_mblk = n_mblk > max_mblk ? max_mblk : n_mblk;
  int64_t mb = ceil_div(ceil_div(M, n_mblk), 32) * 32;
  n_mblk = ceil_div(M, mb);
  pl.n_split = (int)n_split;
  pl.n_mblk = (int)n_mblk;
  pl.mb = mb;
  return ADX_OK;
}

}  // namespace adx

using namespace adx;

// Float64 with K <= 16: h on the float64 MMA tiles of the float64 sweep (em_sweep_dmma.cu);
// `nblk` receives its partial count, and partial == nullptr only queries it.
namespace adx {
int dmma_loglik(const uint8_t* G, const double* P, const double* Q, int64_t M, int64_t N, int K, double* partial,
                int* nblk, cudaStream_t st);
}
constexpr int LL_DMMA_MAX_K = 16;

extern "C" int adx_loglik_workspace_bytes(int64_t M, int64_t N, int K, int precision, size_t* bytes) {
  LlPlan pl;
  const int rc = ll_plan(M, N, K, precision, pl);
  if (rc || !bytes) { adx_set_message("adx_loglik_workspace_bytes: bad arguments"); return rc ? rc : ADX_ERR_ARG; }
  int nblk = pl.n_split * pl.n_mblk;
  if (precision == ADX_F64 && K <= LL_DMMA_MAX_K) {
    int nd = 0;
    if (dmma_loglik(nullptr, nullptr, nullptr, M, N, K, nullptr, &nd, nullptr) == ADX_OK && nd > nblk) nblk = nd;
  }
  *bytes = (size_t)nblk * sizeof(double) + 256;
  return ADX_OK;
}

extern "C" int adx_loglik(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                          const void* P, const void* Q, double* out, void* workspace,
                          size_t workspace_bytes, void* stream) {
  LlPlan pl;
  int rc = ll_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_loglik: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !out || !workspace) { adx_set_message("adx_loglik: null pointer"); return ADX_ERR_ARG; }
  double* part = reinterpret_cast<double*>(workspace);
  cudaStream_t st = as_stream(stream);
  if (precision == ADX_F64 && K <= LL_DMMA_MAX_K) {
    int nd = 0;
    rc = dmma_loglik(G, (const double*)P, (const double*)Q, M, N, K, nullptr, &nd, st);
    if (rc) return rc;
    if (workspace_bytes < (size_t)nd * sizeof(double)) { adx_set_message("adx_loglik: workspace too small"); return ADX_ERR_WORKSPACE; }
    rc = dmma_loglik(G, (const double*)P, (const double*)Q, M, N, K, part, &nd, st);
    if (rc) return rc;
    sum_partials_kernel<<<1, 256, 0, st>>>(part, nd, out);
    ADX_LAUNCH_CHECK();
    return ADX_OK;
  }
  const int nblk = pl.n_split * pl.n_mblk;
  if (workspace_bytes < (size_t)nblk * sizeof(double)) { adx_set_message("adx_loglik: workspace too small"); return ADX_ERR_WORKSPACE; }
  const int vec = ll_vec_loads(G, N, pl.spt);
#define L64(KM) loglik_kernel<double, KM><<<nblk, LL_TPB, 0, st>>>(G, (const double*)P, (const double*)Q, M, N, K, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, vec, part)
#define L32(KM) loglik_kernel<float, KM><<<nblk, LL_TPB, 0, st>>>(G, (const float*)P, (const float*)Q, M, N, K, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, vec, part)
  if (precision == ADX_F64) { ADX_LL_KMAX_SWITCH(pl.kmax, L64) } else { ADX_LL_KMAX_SWITCH(pl.kmax, L32) }
#undef L64
#undef L32
  ADX_LAUNCH_CHECK();
  sum_partials_kernel<<<1, 256, 0, st>>>(part, nblk, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

// ---------------------------------------------------------------- allocation-free variant
//
// adx_loglik_noalloc: the same log-likelihood for callers that cannot allocate device
// memory. Typical ones: a host whose device memory is owned by another allocator (a
// framework pool or a language runtime that must account for every byte), and code
// paths where the implicit device-wide synchronisation of cudaMalloc/cudaFree is not
// acceptable. adx_loglik needs a small caller-provided workspace for its per-block
// partial sums; this variant keeps them in a file-scope device array instead.
//
// Limit: the array holds ADX_LL_NOALLOC_MAX_PARTIALS float64 partial sums (16 KiB) on every
// GPU that loads the library, until the process exits. The launch plan uses at most
// LL_BLOCKS = 1776 partials for any M, N and K, so every problem size fits; a plan that needed more would be rejected with
// ADX_ERR_WORKSPACE.
//
// Set-up: host code cannot use the array's name as a device address (it names a host-side
// stand-in). The first call on each device, with that device current, looks the address
// up with cudaGetSymbolAddress and caches it; make that first call before any stream
// capture begins. The cached address belongs to the device's current primary context: a
// process that calls cudaDeviceReset (which can reload the module at another address)
// must not call this entry point on that device afterwards. The array is shared by every call and keeps the previous call's
// contents; each call overwrites every partial it reads, so nothing needs clearing. Two
// calls whose launches overlap on the GPU (different streams, no ordering) race on it.

#define ADX_LL_NOALLOC_MAX_PARTIALS 2048

static __device__ __align__(256) double g_ll_noalloc_partials[ADX_LL_NOALLOC_MAX_PARTIALS];

static std::mutex g_ll_noalloc_mu;
static double* g_ll_noalloc_ptr[256];

static int ll_noalloc_scratch(double** out) {
  int dev = -1;
  ADX_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) { adx_set_message("adx_loglik_noalloc: device index out of range"); return ADX_ERR_ARG; }
  std::lock_guard<std::mutex> lock(g_ll_noalloc_mu);
  if (!g_ll_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_ll_noalloc_partials);
    if (e != cudaSuccess || !p) {
      adx_set_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
      return ADX_ERR_CUDA;
    }
    g_ll_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_ll_noalloc_ptr[dev];
  return ADX_OK;
}

extern "C" int adx_loglik_noalloc(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                                  const void* P, const void* Q, double* out, void* stream) {
  LlPlan pl;
  int rc = ll_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_loglik_noalloc: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !out) { adx_set_message("adx_loglik_noalloc: null pointer"); return ADX_ERR_ARG; }
  const int nblk = pl.n_split * pl.n_mblk;
  if (nblk > ADX_LL_NOALLOC_MAX_PARTIALS) {
    char msg[160];
    snprintf(msg, sizeof(msg), "adx_loglik_noalloc: plan needs %d partial sums, the static scratch holds %d",
             nblk, ADX_LL_NOALLOC_MAX_PARTIALS);
    adx_set_message(msg);
    return ADX_ERR_WORKSPACE;
  }
  double* part = nullptr;
  rc = ll_noalloc_scratch(&part);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  if (precision == ADX_F64 && K <= LL_DMMA_MAX_K) {
    // the float64 MMA form, as adx_loglik runs it (at most 1776 partials)
    int nd = 0;
    rc = dmma_loglik(G, (const double*)P, (const double*)Q, M, N, K, nullptr, &nd, st);
    if (rc) return rc;
    if (nd > ADX_LL_NOALLOC_MAX_PARTIALS) { adx_set_message("adx_loglik_noalloc: plan too large"); return ADX_ERR_WORKSPACE; }
    rc = dmma_loglik(G, (const double*)P, (const double*)Q, M, N, K, part, &nd, st);
    if (rc) return rc;
    sum_partials_kernel<<<1, 256, 0, st>>>(part, nd, out);
    ADX_LAUNCH_CHECK();
    return ADX_OK;
  }
  const int vec = ll_vec_loads(G, N, pl.spt);
#define N64(KM) loglik_kernel<double, KM><<<nblk, LL_TPB, 0, st>>>(G, (const double*)P, (const double*)Q, M, N, K, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, vec, part)
#define N32(KM) loglik_kernel<float, KM><<<nblk, LL_TPB, 0, st>>>(G, (const float*)P, (const float*)Q, M, N, K, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, vec, part)
  if (precision == ADX_F64) { ADX_LL_KMAX_SWITCH(pl.kmax, N64) } else { ADX_LL_KMAX_SWITCH(pl.kmax, N32) }
#undef N64
#undef N32
  ADX_LAUNCH_CHECK();
  sum_partials_kernel<<<1, 256, 0, st>>>(part, nblk, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}
