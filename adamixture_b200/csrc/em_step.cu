// Fused Adam-EM E-step for the ADMIXTURE binomial model on B200 (sm_100a), CUDA-core form.
//
// One sweep over the packed genotype matrix computes, for every entry (SNP j, sample i),
//   h = P_j . Q_i,  rec = clamp(h, 1e-5, 1-1e-5),  a = g/rec,  b = (2-g)/(1-rec)  (0 if missing)
// and accumulates both sides of the two-sided reduction
//   A_j = sum_i a Q_i,  B_j = sum_i b Q_i           (P side: reduce over samples)
//   T_i = sum_j (a-b) P_j + sum_j b                  (Q side: reduce over SNPs)
// (adamixture/model/em_adam_gpu.py:46-78). The reference materialises ~6 float64 C x N
// temporaries per 8192-SNP chunk and runs 4 DGEMMs; here G is read once, 2 bits per entry.
//
// Work decomposition (deterministic, no atomics):
//  - a block owns a SNP range [j0, j1) ("SNP block", multiple of CH SNPs, quad aligned) and a
//    residue class of sample sub-tiles ("split"); a sub-tile is TPB*SPT consecutive samples,
//    SPT per thread (their Q rows and T accumulators live in registers);
//  - per SNP, each thread forms its SPT samples' contributions to A_j/B_j, a warp
//    reduce-scatter folds the 2K values over 32 lanes, a cross-warp pass folds the 8 warps
//    and adds the block's partial into AB_part[split][j] (the block is the only writer of
//    those rows, and always the same thread adds the same element);
//  - after its SNP range, each thread writes T_part[snp_block][i] for its samples.
// A second kernel reduces AB_part over splits and T_part over SNP blocks in float64, in a
// fixed order, and either writes A/B/T or applies em_final_update + the Adam move directly.
#include "common.cuh"

#include <math.h>

namespace adx {

constexpr int TPB = 256;
constexpr int WARPS = TPB / 32;
// Block count of a sweep, at most (12 per SM on 148 SMs: whole waves at 1, 2, 3, 4 or 6
// resident blocks per SM, which covers every instance); fixed so the partition, hence the
// summation order, never depends on the GPU.
constexpr int PLAN_BLOCKS = 1776;

template <typename R, int KMAX>
struct EmCfg {
  static constexpr int SPT = (sizeof(R) == 4) ? (KMAX <= 16 ? 4 : (KMAX <= 32 ? 2 : 1))
                                              : (KMAX <= 8 ? 2 : 1);
  static constexpr int W = TPB * SPT;            // samples per sub-tile
  static constexpr int V = 2 * KMAX;             // A and B values per SNP
  static constexpr int VP = ((V + 31) / 32) * 32;
  static constexpr int NCH = VP / 32;
  static constexpr int CH_RAW = 40960 / (WARPS * VP * (int)sizeof(R));
  static constexpr int CH = CH_RAW >= 32 ? 32 : (CH_RAW / 4) * 4;  // SNPs staged per chunk
  static_assert(CH >= 4, "chunk must hold a packed quad");
};

struct EmPlan {
  int64_t M, N;
  int K, kmax, prec;
  int W, CH;
  int64_t n_stile;   // sample sub-tiles
  int n_split;       // sample splits (partials of A/B)
  int n_mblk;        // SNP blocks (partials of T)
  int64_t mb;        // SNPs per SNP block
  size_t ab_elems, t_elems, elem_size;
  // Workspace: a 256-byte header whose first word is the sweep's sticky status (the same
  // offset for every shape, so a shared grow-only buffer keeps it), then the partials.
  // The tensor-core sweep also keeps a 16-bit (FP16 or BF16) copy of Q after the partials.
  static constexpr size_t HEADER = 256;
  size_t extra_bytes = 0;
  size_t extra_offset() const { return (HEADER + (ab_elems + t_elems) * elem_size + 255) & ~size_t(255); }
  size_t bytes() const { return extra_offset() + extra_bytes; }
};

// ---------------------------------------------------------------- device helpers

__device__ __forceinline__ float clampr(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ double clampr(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

// a = ga/rec, b = gb/(1-rec). Float: one correctly rounded reciprocal of rec*(1-rec).
// Double: two IEEE divisions, as the reference computes them.
__device__ __forceinline__ void ratios(float ga, float gb, float rec, float omr, float& a, float& b) {
  const float r = __frcp_rn(rec * omr);
  a = ga * (omr * r);
  b = gb * (rec * r);
}
__device__ __forceinline__ void ratios(double ga, double gb, double rec, double omr, double& a, double& b) {
  a = ga / rec;
  b = gb / omr;
}

// Warp reduce-scatter of 32 values: afterwards lane l holds sum over lanes of v[l].
template <typename R>
__device__ __forceinline__ R reduce_scatter32(R (&v)[32], int lane) {
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const bool up = (lane & h) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const R send = up ? v[i] : v[i + h];
      const R keep = up ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
    }
  }
  return v[0];
}

// The same for VR (a power of two below 32) values per lane: the butterfly over the low
// log2(VR) lane bits leaves lane L with value L & (VR - 1) summed over its group of VR lanes,
// and a plain xor-sum across the 32 / VR groups completes it: (VR - 1) + log2(32 / VR)
// shuffles instead of 31 for a vector padded to 32.
template <int VR, typename R>
__device__ __forceinline__ R reduce_scatter_small(R (&v)[VR], int lane) {
#pragma unroll
  for (int h = VR / 2; h >= 1; h >>= 1) {
    const bool up = (lane & h) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const R send = up ? v[i] : v[i + h];
      const R keep = up ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
    }
  }
#pragma unroll
  for (int h = VR; h < 32; h <<= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], h);
  return v[0];
}

// ---------------------------------------------------------------- E-step sweep

template <typename R, int KMAX>
__global__ void __launch_bounds__(TPB)
em_sweep_kernel(const uint8_t* __restrict__ G, const R* __restrict__ P, const R* __restrict__ Q,
                int64_t M, int64_t N, int K, int64_t n_stile, int n_split, int n_mblk, int64_t mb,
                R* __restrict__ ABp, R* __restrict__ Tp) {
  using C = EmCfg<R, KMAX>;
  constexpr int SPT = C::SPT, CH = C::CH, VP = C::VP, V = C::V;
  __shared__ R Ps[CH][KMAX];
  __shared__ R red[WARPS][CH][VP];

  const int mblk = blockIdx.x % n_mblk;
  const int split = blockIdx.x / n_mblk;
  const int64_t j0 = (int64_t)mblk * mb;
  const int64_t j1 = min(M, j0 + mb);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool aligned4 = (SPT == 4) && ((N & 3) == 0);
  const R ELO = (R)E_CLAMP, EHI = (R)(1.0 - E_CLAMP);

  bool first = true;
  for (int64_t st = split; st < n_stile; st += n_split) {
    const int64_t i0 = st * C::W + (int64_t)threadIdx.x * SPT;
    R q[SPT][KMAX], tab[SPT][KMAX], tb[SPT];
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
      tb[u] = 0;
#pragma unroll
      for (int k = 0; k < KMAX; ++k) {
        tab[u][k] = 0;
        q[u][k] = (i0 + u < N && k < K) ? Q[(i0 + u) * K + k] : (R)0;
      }
    }

    for (int64_t c0 = j0; c0 < j1; c0 += CH) {
      const int cn = (int)min((int64_t)CH, j1 - c0);
      __syncthreads();
      for (int e = threadIdx.x; e < CH * KMAX; e += TPB) {
        const int jl = e / KMAX, k = e % KMAX;
        Ps[jl][k] = (jl < cn && k < K) ? P[(c0 + jl) * K + k] : (R)0;
      }
      __syncthreads();

      for (int qd = 0; qd < cn; qd += 4) {
        const int64_t row = (c0 + qd) >> 2;
        uint32_t bytes[SPT];
        if (aligned4 && i0 < N) {
          const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(G + row * N + i0));
#pragma unroll
          for (int u = 0; u < SPT; ++u) bytes[u] = (w >> (8 * u)) & 0xFFu;
        } else {
#pragma unroll
          for (int u = 0; u < SPT; ++u) bytes[u] = (i0 + u < N) ? (uint32_t)__ldg(G + row * N + i0 + u) : 0xFFu;
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const int jl = qd + s;
          if (jl >= cn) break;  // uniform across the block
          R a[SPT], b[SPT], hh[SPT];
#pragma unroll
          for (int u = 0; u < SPT; ++u) {
            R h = 0;
#pragma unroll
            for (int k = 0; k < KMAX; ++k) h += Ps[jl][k] * q[u][k];
            hh[u] = h;
          }
#pragma unroll
          for (int u = 0; u < SPT; ++u) {
            const unsigned g = genotype(bytes[u], s);
            const R rec = clampr(hh[u], ELO, EHI);
            const R omr = (R)1 - rec;
            const R ga = (g == 3u) ? (R)0 : (R)g;
            const R gb = (g == 3u) ? (R)0 : (R)(2u - g);
            ratios(ga, gb, rec, omr, a[u], b[u]);
            const R d = a[u] - b[u];
#pragma unroll
            for (int k = 0; k < KMAX; ++k) tab[u][k] += d * Ps[jl][k];
            tb[u] += b[u];
          }
          // this thread's part of value v of the SNP: A column v (v < KMAX), else B column
          // v - KMAX, summed over its samples
          auto part_of = [&](int v) {
            R acc = 0;
            if (v < KMAX) {
#pragma unroll
              for (int u = 0; u < SPT; ++u) acc += a[u] * q[u][v < KMAX ? v : 0];
            } else if (v < V) {
#pragma unroll
              for (int u = 0; u < SPT; ++u) acc += b[u] * q[u][v >= KMAX && v < V ? v - KMAX : 0];
            }
            return acc;
          };
          if constexpr (V <= 16) {
            // at most 16 values: a power-of-two vector of VR, reduced with fewer shuffles
            constexpr int VR = V <= 4 ? 4 : (V <= 8 ? 8 : 16);
            R part[VR];
#pragma unroll
            for (int v = 0; v < VR; ++v) part[v] = part_of(v);
            // lanes >= VR hold copies of lanes & (VR - 1): slots V.. of red are never read
            red[warp][jl][lane] = reduce_scatter_small<VR>(part, lane);
          } else if constexpr (V < 32 && ((V - 16) & (V - 17)) == 0) {
            // 16 + 4 or 16 + 8 values: two power-of-two vectors, 16 + 6 or 16 + 9 shuffle
            // steps instead of 31; lane l < 16 holds value l, lane 16 + i value 16 + i
            constexpr int VR2 = V - 16;
            R p1[16], p2[VR2];
#pragma unroll
            for (int v = 0; v < 16; ++v) p1[v] = part_of(v);
#pragma unroll
            for (int v = 0; v < VR2; ++v) p2[v] = part_of(16 + v);
            const R r1 = reduce_scatter_small<16>(p1, lane);
            const R r2 = reduce_scatter_small<VR2>(p2, lane);
            red[warp][jl][lane] = lane < 16 ? r1 : r2;
          } else {
#pragma unroll
            for (int c = 0; c < C::NCH; ++c) {
              R part[32];
#pragma unroll
              for (int l = 0; l < 32; ++l) part[l] = part_of(c * 32 + l);
              red[warp][jl][c * 32 + lane] = reduce_scatter32(part, lane);
            }
          }
        }
      }
      __syncthreads();
      const int nv = cn * V;
      for (int e = threadIdx.x; e < nv; e += TPB) {
        const int jl = e / V, v = e % V;
        const int k = v < KMAX ? v : v - KMAX;
        if (k >= K) continue;
        R sum = 0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) sum += red[w][jl][v];
        R* dst = ABp + ((int64_t)split * M + (c0 + jl)) * (2 * K) + (v < KMAX ? k : K + k);
        *dst = first ? sum : *dst + sum;
      }
    }
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
      if (i0 + u < N) {
        R* dst = Tp + ((int64_t)mblk * N + i0 + u) * K;
#pragma unroll
        for (int k = 0; k < KMAX; ++k)
          if (k < K) dst[k] = tab[u][k] + tb[u];
      }
    }
    first = false;
  }
}

// ---------------------------------------------------------------- reduce / targets / Adam

struct AdamArgs {
  double t, lr, b1, b2, eps;
  // captured iterations: the step is *t_dev + t (t the iteration's offset in the replay)
  const double* t_dev = nullptr;
};

__device__ __forceinline__ double adam_step_no(const AdamArgs& ad) { return ad.t_dev ? *ad.t_dev + ad.t : ad.t; }

// mode 0: write A, B, T (float64 statistics). mode 1: EM targets + Adam move on P and Q.
template <typename R, int KMAX>
__global__ void em_update_kernel(const R* __restrict__ ABp, const R* __restrict__ Tp, int64_t M,
                                 int64_t N, int K, int n_split, int n_mblk, int mode,
                                 double* __restrict__ outA, double* __restrict__ outB,
                                 double* __restrict__ outT, const double* __restrict__ q_bat,
                                 double* __restrict__ P, double* __restrict__ Q,
                                 float* __restrict__ P32, float* __restrict__ Q32,
                                 double* __restrict__ mP, double* __restrict__ vP,
                                 double* __restrict__ mQ, double* __restrict__ vQ, AdamArgs ad) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= M + N) return;
  const double t = adam_step_no(ad);
  const double bc1 = 1.0 - pow(ad.b1, t);
  const double bc2 = 1.0 - pow(ad.b2, t);
  if (row < M) {
    const int64_t j = row;
    double A[KMAX], B[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) { A[k] = 0.0; B[k] = 0.0; }
    for (int s = 0; s < n_split; ++s) {
      const R* src = ABp + ((int64_t)s * M + j) * (2 * K);
#pragma unroll
      for (int k = 0; k < KMAX; ++k)
        if (k < K) { A[k] += (double)src[k]; B[k] += (double)src[K + k]; }
    }
    if (mode == 0) {
#pragma unroll
      for (int k = 0; k < KMAX; ++k)
        if (k < K) { outA[j * K + k] = A[k]; outB[j * K + k] = B[k]; }
      return;
    }
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      if (k >= K) continue;
      const int64_t o = j * K + k;
      const double p = P[o];
      // em_final_update order: ((A-B)*P + B) -> clamp(min 1e-5) -> reciprocal -> *P -> *A
      const double den = fmax((A[k] - B[k]) * p + B[k], 1e-5);
      const double target = ((1.0 / den) * p) * A[k];
      const double delta = target - p;
      const double m = mP[o] * ad.b1 + (1.0 - ad.b1) * delta;
      const double v = vP[o] * ad.b2 + (1.0 - ad.b2) * (delta * delta);
      mP[o] = m;
      vP[o] = v;
      double np = p + (ad.lr * (m / bc1)) / (sqrt(v / bc2) + ad.eps);
      np = fmin(fmax(np, DOMAIN), 1.0 - DOMAIN);
      P[o] = np;
      if (P32) P32[o] = (float)np;
    }
    return;
  }
  const int64_t i = row - M;
  double T[KMAX];
#pragma unroll
  for (int k = 0; k < KMAX; ++k) T[k] = 0.0;
  for (int b = 0; b < n_mblk; ++b) {
    const R* src = Tp + ((int64_t)b * N + i) * K;
#pragma unroll
    for (int k = 0; k < KMAX; ++k)
      if (k < K) T[k] += (double)src[k];
  }
  if (mode == 0) {
#pragma unroll
    for (int k = 0; k < KMAX; ++k)
      if (k < K) outT[i * K + k] = T[k];
    return;
  }
  const double scale = 1.0 / fmax(q_bat[i], 1e-5);
  double qe[KMAX];
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    qe[k] = (k < K) ? (Q[i * K + k] * T[k]) * scale : 0.0;
    s += qe[k];
  }
  s = fmax(s, 1e-5);
  double tot = 0.0;
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    if (k >= K) continue;
    const int64_t o = i * K + k;
    const double qv = Q[o];
    const double delta = qe[k] / s - qv;
    const double m = mQ[o] * ad.b1 + (1.0 - ad.b1) * delta;
    const double v = vQ[o] * ad.b2 + (1.0 - ad.b2) * (delta * delta);
    mQ[o] = m;
    vQ[o] = v;
    double nq = qv + (ad.lr * (m / bc1)) / (sqrt(v / bc2) + ad.eps);
    nq = fmin(fmax(nq, DOMAIN), 1.0 - DOMAIN);
    qe[k] = nq;
    tot += nq;
  }
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    if (k >= K) continue;
    const double nq = qe[k] / tot;
    Q[i * K + k] = nq;
    if (Q32) Q32[i * K + k] = (float)nq;
  }
}

// ---------------------------------------------------------------- planning and dispatch

static const int KMAX_LIST[] = {2, 3, 4, 6, 8, 10, 12, 16, 24, 32, 48, 64};

int pick_kmax(int K) {
  for (int km : KMAX_LIST)
    if (K <= km) return km;
  return -1;
}

template <typename R, int KMAX>
static void cfg_of(int& W, int& CH) {
  W = EmCfg<R, KMAX>::W;
  CH = EmCfg<R, KMAX>::CH;
}

#define ADX_KMAX_SWITCH(kmax, MACRO)                                                   \
  switch (kmax) {                                                                      \
    case 2: MACRO(2); break;   case 3: MACRO(3); break;   case 4: MACRO(4); break;     \
    case 6: MACRO(6); break;   case 8: MACRO(8); break;   case 10: MACRO(10); break;   \
    case 12: MACRO(12); break; case 16: MACRO(16); break; case 24: MACRO(24); break;   \
    case 32: MACRO(32); break; case 48: MACRO(48); break; case 64: MACRO(64); break;   \
    default: break;                                                                    \
  }

int tc_plan(int64_t M, int64_t N, int K, int64_t& n_stile, int& n_split, int& n_mblk);
size_t tc_q_bytes(int64_t n_stile);
int tc_sweep(const uint8_t* G, const float* P, const float* Q, int64_t M, int64_t N, int K,
             int64_t n_stile, int n_split, int n_mblk, float* ABp, float* Tp, void* Qb, int* err,
             bool f16, cudaStream_t st);

int dmma_plan_width();
int dmma_plan_chunk();
int dmma_sweep(const uint8_t* G, const double* P, const double* Q, int64_t M, int64_t N, int K,
               int64_t n_stile, int n_split, int n_mblk, int64_t mb, double* ABp, double* Tp,
               cudaStream_t st, double* llp = nullptr, int b0 = 0, int b1 = 0);
// Float64 sweeps for K <= 16 run on the float64 tensor-core MMA (em_sweep_dmma.cu).
constexpr int DMMA_MAX_K = 16;

int em_plan(int64_t M, int64_t N, int K, int prec, EmPlan& pl) {
  if (M <= 0 || N <= 0 || K < 1 || K > ADX_MAX_K) return ADX_ERR_ARG;
  if (prec != ADX_F64 && prec != ADX_F32 && prec != ADX_BF16 && prec != ADX_F16) return ADX_ERR_UNSUPPORTED;
  pl.M = M; pl.N = N; pl.K = K; pl.prec = prec;
  pl.kmax = pick_kmax(K);
  if (prec == ADX_BF16 || prec == ADX_F16) {
    // tensor-core sweep: 896-SNP blocks x 128-sample tiles, float partials
    int64_t n_stile = 0;
    int n_split = 0, n_mblk = 0;
    const int rc = tc_plan(M, N, K, n_stile, n_split, n_mblk);
    if (rc) return rc;
    pl.W = 128; pl.CH = 0;
    pl.elem_size = sizeof(float);
    pl.n_stile = n_stile; pl.n_split = n_split; pl.n_mblk = n_mblk;
    pl.mb = 896;
    pl.ab_elems = (size_t)n_split * (size_t)M * 2 * K;
    pl.t_elems = (size_t)n_mblk * (size_t)N * K;
    pl.extra_bytes = tc_q_bytes(n_stile);
    return ADX_OK;
  }
  int W = 0, CH = 0;
#define CFG64(KM) cfg_of<double, KM>(W, CH)
#define CFG32(KM) cfg_of<float, KM>(W, CH)
  if (prec == ADX_F64) { ADX_KMAX_SWITCH(pl.kmax, CFG64) } else { ADX_KMAX_SWITCH(pl.kmax, CFG32) }
#undef CFG64
#undef CFG32
  if (prec == ADX_F64 && K <= DMMA_MAX_K) {
    W = dmma_plan_width();
    CH = dmma_plan_chunk();
  }
  pl.W = W; pl.CH = CH;
  pl.elem_size = prec == ADX_F64 ? sizeof(double) : sizeof(float);
  pl.n_stile = ceil_div(N, W);
  // minimise split*2MK + mblk*NK with split*mblk ~ PLAN_BLOCKS
  double s = sqrt((double)PLAN_BLOCKS * (double)N / (2.0 * (double)M));
  int64_t n_split = (int64_t)llround(s);
  n_split = n_split < 1 ? 1 : n_split;
  n_split = n_split > pl.n_stile ? pl.n_stile : n_split;
  n_split = n_split > PLAN_BLOCKS ? PLAN_BLOCKS : n_split;  // the grid stays within PLAN_BLOCKS
  int64_t max_mblk = ceil_div(M, CH);
  int64_t n_mblk = PLAN_BLOCKS / n_split;  // the grid stays within PLAN_BLOCKS
  n_mblk = n_mblk < 1 ? 1 : (n_mblk > max_mblk ? max_mblk : n_mblk);
  int64_t mb = ceil_div(ceil_div(M, n_mblk), CH) * CH;
  n_mblk = ceil_div(M, mb);
  pl.n_split = (int)n_split;
  pl.n_mblk = (int)n_mblk;
  pl.mb = mb;
  pl.ab_elems = (size_t)n_split * (size_t)M * 2 * K;
  pl.t_elems = (size_t)n_mblk * (size_t)N * K;
  // the float64 tensor-core sweep can also leave one log-likelihood partial per CTA
  if (prec == ADX_F64 && K <= DMMA_MAX_K) pl.extra_bytes = (size_t)n_split * (size_t)n_mblk * sizeof(double);
  return ADX_OK;
}

template <typename R>
static int launch_sweep(const EmPlan& pl, const uint8_t* G, const void* P, const void* Q, void* ws,
                        cudaStream_t st) {
  R* ABp = reinterpret_cast<R*>(reinterpret_cast<uint8_t*>(ws) + EmPlan::HEADER);
  R* Tp = ABp + pl.ab_elems;
  const dim3 grid((unsigned)(pl.n_split * pl.n_mblk));
#define LAUNCH(KM)                                                                              \
  em_sweep_kernel<R, KM><<<grid, TPB, 0, st>>>(G, (const R*)P, (const R*)Q, pl.M, pl.N, pl.K,   \
                                               pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, ABp, Tp)
  ADX_KMAX_SWITCH(pl.kmax, LAUNCH)
#undef LAUNCH
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

template <typename R>
static int launch_update_from(const EmPlan& pl, const R* ABp, const R* Tp, int mode, double* A, double* B,
                              double* T, const double* q_bat, double* P, double* Q, float* P32, float* Q32,
                              double* mP, double* vP, double* mQ, double* vQ, AdamArgs ad, cudaStream_t st) {
  const int threads = 128;
  const dim3 grid((unsigned)ceil_div(pl.M + pl.N, threads));
#define LAUNCH(KM)                                                                          \
  em_update_kernel<R, KM><<<grid, threads, 0, st>>>(ABp, Tp, pl.M, pl.N, pl.K, pl.n_split,  \
                                                    pl.n_mblk, mode, A, B, T, q_bat, P, Q,  \
                                                    P32, Q32, mP, vP, mQ, vQ, ad)
  ADX_KMAX_SWITCH(pl.kmax, LAUNCH)
#undef LAUNCH
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

template <typename R>
static int launch_update(const EmPlan& pl, void* ws, int mode, double* A, double* B, double* T,
                         const double* q_bat, double* P, double* Q, float* P32, float* Q32,
                         double* mP, double* vP, double* mQ, double* vQ, AdamArgs ad,
                         cudaStream_t st) {
  const R* ABp = reinterpret_cast<const R*>(reinterpret_cast<const uint8_t*>(ws) + EmPlan::HEADER);
  return launch_update_from<R>(pl, ABp, ABp + pl.ab_elems, mode, A, B, T, q_bat, P, Q, P32, Q32, mP, vP, mQ,
                               vQ, ad, st);
}

int em_sweep(const EmPlan& pl, const uint8_t* G, const void* P, const void* Q, void* ws,
             cudaStream_t st) {
  if (pl.prec == ADX_BF16 || pl.prec == ADX_F16) {
    float* ABp = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(ws) + EmPlan::HEADER);
    int* err = reinterpret_cast<int*>(ws);
    void* Qb = reinterpret_cast<uint8_t*>(ws) + pl.extra_offset();
    return tc_sweep(G, (const float*)P, (const float*)Q, pl.M, pl.N, pl.K, pl.n_stile, pl.n_split,
                    pl.n_mblk, ABp, ABp + pl.ab_elems, Qb, err, pl.prec == ADX_F16, st);
  }
  if (pl.prec == ADX_F64 && pl.K <= DMMA_MAX_K) {
    double* ABp = reinterpret_cast<double*>(reinterpret_cast<uint8_t*>(ws) + EmPlan::HEADER);
    return dmma_sweep(G, (const double*)P, (const double*)Q, pl.M, pl.N, pl.K, pl.n_stile, pl.n_split,
                      pl.n_mblk, pl.mb, ABp, ABp + pl.ab_elems, st);
  }
  return pl.prec == ADX_F64 ? launch_sweep<double>(pl, G, P, Q, ws, st)
                            : launch_sweep<float>(pl, G, P, Q, ws, st);
}

int em_update(const EmPlan& pl, void* ws, int mode, double* A, double* B, double* T,
              const double* q_bat, double* P, double* Q, float* P32, float* Q32, double* mP,
              double* vP, double* mQ, double* vQ, AdamArgs ad, cudaStream_t st) {
  return pl.prec == ADX_F64
             ? launch_update<double>(pl, ws, mode, A, B, T, q_bat, P, Q, P32, Q32, mP, vP, mQ, vQ, ad, st)
             : launch_update<float>(pl, ws, mode, A, B, T, q_bat, P, Q, P32, Q32, mP, vP, mQ, vQ, ad, st);
}

// Elementwise kernels for the unfused API (em_final_update and step as separate calls).
__global__ void em_targets_kernel(const double* __restrict__ P, const double* __restrict__ Q,
                                  const double* __restrict__ A, const double* __restrict__ B,
                                  const double* __restrict__ T, const double* __restrict__ q_bat,
                                  int64_t M, int64_t N, int K, double* __restrict__ P_EM,
                                  double* __restrict__ Q_EM) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row < M) {
    for (int k = 0; k < K; ++k) {
      const int64_t o = row * K + k;
      const double den = fmax((A[o] - B[o]) * P[o] + B[o], 1e-5);
      P_EM[o] = ((1.0 / den) * P[o]) * A[o];
    }
  } else if (row < M + N) {
    const int64_t i = row - M;
    const double scale = 1.0 / fmax(q_bat[i], 1e-5);
    double s = 0.0;
    for (int k = 0; k < K; ++k) s += (Q[i * K + k] * T[i * K + k]) * scale;
    s = fmax(s, 1e-5);
    for (int k = 0; k < K; ++k) Q_EM[i * K + k] = ((Q[i * K + k] * T[i * K + k]) * scale) / s;
  }
}

__global__ void adam_step_kernel(double* __restrict__ P, double* __restrict__ Q,
                                 const double* __restrict__ P_EM, const double* __restrict__ Q_EM,
                                 double* __restrict__ mP, double* __restrict__ vP,
                                 double* __restrict__ mQ, double* __restrict__ vQ, int64_t M,
                                 int64_t N, int K, AdamArgs ad, float* __restrict__ P32,
                                 float* __restrict__ Q32) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= M + N) return;
  const double t = adam_step_no(ad);
  const double bc1 = 1.0 - pow(ad.b1, t);
  const double bc2 = 1.0 - pow(ad.b2, t);
  const bool isP = row < M;
  const int64_t r = isP ? row : row - M;
  double* X = isP ? P : Q;
  const double* Xt = isP ? P_EM : Q_EM;
  double* m = isP ? mP : mQ;
  double* v = isP ? vP : vQ;
  float* X32 = isP ? P32 : Q32;
  double tot = 0.0;
  for (int k = 0; k < K; ++k) {
    const int64_t o = r * K + k;
    const double x = X[o];
    const double delta = Xt[o] - x;
    const double mm = m[o] * ad.b1 + (1.0 - ad.b1) * delta;
    const double vv = v[o] * ad.b2 + (1.0 - ad.b2) * (delta * delta);
    m[o] = mm;
    v[o] = vv;
    double nx = x + (ad.lr * (mm / bc1)) / (sqrt(vv / bc2) + ad.eps);
    nx = fmin(fmax(nx, DOMAIN), 1.0 - DOMAIN);
    X[o] = nx;
    tot += nx;
  }
  for (int k = 0; k < K; ++k) {
    const int64_t o = r * K + k;
    if (!isP) X[o] = X[o] / tot;
    if (X32) X32[o] = (float)X[o];
  }
}

}  // namespace adx

using namespace adx;

extern "C" int adx_em_workspace_bytes(int64_t M, int64_t N, int K, int precision, size_t* bytes) {
  if (!bytes) return ADX_ERR_ARG;
  EmPlan pl;
  const int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_workspace_bytes: bad shape or precision"); return rc; }
  *bytes = pl.bytes();
  return ADX_OK;
}

extern "C" int adx_em_status(void* workspace, size_t workspace_bytes, int64_t M, int64_t N, int K,
                             int precision, int* status, void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_status: bad shape or precision"); return rc; }
  if (!workspace || !status) { adx_set_message("adx_em_status: null pointer"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_status: workspace too small"); return ADX_ERR_WORKSPACE; }
  cudaStream_t st = as_stream(stream);
  int* word = reinterpret_cast<int*>(workspace);
  ADX_CUDA_TRY(cudaMemcpyAsync(status, word, sizeof(int), cudaMemcpyDeviceToHost, st));
  ADX_CUDA_TRY(cudaStreamSynchronize(st));
  ADX_CUDA_TRY(cudaMemsetAsync(word, 0, sizeof(int), st));
  return ADX_OK;
}

extern "C" int adx_em_stats(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                            const void* P, const void* Q, double* A, double* B, double* T,
                            void* workspace, size_t workspace_bytes, void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_stats: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !A || !B || !T || !workspace) { adx_set_message("adx_em_stats: null pointer"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_stats: workspace too small"); return ADX_ERR_WORKSPACE; }
  cudaStream_t st = as_stream(stream);
  rc = em_sweep(pl, G, P, Q, workspace, st);
  if (rc) return rc;
  return em_update(pl, workspace, 0, A, B, T, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                   nullptr, nullptr, nullptr, AdamArgs{1, 0, 0, 0, 0}, st);
}

extern "C" int adx_em_sweep(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                            const void* P, const void* Q, void* workspace, size_t workspace_bytes,
                            void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_sweep: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !workspace) { adx_set_message("adx_em_sweep: null pointer"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_sweep: workspace too small"); return ADX_ERR_WORKSPACE; }
  return em_sweep(pl, G, P, Q, workspace, as_stream(stream));
}

extern "C" int adx_em_targets(const double* P, const double* Q, const double* A, const double* B,
                              const double* T, const double* q_bat, int64_t M, int64_t N, int K,
                              double* P_EM, double* Q_EM, void* stream) {
  if (M <= 0 || N <= 0 || K < 1 || K > ADX_MAX_K) { adx_set_message("adx_em_targets: bad shape"); return ADX_ERR_ARG; }
  const int threads = 128;
  em_targets_kernel<<<(unsigned)ceil_div(M + N, threads), threads, 0, as_stream(stream)>>>(
      P, Q, A, B, T, q_bat, M, N, K, P_EM, Q_EM);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_adam_step(double* P, double* Q, const double* P_EM, const double* Q_EM,
                             double* mP, double* vP, double* mQ, double* vQ, int64_t M, int64_t N,
                             int K, double t, double lr, double beta1, double beta2, double eps,
                             float* P32, float* Q32, void* stream) {
  if (M <= 0 || N <= 0 || K < 1 || K > ADX_MAX_K || t < 1) { adx_set_message("adx_adam_step: bad arguments"); return ADX_ERR_ARG; }
  const int threads = 128;
  adam_step_kernel<<<(unsigned)ceil_div(M + N, threads), threads, 0, as_stream(stream)>>>(
      P, Q, P_EM, Q_EM, mP, vP, mQ, vQ, M, N, K, AdamArgs{t, lr, beta1, beta2, eps}, P32, Q32);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_em_adam_iteration(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                                     double* P, double* Q, float* P32, float* Q32, double* mP,
                                     double* vP, double* mQ, double* vQ, const double* q_bat,
                                     double t, double lr, double beta1, double beta2, double eps,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_adam_iteration: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !mP || !vP || !mQ || !vQ || !q_bat || !workspace || t < 1) {
    adx_set_message("adx_em_adam_iteration: bad arguments");
    return ADX_ERR_ARG;
  }
  if (precision != ADX_F64 && (!P32 || !Q32)) { adx_set_message("adx_em_adam_iteration: P32/Q32 required"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_adam_iteration: workspace too small"); return ADX_ERR_WORKSPACE; }
  cudaStream_t st = as_stream(stream);
  const void* Pin = precision == ADX_F64 ? (const void*)P : (const void*)P32;
  const void* Qin = precision == ADX_F64 ? (const void*)Q : (const void*)Q32;
  rc = em_sweep(pl, G, Pin, Qin, workspace, st);
  if (rc) return rc;
  return em_update(pl, workspace, 1, nullptr, nullptr, nullptr, q_bat, P, Q, P32, Q32, mP, vP, mQ,
                   vQ, AdamArgs{t, lr, beta1, beta2, eps}, st);
}

// ---------------------------------------------------------------- captured iterations
//
// n fused Adam-EM iterations (adx_em_adam_iteration) captured once into a CUDA graph and
// replayed with one launch: 2n kernel launches and their host-side cost become one graph
// launch, which matters when an iteration takes tens of microseconds (small cohorts). The
// Adam step of the replay's iteration i (1..n) is *step_counter + i; adx_em_graph_launch
// first sets the counter to the steps already taken, so a replay computes exactly the n
// eager iterations t0+1..t0+n. Pointers, shapes and the learning rate are fixed at capture;
// the caller keeps every buffer alive, at the same address, for the graph's lifetime.

namespace adx {
__global__ void set_counter_kernel(double* c, double v) { *c = v; }
}  // namespace adx

struct AdxEmGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double* counter = nullptr;
  int n = 0;
};

extern "C" int adx_em_graph_create(const uint8_t* G, int64_t M, int64_t N, int K, int precision, double* P,
                                   double* Q, float* P32, float* Q32, double* mP, double* vP, double* mQ,
                                   double* vQ, const double* q_bat, int n_iters, double lr, double beta1,
                                   double beta2, double eps, double* step_counter, void* workspace,
                                   size_t workspace_bytes, void** graph) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_graph_create: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !mP || !vP || !mQ || !vQ || !q_bat || !workspace || !step_counter || !graph ||
      n_iters < 1 || n_iters > 4096) {
    adx_set_message("adx_em_graph_create: bad arguments (1 <= n_iters <= 4096, non-null buffers)");
    return ADX_ERR_ARG;
  }
  if (precision != ADX_F64 && (!P32 || !Q32)) { adx_set_message("adx_em_graph_create: P32/Q32 required"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_graph_create: workspace too small"); return ADX_ERR_WORKSPACE; }
  *graph = nullptr;
  const void* Pin = precision == ADX_F64 ? (const void*)P : (const void*)P32;
  const void* Qin = precision == ADX_F64 ? (const void*)Q : (const void*)Q32;
  // capture on a private stream (the caller's may be the legacy default stream, which cannot
  // be captured); relaxed mode, so a kernel's first-use attribute setup may run inside
  cudaStream_t cs = nullptr;
  ADX_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  if (ce != cudaSuccess) {
    cudaStreamDestroy(cs);
    adx_set_cuda_error(ce);
    return ADX_ERR_CUDA;
  }
  for (int i = 1; i <= n_iters && !rc; ++i) {
    rc = em_sweep(pl, G, Pin, Qin, workspace, cs);
    if (!rc)
      rc = em_update(pl, workspace, 1, nullptr, nullptr, nullptr, q_bat, P, Q, P32, Q32, mP, vP, mQ, vQ,
                     AdamArgs{(double)i, lr, beta1, beta2, eps, step_counter}, cs);
  }
  cudaGraph_t g = nullptr;
  ce = cudaStreamEndCapture(cs, &g);
  cudaStreamDestroy(cs);
  if (rc || ce != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    if (!rc) {
      adx_set_cuda_error(ce != cudaSuccess ? ce : cudaErrorStreamCaptureInvalidated);
      rc = ADX_ERR_CUDA;
    }
    cudaGetLastError();
    return rc;
  }
  cudaGraphExec_t ex = nullptr;
  ce = cudaGraphInstantiate(&ex, g, 0ULL);
  if (ce != cudaSuccess) {
    cudaGraphDestroy(g);
    adx_set_cuda_error(ce);
    return ADX_ERR_CUDA;
  }
  *graph = new AdxEmGraph{g, ex, step_counter, n_iters};
  return ADX_OK;
}

extern "C" int adx_em_graph_launch(void* graph, double t0, void* stream) {
  auto* h = static_cast<AdxEmGraph*>(graph);
  if (!h || t0 < 0) { adx_set_message("adx_em_graph_launch: bad arguments"); return ADX_ERR_ARG; }
  cudaStream_t st = as_stream(stream);
  adx::set_counter_kernel<<<1, 1, 0, st>>>(h->counter, t0);
  ADX_LAUNCH_CHECK();
  ADX_CUDA_TRY(cudaGraphLaunch(h->exec, st));
  return ADX_OK;
}

extern "C" int adx_em_graph_iterations(void* graph, int* n_iters) {
  auto* h = static_cast<AdxEmGraph*>(graph);
  if (!h || !n_iters) { adx_set_message("adx_em_graph_iterations: bad arguments"); return ADX_ERR_ARG; }
  *n_iters = h->n;
  return ADX_OK;
}

extern "C" int adx_em_graph_destroy(void* graph) {
  auto* h = static_cast<AdxEmGraph*>(graph);
  if (!h) return ADX_OK;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  delete h;
  return ADX_OK;
}

// ---------------------------------------------------------------- sweep + log-likelihood
//
// The reference checks the log-likelihood of (P, Q) after an iteration's Adam move, and the
// next iteration's E-step sweeps the same (P, Q). adx_em_sweep_loglik is that sweep with the
// check folded in (float64, K <= 16): the same partials as adx_em_sweep plus the log-
// likelihood of its input, bit-identical to adx_loglik's float64 form; the optimiser reads
// it (adx_em_loglik_from_sweep), takes its decisions, then applies the move
// (adx_em_adam_update), so a check costs no pass of its own.

namespace adx {
// The partials' sum in the order adx_loglik's final sum uses (256 strided sums, then a tree),
// so the two log-likelihoods are bit-identical.
__global__ void ll_sum_kernel(const double* __restrict__ partial, int n, double* __restrict__ out) {
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
}  // namespace adx

static int ll_layout(const EmPlan& pl, void* ws, double** llp) {
  if (pl.prec != ADX_F64 || pl.K > DMMA_MAX_K) return ADX_ERR_UNSUPPORTED;
  *llp = reinterpret_cast<double*>(static_cast<uint8_t*>(ws) + pl.extra_offset());
  return ADX_OK;
}

extern "C" int adx_em_sweep_loglik(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
                                   const void* Q, void* workspace, size_t workspace_bytes, void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_sweep_loglik: bad shape or precision"); return rc; }
  if (!G || !P || !Q || !workspace) { adx_set_message("adx_em_sweep_loglik: null pointer"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_sweep_loglik: workspace too small"); return ADX_ERR_WORKSPACE; }
  double* llp = nullptr;
  if (ll_layout(pl, workspace, &llp)) {
    adx_set_message("adx_em_sweep_loglik: float64 with K <= 16 only");
    return ADX_ERR_UNSUPPORTED;
  }
  double* ABp = reinterpret_cast<double*>(static_cast<uint8_t*>(workspace) + EmPlan::HEADER);
  return dmma_sweep(G, (const double*)P, (const double*)Q, M, N, K, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, ABp,
                    ABp + pl.ab_elems, as_stream(stream), llp);
}

extern "C" int adx_em_loglik_from_sweep(void* workspace, size_t workspace_bytes, int64_t M, int64_t N, int K,
                                        int precision, double* out, void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_loglik_from_sweep: bad shape or precision"); return rc; }
  if (!workspace || !out) { adx_set_message("adx_em_loglik_from_sweep: null pointer"); return ADX_ERR_ARG; }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_loglik_from_sweep: workspace too small"); return ADX_ERR_WORKSPACE; }
  double* llp = nullptr;
  if (ll_layout(pl, workspace, &llp)) {
    adx_set_message("adx_em_loglik_from_sweep: float64 with K <= 16 only");
    return ADX_ERR_UNSUPPORTED;
  }
  ll_sum_kernel<<<1, 256, 0, as_stream(stream)>>>(llp, pl.n_split * pl.n_mblk, out);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

extern "C" int adx_em_adam_update(int64_t M, int64_t N, int K, int precision, double* P, double* Q, float* P32,
                                  float* Q32, double* mP, double* vP, double* mQ, double* vQ, const double* q_bat,
                                  double t, double lr, double beta1, double beta2, double eps, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_adam_update: bad shape or precision"); return rc; }
  if (!P || !Q || !mP || !vP || !mQ || !vQ || !q_bat || !workspace || t < 1) {
    adx_set_message("adx_em_adam_update: bad arguments");
    return ADX_ERR_ARG;
  }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_adam_update: workspace too small"); return ADX_ERR_WORKSPACE; }
  return em_update(pl, workspace, 1, nullptr, nullptr, nullptr, q_bat, P, Q, P32, Q32, mP, vP, mQ, vQ,
                   AdamArgs{t, lr, beta1, beta2, eps}, as_stream(stream));
}

// ---------------------------------------------------------------- block-range sweeps
//
// The float64 sweep (K <= 16) over a range of its SNP blocks, for callers that upload the
// packed matrix in pieces and sweep each piece as it lands: the partition is the full
// sweep's, each block's partial sums depend on that block alone, so the ranges of one
// workspace add up to exactly the full sweep.

extern "C" int adx_em_sweep_blocks_info(int64_t M, int64_t N, int K, int precision, int64_t* snps_per_block,
                                        int* n_blocks, int* ctas_per_block) {
  EmPlan pl;
  const int rc = em_plan(M, N, K, precision, pl);
  if (rc || !snps_per_block || !n_blocks || !ctas_per_block) { adx_set_message("adx_em_sweep_blocks_info: bad arguments"); return rc ? rc : ADX_ERR_ARG; }
  if (precision != ADX_F64 || K > DMMA_MAX_K) {
    adx_set_message("adx_em_sweep_blocks_info: float64 with K <= 16 only");
    return ADX_ERR_UNSUPPORTED;
  }
  *snps_per_block = pl.mb;
  *n_blocks = pl.n_mblk;
  *ctas_per_block = pl.n_split;
  return ADX_OK;
}

extern "C" int adx_em_sweep_blocks(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
                                   const void* Q, int b0, int b1, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  EmPlan pl;
  int rc = em_plan(M, N, K, precision, pl);
  if (rc) { adx_set_message("adx_em_sweep_blocks: bad shape or precision"); return rc; }
  if (precision != ADX_F64 || K > DMMA_MAX_K) {
    adx_set_message("adx_em_sweep_blocks: float64 with K <= 16 only");
    return ADX_ERR_UNSUPPORTED;
  }
  if (!G || !P || !Q || !workspace || b0 < 0 || b1 > pl.n_mblk || b0 >= b1) {
    adx_set_message("adx_em_sweep_blocks: bad arguments (0 <= b0 < b1 <= n_blocks)");
    return ADX_ERR_ARG;
  }
  if (workspace_bytes < pl.bytes()) { adx_set_message("adx_em_sweep_blocks: workspace too small"); return ADX_ERR_WORKSPACE; }
  double* ABp = reinterpret_cast<double*>(static_cast<uint8_t*>(workspace) + EmPlan::HEADER);
  return dmma_sweep(G, (const double*)P, (const double*)Q, M, N, K, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb, ABp,
                    ABp + pl.ab_elems, as_stream(stream), nullptr, b0, b1);
}

// The float64 log-likelihood on the float64 MMA (em_sweep_dmma.cu) uses the float64 sweep's
// partition; ADX_ERR_UNSUPPORTED when K > 16.
namespace adx {
int dmma_loglik_plan(int64_t M, int64_t N, int K, int64_t& n_stile, int& n_split, int& n_mblk, int64_t& mb) {
  if (K > DMMA_MAX_K) return ADX_ERR_UNSUPPORTED;
  EmPlan pl;
  const int rc = em_plan(M, N, K, ADX_F64, pl);
  if (rc) return rc;
  n_stile = pl.n_stile;
  n_split = pl.n_split;
  n_mblk = pl.n_mblk;
  mb = pl.mb;
  return ADX_OK;
}
}  // namespace adx

// ---------------------------------------------------------------- batched float64 E-step
//
// Several E-step problems on one cohort (K <= 16 each; e.g. the K sweep and its cross-
// validation folds) in one launch of the float64 tensor-core sweep. All of them share the
// float64 sweep's partition (it does not depend on K), so each problem's partial sums, and
// hence its statistics, are bit-identical to a single-problem sweep of the same P, Q and
// (fold-masked) genotypes. Workspace: a 256-byte header, then per problem its A/B partials
// and T partials, each 256-byte aligned.

namespace adx {
int dmma_sweep_batch(int64_t M, int64_t N, int n, const int* K, const uint8_t* const* G, const double* const* P,
                     const double* const* Q, double* const* ABp, double* const* Tp, int64_t n_stile, int n_split,
                     int n_mblk, int64_t mb, cudaStream_t st);
}

static int batch_layout(int64_t M, int64_t N, int n, const int* K, EmPlan& pl, size_t* offs, size_t* total) {
  if (n < 1 || n > 64 || !K) return ADX_ERR_ARG;
  for (int p = 0; p < n; ++p)
    if (K[p] < 1 || K[p] > DMMA_MAX_K) return ADX_ERR_ARG;
  const int rc = em_plan(M, N, K[0], ADX_F64, pl);
  if (rc) return rc;
  size_t off = EmPlan::HEADER;
  for (int p = 0; p < n; ++p) {
    if (offs) offs[p] = off;
    const size_t ab = (size_t)pl.n_split * (size_t)M * 2 * K[p], tt = (size_t)pl.n_mblk * (size_t)N * K[p];
    off = (off + (ab + tt) * sizeof(double) + 255) & ~size_t(255);
  }
  *total = off;
  return ADX_OK;
}

extern "C" int adx_em_batch_workspace_bytes(int64_t M, int64_t N, int n, const int* K, size_t* bytes) {
  EmPlan pl;
  if (!bytes) return ADX_ERR_ARG;
  const int rc = batch_layout(M, N, n, K, pl, nullptr, bytes);
  if (rc) adx_set_message("adx_em_batch_workspace_bytes: bad shape or K (1 <= n <= 64 problems, 1 <= K <= 16)");
  return rc;
}

extern "C" int adx_em_sweep_batch(int64_t M, int64_t N, int n, const int* K, const uint8_t* const* G,
                                  const double* const* P, const double* const* Q, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  EmPlan pl;
  size_t offs[64], total = 0;
  int rc = batch_layout(M, N, n, K, pl, offs, &total);
  if (rc || !G || !P || !Q || !workspace) {
    adx_set_message("adx_em_sweep_batch: bad argument (1 <= n <= 64 problems, 1 <= K <= 16)");
    return rc ? rc : ADX_ERR_ARG;
  }
  if (workspace_bytes < total) { adx_set_message("adx_em_sweep_batch: workspace too small"); return ADX_ERR_WORKSPACE; }
  double* ABp[64];
  double* Tp[64];
  for (int p = 0; p < n; ++p) {
    if (!G[p] || !P[p] || !Q[p]) { adx_set_message("adx_em_sweep_batch: null pointer"); return ADX_ERR_ARG; }
    ABp[p] = reinterpret_cast<double*>(static_cast<uint8_t*>(workspace) + offs[p]);
    Tp[p] = ABp[p] + (size_t)pl.n_split * (size_t)M * 2 * K[p];
  }
  return dmma_sweep_batch(M, N, n, K, G, P, Q, ABp, Tp, pl.n_stile, pl.n_split, pl.n_mblk, pl.mb,
                          as_stream(stream));
}

extern "C" int adx_em_batch_apply(int64_t M, int64_t N, int n, const int* K, int p, int mode, double* A, double* B,
                                  double* T, const double* q_bat, double* P, double* Q, double* mP, double* vP,
                                  double* mQ, double* vQ, double t, double lr, double beta1, double beta2,
                                  double eps, void* workspace, size_t workspace_bytes, void* stream) {
  EmPlan pl;
  size_t offs[64], total = 0;
  const int rc = batch_layout(M, N, n, K, pl, offs, &total);
  if (rc || p < 0 || p >= n || !workspace || (mode != 0 && mode != 1)) {
    adx_set_message("adx_em_batch_apply: bad argument");
    return rc ? rc : ADX_ERR_ARG;
  }
  if (workspace_bytes < total) { adx_set_message("adx_em_batch_apply: workspace too small"); return ADX_ERR_WORKSPACE; }
  if (mode == 0 ? (!A || !B || !T) : (!q_bat || !P || !Q || !mP || !vP || !mQ || !vQ || t < 1)) {
    adx_set_message("adx_em_batch_apply: bad argument");
    return ADX_ERR_ARG;
  }
  EmPlan pp;
  em_plan(M, N, K[p], ADX_F64, pp);
  const double* ABp = reinterpret_cast<const double*>(static_cast<const uint8_t*>(workspace) + offs[p]);
  const double* Tp = ABp + (size_t)pl.n_split * (size_t)M * 2 * K[p];
  return launch_update_from<double>(pp, ABp, Tp, mode, A, B, T, q_bat, P, Q, nullptr, nullptr, mP, vP, mQ, vQ,
                                    AdamArgs{t, lr, beta1, beta2, eps}, as_stream(stream));
}
