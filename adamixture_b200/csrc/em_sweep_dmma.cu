// Float64 E-step sweep on the float64 tensor-core MMA (sm_100a), K <= 16.
//
// The same statistics as em_sweep_kernel<double> (adamixture/model/em_adam_gpu.py:46-78):
//   h = P_j . Q_i,  rec = clamp(h, 1e-5, 1-1e-5),  a = g/rec,  b = (2-g)/(1-rec)  (0 if missing)
//   A_j = sum_i a Q_i,  B_j = sum_i b Q_i,  T_i = sum_j (a-b) P_j + sum_j b
// with the same partition into SNP blocks x sample splits and the same partial-sum layout
// (AB_part[split][j][2K], T_part[snp_block][i][K], float64), so em_update_kernel<double>
// reduces them unchanged. The CUDA-core form spends most of its issue slots folding the 2K
// A/B values of every SNP over the warp with shuffles; here the three contractions and h
// are float64 MMAs (mma.sync .f64: m16n8k4 for h, m16n8k8 -- 1024 FMAs a warp instruction
// -- for A, B and T) and the CUDA cores do only the per-entry ratios.
//
// CTA: 8 warps over a 256-sample sub-tile, 32 samples per warp, walking the block's SNPs in
// chunks of 16 (groups of 8 chunks staged in shared memory). (Two 4-warp CTAs per SM ran
// at the same speed with 4x the DRAM traffic: twice the A/B partial read-modify-writes,
// which no longer stayed in L2.) Per chunk a warp owns a 16-SNP
// x 32-sample tile as four 16 x 8 MMA tiles (fragment element: SNP row g or g+8, columns
// 2t, 2t+1; g = lane / 4, t = lane % 4). Column j of tile nt is local sample
// 8 (j / 2) + 2 nt + (j % 2), so a thread's 8 entries per SNP row are 8 consecutive
// samples (one 8-byte genotype load) and the 8 columns of a tile are one 8-sample k-step
// of the contraction over samples (k-slot t: column 2t, k-slot t + 4: column 2t + 1):
//   * H (16 x 8 per tile) = P_chunk (16 x K) . Q^T: ceil(K/4) k-steps of 4;
//   * the ratios a, b per entry; a and b, read straight from the H fragments, are the A
//     operands of A += a Q and B += b Q (16 SNPs x 8 K-columns per MMA, the tile's 8
//     samples per k-step; Q as the B operand);
//   * d = a - b goes through a per-warp shared-memory transpose (samples x SNPs) to become
//     the A operand of T += d^T P (16 samples x 8 K-columns, 8 SNPs per k-step); sum_j b
//     is added per thread and folded over the SNP lanes at the end.
// An m16n8k8 MMA gives the same float64 results, bit for bit, as the two m16n8k4 MMAs over
// the same k-slots that it replaced (measured), with half the MMA instructions.
// A and B of a chunk are summed over the CTA's warps in shared memory (fixed order, double
// buffered: one barrier per chunk) and added into the block's own AB_part rows; T lives in
// the MMA accumulators for the whole SNP block and is written once per sub-tile.
// Shared-memory layouts are chosen so that every fragment load and store is free of bank
// conflicts (row strides and column swizzles below).
#include <atomic>

#include "common.cuh"

namespace adx {
namespace dm {

constexpr int WARPS = 8;
constexpr int TPB = WARPS * 32;
constexpr int WS = 32;                 // samples per warp
constexpr int W = WARPS * WS;          // samples per sub-tile
constexpr int CH = 16;                 // SNPs per chunk
constexpr int GRP = 8;                 // chunks per staged P group
constexpr int GS = CH * GRP;           // SNPs per group
constexpr int QSTR = 24;               // Q tile row stride (doubles); column swizzle qsw()
constexpr int PSTR = 20;               // P tile row stride (doubles)
constexpr int DSTR = 20;               // transpose tile row stride (doubles); swizzle dsw()
constexpr int NV = 16;                 // A/B accumulator values per thread (2 x 2 tiles x 4)

// shared memory (doubles)
constexpr int Q_OFF = 0;
constexpr int P_OFF = Q_OFF + W * QSTR;
constexpr int D_OFF = P_OFF + GS * PSTR;
constexpr int R_OFF = D_OFF + WARPS * WS * DSTR;
constexpr int S_OFF = R_OFF + 2 * WARPS * NV * 32;
constexpr int SMEM_DOUBLES = S_OFF + WARPS * WS;
constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;

__device__ __forceinline__ int qsw(int r) { return ((r >> 3) & 3) << 2; }
__device__ __forceinline__ int dsw(int r) { return ((r >> 3) & 3) << 2; }

// Shared-memory layouts of the sweep ("tiles"). A layout decides only where the Q and P
// tiles and the A/B reduction values sit in shared memory, how many SNPs one P group
// stages, and how many CTAs share an SM -- never the arithmetic or its order, so every
// layout gives bit-identical statistics and partial sums.
//   0 (any K <= 16): Q rows of 24 doubles (16 columns, swizzled by Lay<0>::sw = qsw), P groups of 8
//     chunks in rows of 20, 16 A/B values a thread in the reduction buffers; 174 KiB, one
//     CTA per SM (up to 255 registers a thread).
//   1 (K <= 8): Q rows of 16 doubles (8 columns, swizzled by Lay<1>::sw), P groups of 4
//     chunks in rows of 12, 8 A/B values a thread; 112 KiB and at most 128 registers a
//     thread, so two CTAs share an SM.
// Both layouts' fragment loads and stores are checked exhaustively (every half-warp of every
// access pattern: in bounds, free of bank conflicts) by tests/test_dmma_layouts_cpu.py.
template <int TL> struct Lay;
template <> struct Lay<0> {
  static constexpr int QSTR = 24, QC = 16, PSTR = 20, PC = 16, GRP = 8, NV = 16, OCC = 1, KSMAX = 4;
  static __device__ __forceinline__ int sw(int r) { return ((r >> 3) & 3) << 2; }
};
template <> struct Lay<1> {
  static constexpr int QSTR = 16, QC = 8, PSTR = 12, PC = 8, GRP = 4, NV = 8, OCC = 2, KSMAX = 2;
  static __device__ __forceinline__ int sw(int r) { return (((r >> 3) & 3) << 2) ^ ((r & 1) << 3); }
};
// Offsets (doubles) of a layout's regions: Q tile, P group, transpose tiles, A/B reduction
// buffers (two), per-warp sums.
template <int TL> struct Off {
  using L = Lay<TL>;
  static constexpr int GS = CH * L::GRP;
  static constexpr int Q = 0;
  static constexpr int P = Q + W * L::QSTR;
  static constexpr int D = P + GS * L::PSTR;
  static constexpr int R = D + WARPS * WS * DSTR;
  static constexpr int S = R + 2 * WARPS * L::NV * 32;
  static constexpr int DOUBLES = S + WARPS * WS;
  static constexpr size_t BYTES = sizeof(double) * DOUBLES;
  static constexpr int RU = L::NV * 32 / TPB;   // A/B values a thread sums over the warps per chunk
  static constexpr int NVH = L::NV / 2;         // A values first, then B
  static_assert(NVH == 4 || NVH == 8, "one or two column tiles");
};
static_assert(Off<0>::BYTES == SMEM_BYTES, "layout 0 is the original map");
static_assert(2 * (Off<1>::BYTES + 1024) <= 228 * 1024, "two layout-1 CTAs fit in an SM's shared memory");
static_assert(Off<1>::RU * TPB == Lay<1>::NV * 32, "reduction values divide over the threads");

__device__ __forceinline__ void mma_f64_k8(double (&d)[4], double a0, double a1, double a2, double a3, double b0,
                                           double b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}
__device__ __forceinline__ void mma_f64(double (&d)[4], double a0, double a1, double b0) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a0), "d"(a1), "d"(b0));
}

// The genotype weight g and 2 - g (0 when missing) as doubles: the high words of 0, 1.0 and
// 2.0 picked from a 64-bit table by the 2-bit code (low word 0).
__device__ __forceinline__ double weight_a(uint32_t code) {
  const uint32_t hi = (uint32_t)(0x000040003FF00000ull >> (code << 4)) << 16;
  return __hiloint2double((int)hi, 0);
}
__device__ __forceinline__ double weight_b(uint32_t code) {
  const uint32_t hi = (uint32_t)(0x000000003FF04000ull >> (code << 4)) << 16;
  return __hiloint2double((int)hi, 0);
}

// The genotype bytes of SNP rows g and g+8 of the chunk at jc for the thread's 8 samples
// from s0 (0xFF, all missing, past N); rows past the matrix read its last row (those SNPs
// are masked as missing by the caller).
__device__ __forceinline__ void load_words(const uint8_t* __restrict__ G, int64_t N, int64_t rows, int64_t jc,
                                           int g, int64_t s0, bool full8, uint64_t (&w)[2]) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int64_t row = min(((jc + g + 8 * h) >> 2), rows - 1);
    const uint8_t* src = G + row * N + s0;
    if (full8) {
      w[h] = __ldg(reinterpret_cast<const unsigned long long*>(src));
    } else {
      uint64_t v = 0;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const uint64_t by = (s0 + u < N) ? (uint64_t)__ldg(src + u) : 0xFFull;
        v |= by << (8 * u);
      }
      w[h] = v;
    }
  }
}

struct Args {
  int64_t M, N;
  int64_t n_stile;
  int n_split, n_mblk;
  int64_t mb;
  double* llp;        // the sweep with the log-likelihood: one partial per CTA
  int mblk0 = 0;      // the launch covers SNP blocks [mblk0, mblk0 + nmb) (all: 0, n_mblk)
  int nmb = 0;
};

// Split x = m * 2^e with m in [0.5, 1): returns m, adds e to e.
__device__ __forceinline__ double renorm_dm(double x, int& e) {
  int hi = __double2hiint(x);
  const int lo = __double2loint(x);
  e += ((hi >> 20) & 0x7FF) - 1022;
  hi = (hi & 0x800FFFFF) | (1022 << 20);
  return __hiloint2double(hi, lo);
}

// The log-likelihood factor h^g (1-h)^(2-g) of 4 entries (1 when missing), h clamped to
// [1e-10, 1-1e-10], multiplied into the thread's running product.
__device__ __forceinline__ void ll_factors(const double (&hacc)[4], const uint64_t (&w)[2], int nt, double& prod,
                                           int& ex) {
  double f[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint32_t code = (uint32_t)(w[e >> 1] >> (8 * (2 * nt + (e & 1)))) & 3u;
    const double h = fmin(fmax(hacc[e], LL_CLAMP), 1.0 - LL_CLAMP);
    const double om = 1.0 - h;
    const double x = code == 2u ? h : om;
    const double y = code == 0u ? om : h;
    f[e] = code == 3u ? 1.0 : x * y;
  }
  prod *= (f[0] * f[1]) * (f[2] * f[3]);
  prod = renorm_dm(prod, ex);
}

// The CTA's log-likelihood partial: each thread's log(prod) + ex ln 2, summed over the warp
// by shuffles and over the warps in order.
__device__ __forceinline__ void ll_block_sum(double prod, int ex, double* wsum, double* out) {
  double acc = log(prod) + (double)ex * 0.69314718055994530942;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __syncthreads();
  if (lane == 0) wsum[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w2 = 0; w2 < WARPS; ++w2) s += wsum[w2];
    *out = s;
  }
}

// One E-step problem: its packed genotypes (cross-validation folds pass a copy with the
// fold's entries hidden), P [M][K] and Q [N][K] (float64), and its partial sums.
struct Prob {
  const uint8_t* G;
  const double* P;
  const double* Q;
  double* ABp;
  double* Tp;
  int K;
  int vec;            // 8-byte genotype loads allowed (N % 8 == 0, G 8-byte aligned)
};

template <int MAXP>
struct Probs {
  Prob p[MAXP];
  int n;
};

// KS: k-steps of 4 covering the problem's K (K <= 4 KS); NK = ceil(KS / 2) column tiles of
// 8. One (problem, sample sub-tile) of a CTA: the sub-tile's Q rows, then the CTA's SNP
// block in groups of 8 chunks of 16 SNPs, then the sub-tile's T partials.
// LL: also multiply every entry's log-likelihood factor into (prod, ex), in the order and
// arithmetic of loglik_dmma_kernel, so the CTA's partial equals that kernel's.
template <int KS, bool LL, int TL>
__device__ __forceinline__ void sweep_subtile(const Args& a, const Prob& pr, int64_t st, int split, int mblk,
                                              int& chunk_no, double* sm, double& prod, int& ex) {
  using L = Lay<TL>;
  using O = Off<TL>;
  static_assert(KS <= L::KSMAX, "the layout holds the K columns");
  constexpr int NK = (KS + 1) / 2;
  constexpr int QSTR = L::QSTR, PSTR = L::PSTR, GS = O::GS, NV = L::NV, RU = O::RU, NVH = O::NVH;
  double* qt = sm + O::Q;    // [W][QSTR]: Q rows of the sub-tile, columns swizzled by L::sw(row)
  double* pt = sm + O::P;    // [GS][PSTR]: P rows of the group
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  double* dT = sm + O::D + warp * WS * DSTR;  // [WS][DSTR]: d^T of the warp's tile
  double* sbuf = sm + O::S + warp * WS;
  const int64_t N = a.N, M = a.M;
  const int64_t j0 = (int64_t)mblk * a.mb;
  const int64_t j1 = min(M, j0 + a.mb);
  const int64_t rows = (M + 3) >> 2;
    const int K = pr.K;
    constexpr int ksp = KS, nkp = NK;
    const bool first = st == split;   // this CTA's first sub-tile: AB_part rows are written
    const int64_t i0 = st * W;
    // Q rows of the sub-tile (zero beyond N and K); the previous sub-tile's last reads of
    // qt and pt came before its last chunk barrier
    for (int e = threadIdx.x; e < W * L::QC; e += TPB) {
      const int r = e / L::QC, k = e % L::QC;
      const int64_t i = i0 + r;
      qt[r * QSTR + (k ^ L::sw(r))] = (i < N && k < K) ? pr.Q[i * K + k] : 0.0;
    }
    double tacc[2][NK][4];
    double sb[4][2];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int n = 0; n < NK; ++n)
#pragma unroll
        for (int e = 0; e < 4; ++e) tacc[m][n][e] = 0.0;
#pragma unroll
    for (int n = 0; n < 4; ++n) sb[n][0] = sb[n][1] = 0.0;

    // this thread's 8 consecutive samples; the first chunk's genotype words are loaded
    // here and each chunk loads the next one's, a chunk ahead of their use
    const int64_t s0 = i0 + warp * WS + 8 * t;
    const bool full8 = pr.vec && (s0 + 8 <= N);
    uint64_t wnext[2];
    load_words(pr.G, N, rows, j0, g, s0, full8, wnext);

    for (int64_t gj = j0; gj < j1; gj += GS) {
      const int gn = (int)min((int64_t)GS, j1 - gj);
      for (int e = threadIdx.x; e < GS * L::PC; e += TPB) {
        const int r = e / L::PC, k = e % L::PC;
        pt[r * PSTR + k] = (r < gn && k < K) ? pr.P[(gj + r) * K + k] : 0.0;
      }
      __syncthreads();
      const int nch = (gn + CH - 1) / CH;
      for (int ch = 0; ch < nch; ++ch) {
        const int64_t jc = gj + ch * CH;
        const double* pc = pt + ch * CH * PSTR;
        uint64_t w[2] = {wnext[0], wnext[1]};
        if (jc + CH < j1) load_words(pr.G, N, rows, jc + CH, g, s0, full8, wnext);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          // SNPs past the block end are missing (code 3)
          if (jc + g + 8 * h >= j1) w[h] |= 0x0303030303030303ull << (2 * (g & 3));
          w[h] >>= 2 * (g & 3);
        }
        // this thread's two A/B partial sums of the chunk, read now so that the read's
        // latency overlaps the chunk's arithmetic (added after the chunk barrier)
        double old_ab[RU];
#pragma unroll
        for (int u = 0; u < RU; ++u) old_ab[u] = 0.0;
        if (!first) {
#pragma unroll
          for (int u = 0; u < RU; ++u) {
            const int e = threadIdx.x + u * TPB;
            const int v = e >> 5, l = e & 31, n = (v >> 2) & (NVH / 4 - 1), el = v & 3;
            const int row = (l >> 2) + 8 * (el >> 1);
            const int col = 8 * n + 2 * (l & 3) + (el & 1);
            if (n < NK && col < K && jc + row < j1)
              old_ab[u] = pr.ABp[((int64_t)split * M + jc + row) * (2 * K) + (v < NVH ? col : K + col)];
          }
        }
        // P fragments: H's A operand (rows g, g+8; columns 4ks + t)
        double ph[KS][2];
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          ph[ks][0] = ks < ksp ? pc[g * PSTR + 4 * ks + t] : 0.0;
          ph[ks][1] = ks < ksp ? pc[(g + 8) * PSTR + 4 * ks + t] : 0.0;
        }
        double aacc[NK][4], bacc[NK][4];
#pragma unroll
        for (int n = 0; n < NK; ++n)
#pragma unroll
          for (int e = 0; e < 4; ++e) aacc[n][e] = bacc[n][e] = 0.0;

        // H of tile nt + 1 is issued before tile nt's ratios, so the MMAs' latency overlaps them.
        // k-steps 2s and 2s+1 of 4 run as one m16n8k8 (k-slots t and t + 4), an odd last one
        // as an m16n8k4: the same sums as KS k-steps of 4.
        auto h_tile = [&](double (&hacc)[4], int qrow_h) {
#pragma unroll
          for (int ks = 0; ks + 1 < KS; ks += 2)
            mma_f64_k8(hacc, ph[ks][0], ph[ks][1], ph[ks + 1][0], ph[ks + 1][1],
                       qt[qrow_h * QSTR + ((4 * ks + t) ^ L::sw(qrow_h))],
                       qt[qrow_h * QSTR + ((4 * ks + 4 + t) ^ L::sw(qrow_h))]);
          if constexpr (KS & 1)
            mma_f64(hacc, ph[KS - 1][0], ph[KS - 1][1], qt[qrow_h * QSTR + ((4 * (KS - 1) + t) ^ L::sw(qrow_h))]);
        };
        double hcur[4] = {0.0, 0.0, 0.0, 0.0}, hnext[4];
        h_tile(hcur, warp * WS + 8 * (g >> 1) + (g & 1));
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          if (nt < 3) {
            // H tile nt+1: column g of the B operand is local sample 8 (g / 2) + 2 (nt+1) + g % 2
            hnext[0] = hnext[1] = hnext[2] = hnext[3] = 0.0;
            h_tile(hnext, warp * WS + 8 * (g >> 1) + 2 * (nt + 1) + (g & 1));
          }
          const double (&hacc)[4] = hcur;
          if constexpr (LL) ll_factors(hacc, w, nt, prod, ex);
          double av[4], bv[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            // element e: SNP row g + 8 (e / 2), local sample 8t + 2nt + e % 2
            const uint32_t code = (uint32_t)(w[e >> 1] >> (8 * (2 * nt + (e & 1)))) & 3u;
            const double rec = fmin(fmax(hacc[e], E_CLAMP), 1.0 - E_CLAMP);
            const double omr = 1.0 - rec;
            // 1/rec and 1/(1-rec) from one reciprocal of x = rec (1 - rec) in [~1e-5, 0.25]:
            // the hardware approximation refined by two Newton-Raphson steps
            // r <- r (2 - x r), each squaring the relative error
            const double x = rec * omr;
            double r;
            asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
            r = fma(r, fma(-x, r, 1.0), r);
            r = fma(r, fma(-x, r, 1.0), r);
            av[e] = weight_a(code) * (omr * r);
            bv[e] = weight_b(code) * (rec * r);
            const int srow = 8 * t + 2 * nt + (e & 1);
            const int scol = g + 8 * (e >> 1);
            dT[srow * DSTR + (scol ^ dsw(srow))] = av[e] - bv[e];
          }
          sb[nt][0] += bv[0] + bv[2];
          sb[nt][1] += bv[1] + bv[3];
          // A += a Q, B += b Q, one 8-sample k-step: k-slot t is column 2t (sample 8t + 2nt),
          // k-slot t + 4 column 2t + 1 (sample 8t + 2nt + 1)
          {
            const int qrow0 = warp * WS + 8 * t + 2 * nt, qrow1 = qrow0 + 1;
#pragma unroll
            for (int n = 0; n < NK; ++n) {
              if (n >= nkp) continue;
              const double qb0 = qt[qrow0 * QSTR + ((8 * n + g) ^ L::sw(qrow0))];
              const double qb1 = qt[qrow1 * QSTR + ((8 * n + g) ^ L::sw(qrow1))];
              mma_f64_k8(aacc[n], av[0], av[2], av[1], av[3], qb0, qb1);
              mma_f64_k8(bacc[n], bv[0], bv[2], bv[1], bv[3], qb0, qb1);
            }
          }
          if (nt < 3) {
#pragma unroll
            for (int e = 0; e < 4; ++e) hcur[e] = hnext[e];
          }
        }
        __syncwarp();
        // T += d^T P: rows = local samples 16 m + g (+8), k-step q = SNPs 8q + t (k-slot t) and
        // 8q + t + 4 (k-slot t + 4)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          double pb0[NK], pb1[NK];
#pragma unroll
          for (int n = 0; n < NK; ++n) {
            pb0[n] = pc[(8 * q + t) * PSTR + 8 * n + g];
            pb1[n] = pc[(8 * q + t + 4) * PSTR + 8 * n + g];
          }
#pragma unroll
          for (int m = 0; m < 2; ++m) {
            const int r0 = 16 * m + g, r1 = r0 + 8;
            const double d0 = dT[r0 * DSTR + ((8 * q + t) ^ dsw(r0))];
            const double d1 = dT[r1 * DSTR + ((8 * q + t) ^ dsw(r1))];
            const double d2 = dT[r0 * DSTR + ((8 * q + t + 4) ^ dsw(r0))];
            const double d3 = dT[r1 * DSTR + ((8 * q + t + 4) ^ dsw(r1))];
#pragma unroll
            for (int n = 0; n < NK; ++n)
              if (n < nkp) mma_f64_k8(tacc[m][n], d0, d1, d2, d3, pb0[n], pb1[n]);
          }
        }
        // A/B of the chunk: this warp's share into the reduction buffer
        double* red = sm + O::R + (chunk_no & 1) * (WARPS * NV * 32);
#pragma unroll
        for (int n = 0; n < NK; ++n)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            red[(warp * NV + n * 4 + e) * 32 + lane] = aacc[n][e];
            red[(warp * NV + NVH + n * 4 + e) * 32 + lane] = bacc[n][e];
          }
        __syncthreads();
        // sum over the warps in a fixed order; value v of lane l is (A if v < NV/2 else B),
        // column tile (v / 4) mod (NV / 8), element v % 4 of lane l's fragment
#pragma unroll
        for (int u = 0; u < RU; ++u) {
          const int e = threadIdx.x + u * TPB;
          const int v = e >> 5, l = e & 31;
          const int n = (v >> 2) & (NVH / 4 - 1);
          if (n >= nkp) continue;
          const int el = v & 3;
          const int row = (l >> 2) + 8 * (el >> 1);
          const int col = 8 * n + 2 * (l & 3) + (el & 1);
          const int64_t j = jc + row;
          if (col >= K || j >= j1) continue;
          double s = 0.0;
#pragma unroll
          for (int ww = 0; ww < WARPS; ++ww) s += red[(ww * NV + v) * 32 + l];
          double* dst = pr.ABp + ((int64_t)split * M + j) * (2 * K) + (v < NVH ? col : K + col);
          *dst = first ? s : old_ab[u] + s;
        }
        ++chunk_no;
      }
      // the next group's P rows overwrite pt: every warp's T MMAs of this group are done
      // (they precede the last chunk barrier)
    }
    // sum_j b over the SNP rows (lanes with the same t), then T_part = T + sum_j b
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        double v = sb[nt][c];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        sb[nt][c] = v;
      }
    if (g == 0) {
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int c = 0; c < 2; ++c) sbuf[8 * t + 2 * nt + c] = sb[nt][c];
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int r = 16 * m + g + 8 * hh;
        const int64_t i = i0 + warp * WS + r;
        if (i >= N) continue;
        const double sbr = sbuf[r];
        double* dst = pr.Tp + ((int64_t)mblk * N + i) * K;
#pragma unroll
        for (int n = 0; n < NK; ++n)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const int col = 8 * n + 2 * t + c;
            if (col < K) dst[col] = tacc[m][n][2 * hh + c] + sbr;
          }
      }
    __syncwarp();
    // qt is rewritten at the next (sub-tile, problem)'s start: every warp's reads of it precede the
    // last chunk barrier, which all threads have passed
}

// A single problem (MAXP = 1, KS its own) or a batch of up to MAXP problems (each run by the
// instance of its own K). A CTA runs the problems in order, each over the CTA's whole share
// of the matrix (its SNP block x its sample sub-tiles), so consecutive problems on the same
// genotypes find the CTA's genotype region (about 0.3 MB at N=20k, M=100k) still in L2 and
// read it from memory once; a problem's arithmetic and summation order do not depend on the
// other problems.
// LL (single problem only): the sweep also sums the log-likelihood of its input (P, Q) into
// a.llp[blockIdx.x], bit-identical to loglik_dmma_kernel's partials.
// TL: the shared-memory layout (Lay<TL>); it sets how many CTAs share an SM.
template <int KS, int MAXP, bool LL, int TL>
__global__ void __launch_bounds__(TPB, Lay<TL>::OCC) em_sweep_dmma_kernel(Args a, Probs<MAXP> ps) {
  static_assert(!LL || MAXP == 1, "the log-likelihood rides on single-problem sweeps");
  extern __shared__ __align__(16) double sm[];
  const int mblk = a.mblk0 + (int)(blockIdx.x % a.nmb);
  const int split = blockIdx.x / a.nmb;
  int chunk_no = 0;   // parity of the A/B reduction buffer
  double prod = 1.0;
  int ex = 0;
  for (int pi = 0; pi < (MAXP == 1 ? 1 : ps.n); ++pi) {
    const Prob pr = ps.p[pi];
    for (int64_t st = split; st < a.n_stile; st += a.n_split) {
      if constexpr (MAXP == 1) {
        sweep_subtile<KS, LL, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex);
      } else if constexpr (Lay<TL>::KSMAX <= 2) {
        // the host launches this layout only for batches whose every K is <= 8
        if (((pr.K + 3) >> 2) == 1) sweep_subtile<1, false, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex);
        else sweep_subtile<2, false, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex);
      } else {
        switch ((pr.K + 3) >> 2) {
          case 1: sweep_subtile<1, false, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex); break;
          case 2: sweep_subtile<2, false, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex); break;
          case 3: sweep_subtile<3, false, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex); break;
          default: sweep_subtile<4, false, TL>(a, pr, st, split, mblk, chunk_no, sm, prod, ex); break;
        }
      }
    }
  }
  if constexpr (LL) ll_block_sum(prod, ex, sm + Off<TL>::S, a.llp + blockIdx.x);
}

// ---------------------------------------------------------------- float64 log-likelihood
//
// The log-likelihood of (P, Q) (adamixture/model/em_adam_gpu.py:226-279) with h on the same
// float64 MMA tiles as the sweep: L = sum over observed (j, i) of g log h + (2-g) log(1-h),
// h = clamp(P_j . Q_i, 1e-10, 1-1e-10). As in loglik_kernel, each thread multiplies the
// per-entry factors h^g (1-h)^(2-g) (the product x*y of two values picked by the genotype's
// two bits; 1 when missing) into one float64 running product, moves its exponent into an
// integer after every 4 factors (>= 1e-80 together, so the product stays normal), and takes
// one log at the end; per-CTA sums in a fixed order, per-CTA partials summed in block order.

// shared memory of the log-likelihood: the Q and P tiles and the warp sums (doubles)
constexpr int LL_SMEM_DOUBLES = P_OFF + GS * PSTR + WARPS;
constexpr size_t LL_SMEM_BYTES = sizeof(double) * LL_SMEM_DOUBLES;

template <int KS>
__global__ void __launch_bounds__(TPB, 2) loglik_dmma_kernel(Args a, const uint8_t* __restrict__ G,
                                                             const double* __restrict__ P,
                                                             const double* __restrict__ Q, int K, int vec,
                                                             double* __restrict__ partial) {
  extern __shared__ __align__(16) double sm[];
  double* qt = sm + Q_OFF;
  double* pt = sm + P_OFF;
  double* wsum = sm + P_OFF + GS * PSTR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int64_t N = a.N, M = a.M;
  const int mblk = blockIdx.x % a.n_mblk;
  const int split = blockIdx.x / a.n_mblk;
  const int64_t j0 = (int64_t)mblk * a.mb;
  const int64_t j1 = min(M, j0 + a.mb);
  const int64_t rows = (M + 3) >> 2;
  double prod = 1.0;
  int ex = 0;
  for (int64_t st = split; st < a.n_stile; st += a.n_split) {
    const int64_t i0 = st * W;
    __syncthreads();   // the previous sub-tile's reads of qt and pt are done
    for (int e = threadIdx.x; e < W * 16; e += TPB) {
      const int r = e >> 4, k = e & 15;
      const int64_t i = i0 + r;
      qt[r * QSTR + (k ^ qsw(r))] = (i < N && k < K) ? Q[i * K + k] : 0.0;
    }
    const int64_t s0 = i0 + warp * WS + 8 * t;
    const bool full8 = vec && (s0 + 8 <= N);
    uint64_t wnext[2];
    load_words(G, N, rows, j0, g, s0, full8, wnext);
    for (int64_t gj = j0; gj < j1; gj += GS) {
      const int gn = (int)min((int64_t)GS, j1 - gj);
      __syncthreads();
      for (int e = threadIdx.x; e < GS * 16; e += TPB) {
        const int r = e >> 4, k = e & 15;
        pt[r * PSTR + k] = (r < gn && k < K) ? P[(gj + r) * K + k] : 0.0;
      }
      __syncthreads();
      const int nch = (gn + CH - 1) / CH;
      for (int ch = 0; ch < nch; ++ch) {
        const int64_t jc = gj + ch * CH;
        const double* pc = pt + ch * CH * PSTR;
        uint64_t w[2] = {wnext[0], wnext[1]};
        if (jc + CH < j1) load_words(G, N, rows, jc + CH, g, s0, full8, wnext);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (jc + g + 8 * h >= j1) w[h] |= 0x0303030303030303ull << (2 * (g & 3));
          w[h] >>= 2 * (g & 3);
        }
        double ph[KS][2];
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          ph[ks][0] = pc[g * PSTR + 4 * ks + t];
          ph[ks][1] = pc[(g + 8) * PSTR + 4 * ks + t];
        }
        double hacc[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int qrow = warp * WS + 8 * (g >> 1) + 2 * nt + (g & 1);
          hacc[nt][0] = hacc[nt][1] = hacc[nt][2] = hacc[nt][3] = 0.0;
          // as in the sweep: k-step pairs on one m16n8k8, an odd last k-step on an m16n8k4
#pragma unroll
          for (int ks = 0; ks + 1 < KS; ks += 2)
            mma_f64_k8(hacc[nt], ph[ks][0], ph[ks][1], ph[ks + 1][0], ph[ks + 1][1],
                       qt[qrow * QSTR + ((4 * ks + t) ^ qsw(qrow))], qt[qrow * QSTR + ((4 * ks + 4 + t) ^ qsw(qrow))]);
          if constexpr (KS & 1)
            mma_f64(hacc[nt], ph[KS - 1][0], ph[KS - 1][1], qt[qrow * QSTR + ((4 * (KS - 1) + t) ^ qsw(qrow))]);
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) ll_factors(hacc[nt], w, nt, prod, ex);
      }
    }
  }
  ll_block_sum(prod, ex, wsum, partial + blockIdx.x);
}

}  // namespace dm

int dmma_plan_width() { return dm::W; }
int dmma_plan_chunk() { return dm::CH; }

template <int KS, int MAXP, bool LL, int TL>
static int dmma_launch(const dm::Args& a, const dm::Probs<MAXP>& ps, cudaStream_t st) {
  static bool attr_set[64] = {false};
  int dev = 0;
  ADX_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    ADX_CUDA_TRY(cudaFuncSetAttribute(dm::em_sweep_dmma_kernel<KS, MAXP, LL, TL>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dm::Off<TL>::BYTES));
    // all of the unified L1/shared storage as shared memory, so that OCC CTAs fit on an SM
    ADX_CUDA_TRY(cudaFuncSetAttribute(dm::em_sweep_dmma_kernel<KS, MAXP, LL, TL>,
                                      cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
    attr_set[dev] = true;
  }
  dm::em_sweep_dmma_kernel<KS, MAXP, LL, TL>
      <<<(unsigned)(a.n_split * a.nmb), dm::TPB, dm::Off<TL>::BYTES, st>>>(a, ps);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

// The layout each (device, K) launches its float64 sweeps with, set by adx_dmma_tile_set
// (the autotuner's choice) and read at every launch: 0 until set. Layouts never change
// the results, so a choice made while other threads launch only changes their speed.
constexpr int DMMA_TILE_DEVICES = 64;
static std::atomic<int> g_dmma_tile[DMMA_TILE_DEVICES][17];

int dmma_tile_count(int K) { return (K >= 1 && K <= 8) ? 2 : (K >= 9 && K <= 16) ? 1 : 0; }

static int dmma_tile_of(int K) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= DMMA_TILE_DEVICES || K < 1 || K > 16) return 0;
  const int tl = g_dmma_tile[dev][K].load(std::memory_order_relaxed);
  return tl < dmma_tile_count(K) ? tl : 0;
}

int dmma_tile_set(int device, int K, int tile) {
  if (device < 0 || device >= DMMA_TILE_DEVICES || K < 1 || K > 16 || tile < 0 || tile >= dmma_tile_count(K))
    return ADX_ERR_ARG;
  g_dmma_tile[device][K].store(tile, std::memory_order_relaxed);
  return ADX_OK;
}

int dmma_tile_get(int device, int K) {
  if (device < 0 || device >= DMMA_TILE_DEVICES || K < 1 || K > 16) return -1;
  return g_dmma_tile[device][K].load(std::memory_order_relaxed);
}

static int dmma_vec(const uint8_t* G, int64_t N) {
  return ((N & 7) == 0 && (reinterpret_cast<uintptr_t>(G) & 7) == 0) ? 1 : 0;
}

// llp != nullptr: the sweep also writes one log-likelihood partial of its input per CTA.
// Blocks [b0, b1) of the partition only (b1 <= 0: all of them); llp needs all blocks.
int dmma_sweep(const uint8_t* G, const double* P, const double* Q, int64_t M, int64_t N, int K,
               int64_t n_stile, int n_split, int n_mblk, int64_t mb, double* ABp, double* Tp,
               cudaStream_t st, double* llp, int b0, int b1) {
  if (K < 1 || K > 16) return ADX_ERR_UNSUPPORTED;
  if (b1 <= 0) { b0 = 0; b1 = n_mblk; }
  if (b0 < 0 || b1 > n_mblk || b0 >= b1 || (llp && (b0 != 0 || b1 != n_mblk))) return ADX_ERR_ARG;
  dm::Args a{M, N, n_stile, n_split, n_mblk, mb, llp};
  a.mblk0 = b0;
  a.nmb = b1 - b0;
  dm::Probs<1> ps;
  ps.p[0] = dm::Prob{G, P, Q, ABp, Tp, K, dmma_vec(G, N)};
  ps.n = 1;
  const int tl = dmma_tile_of(K);
#define ADX_DM_ONE(KS, TL) \
  return llp ? dmma_launch<KS, 1, true, TL>(a, ps, st) : dmma_launch<KS, 1, false, TL>(a, ps, st)
  switch ((K + 3) / 4) {
    case 1: if (tl == 1) { ADX_DM_ONE(1, 1); } ADX_DM_ONE(1, 0);
    case 2: if (tl == 1) { ADX_DM_ONE(2, 1); } ADX_DM_ONE(2, 0);
    case 3: ADX_DM_ONE(3, 0);
    default: ADX_DM_ONE(4, 0);
  }
#undef ADX_DM_ONE
}

constexpr int DMMA_MAX_PROBLEMS = 64;

// A batch launches with layout 1 when every problem's K has layout 1 selected, else 0.
int dmma_sweep_batch(int64_t M, int64_t N, int n, const int* K, const uint8_t* const* G, const double* const* P,
                     const double* const* Q, double* const* ABp, double* const* Tp, int64_t n_stile, int n_split,
                     int n_mblk, int64_t mb, cudaStream_t st) {
  if (n < 1 || n > DMMA_MAX_PROBLEMS) return ADX_ERR_ARG;
  dm::Args a{M, N, n_stile, n_split, n_mblk, mb, nullptr};
  a.nmb = n_mblk;
  dm::Probs<DMMA_MAX_PROBLEMS> ps;
  bool all1 = true;
  for (int p = 0; p < n; ++p) {
    if (K[p] < 1 || K[p] > 16 || !G[p]) return ADX_ERR_ARG;
    ps.p[p] = dm::Prob{G[p], P[p], Q[p], ABp[p], Tp[p], K[p], dmma_vec(G[p], N)};
    all1 = all1 && dmma_tile_of(K[p]) == 1;
  }
  ps.n = n;
  return all1 ? dmma_launch<2, DMMA_MAX_PROBLEMS, false, 1>(a, ps, st)
              : dmma_launch<4, DMMA_MAX_PROBLEMS, false, 0>(a, ps, st);
}

}  // namespace adx

namespace adx {

// Float64 log-likelihood on the float64 MMA for K <= 16: the float64 sweep's partition
// (n_split x n_mblk CTAs, at most 1776), one partial per CTA. Returns the partial count
// through *nblk (0 when this form does not apply).
int dmma_loglik_plan(int64_t M, int64_t N, int K, int64_t& n_stile, int& n_split, int& n_mblk, int64_t& mb);

int dmma_loglik(const uint8_t* G, const double* P, const double* Q, int64_t M, int64_t N, int K, double* partial,
                int* nblk, cudaStream_t st) {
  int64_t n_stile = 0, mb = 0;
  int n_split = 0, n_mblk = 0;
  int rc = dmma_loglik_plan(M, N, K, n_stile, n_split, n_mblk, mb);
  if (rc) return rc;
  *nblk = n_split * n_mblk;
  if (!partial) return ADX_OK;
  const dm::Args a{M, N, n_stile, n_split, n_mblk, mb, nullptr};
  const int vec = dmma_vec(G, N);
#define ADX_LL_DM(KS)                                                                                          \
  {                                                                                                            \
    static bool attr_set[64] = {false};                                                                        \
    int dev = 0;                                                                                               \
    ADX_CUDA_TRY(cudaGetDevice(&dev));                                                                         \
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {                                                              \
      ADX_CUDA_TRY(cudaFuncSetAttribute(dm::loglik_dmma_kernel<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                        (int)dm::LL_SMEM_BYTES));                                              \
      attr_set[dev] = true;                                                                                    \
    }                                                                                                          \
    dm::loglik_dmma_kernel<KS><<<(unsigned)(n_split * n_mblk), dm::TPB, dm::LL_SMEM_BYTES, st>>>(a, G, P, Q, K,  \
                                                                                              vec, partial);   \
  }
  switch ((K + 3) / 4) {
    case 1: ADX_LL_DM(1) break;
    case 2: ADX_LL_DM(2) break;
    case 3: ADX_LL_DM(3) break;
    default: ADX_LL_DM(4) break;
  }
#undef ADX_LL_DM
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

}  // namespace adx

// ---------------------------------------------------------------- tile choice (C ABI)

extern "C" int adx_dmma_tiles(int K, int* count) {
  if (!count || K < 1 || K > 16) { adx_set_message("adx_dmma_tiles: K must be in 1..16"); return ADX_ERR_ARG; }
  *count = adx::dmma_tile_count(K);
  return ADX_OK;
}

extern "C" int adx_dmma_tile_set(int device, int K, int tile) {
  const int rc = adx::dmma_tile_set(device, K, tile);
  if (rc) adx_set_message("adx_dmma_tile_set: device, K (1..16) or tile (< adx_dmma_tiles) out of range");
  return rc;
}

extern "C" int adx_dmma_tile_get(int device, int K, int* tile) {
  const int tl = tile ? adx::dmma_tile_get(device, K) : -1;
  if (tl < 0) { adx_set_message("adx_dmma_tile_get: device or K (1..16) out of range"); return ADX_ERR_ARG; }
  *tile = tl;
  return ADX_OK;
}
