// Tensor-core (tcgen05, sm_100a) form of the E-step sweep: BF16 operands, FP32 accumulation
// in tensor memory. Same statistics and the same partial-sum layout as em_sweep_kernel
// (adamixture/model/em_adam_gpu.py:46-78), for 1 <= K <= 16 (K padded to 16 in the MMAs).
//
// Per CTA: R = 7 SNP tiles of 128 SNPs (896 SNPs) and a residue class of 128-sample tiles.
// For each (sample tile s, SNP tile r):
//   H  = P_r  . Q_s^T      (tcgen05.mma M=128 SNPs, N=128 samples, K=16)       -> TMEM
//   Hc = (1-P_r) . Q_s^T   (the complement, so 1-h stays accurate when h -> 1)  -> TMEM
//   8 warps read H/Hc rows from TMEM and form, per entry (one reciprocal each),
//     a = g / max(h,1e-5),  b = (2-g) / max(1-h,1e-5)   (0 where missing)
//   as BF16 tiles in shared memory, then
//   A_r += a . Q_s, B_r += b . Q_s   (M=128 SNPs, N=16, K=128 samples; TMEM, all sample tiles)
//   T   += a^T . P_r + b^T . (1-P_r) (M=128 samples, N=16, K=128 SNPs; TMEM, all SNP tiles)
// After the R SNP tiles of a sample tile, T (over the CTA's 896 SNPs) goes to the T partials;
// after the last sample tile, A_r/B_r go to the A/B partials of the CTA's split.
//
// TMEM (512 columns, one CTA per SM): H [0,128) | Hc [128,256) | T [256,272) |
// A_r,B_r [272+32r, 304+32r) for r < 7.
// Shared-memory operands use the no-swizzle canonical layout (8-row x 16-byte core
// matrices). One copy of each tile serves both of its MMA views: P_r is the K-major A of H
// and the MN-major B of T; Q_s is the K-major B of H and the MN-major B of A/B; the a/b
// tiles are the K-major A of A/B and the MN-major A of T.
//
// Synchronisation: one mbarrier signalled by tcgen05.commit after each batch of MMAs. Every
// wait on it is bounded; the outcome is voted across the block (__syncthreads_or) so all
// threads leave together: on a timeout the kernel records ADX_ERR_TIMEOUT in the error word,
// waits (bounded) for its MMAs in flight, frees its TMEM and returns.
#include "common.cuh"

#include <cuda_bf16.h>

namespace adx {
namespace tc {

constexpr int TPB = 256;
constexpr int TILE = 128;      // SNPs per SNP tile, samples per sample tile
constexpr int KP = 16;         // padded K
constexpr int R = 7;           // SNP tiles per CTA
constexpr int SNP_BLOCK = R * TILE;

// shared-memory map (bytes)
constexpr int P_TILE_BYTES = TILE * KP * 2;             // 4096
constexpr int OFF_P = 0;                                // R x (P, 1-P)
constexpr int OFF_Q = OFF_P + R * 2 * P_TILE_BYTES;     // 2 buffers
constexpr int OFF_G = OFF_Q + 2 * P_TILE_BYTES;         // 2 buffers x 32 rows x 128 bytes
constexpr int G_TILE_BYTES = (TILE / 4) * TILE;         // 4096
constexpr int OFF_A = OFF_G + 2 * G_TILE_BYTES;
constexpr int AB_TILE_BYTES = TILE * TILE * 2;          // 32768
constexpr int OFF_B = OFF_A + AB_TILE_BYTES;
constexpr int OFF_BAR = OFF_B + AB_TILE_BYTES;
constexpr int OFF_TMEM = OFF_BAR + 16;
constexpr int SMEM_BYTES = OFF_TMEM + 16;
constexpr int SMEM_ALLOC = SMEM_BYTES + 1024;           // room to align the base to 1024

// TMEM columns
constexpr uint32_t COL_H = 0, COL_HC = 128, COL_T = 256, COL_AB = 272;

constexpr uint32_t WAIT_LIMIT = 1u << 26;  // ~seconds of polling before giving up

// ---------------------------------------------------------------- descriptors

// Instruction descriptor, kind::f16: BF16 A/B, FP32 D, M = 128.
__host__ __device__ constexpr uint32_t idesc(int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}
constexpr uint32_t ID_H = idesc(TILE, 0, 0);   // A = P (K-major), B = Q (K-major)
constexpr uint32_t ID_AB = idesc(KP, 0, 1);    // A = a (K-major), B = Q (MN-major)
constexpr uint32_t ID_T = idesc(KP, 1, 1);     // A = a^T (MN-major), B = P (MN-major)

// Shared-memory matrix descriptor, no swizzle, Blackwell version bit.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Byte offsets inside the tiles (element size 2).
// P / Q tiles: (row, k), rows of 8 form core matrices of 128 B; k halves 128 B apart.
__device__ __forceinline__ uint32_t off_pq(int row, int k) {
  return (uint32_t)((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
// a / b tiles: (snp j, sample i): sample groups of 8 are 128 B apart, SNP groups 2048 B.
__device__ __forceinline__ uint32_t off_ab(int j, int i) {
  return (uint32_t)((i >> 3) * 128 + (j >> 3) * 2048 + (j & 7) * 16 + (i & 7) * 2);
}

// ---------------------------------------------------------------- PTX wrappers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t id,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(ad), "l"(bd), "r"(id), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try(bar, parity)) return true;
    if (it > 64) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ uint32_t mul_bf16x2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
  return r;
}

// Genotype weights as BF16 pairs, looked up with one byte permute per pair:
// entry g (16 bits) at bytes 2g..2g+1 of {hi:lo}.
constexpr uint32_t GA_LO = 0x3F800000u, GA_HI = 0x00004000u;  // g -> {0, 1, 2, 0}
constexpr uint32_t GB_LO = 0x3F804000u, GB_HI = 0x00000000u;  // g -> {2, 1, 0, 0}

// ---------------------------------------------------------------- kernel

struct Args {
  const uint8_t* G;
  const float* P;     // [M][K] float32
  const float* Q;     // [N][K] float32
  int64_t M, N;
  int K;
  int64_t n_stile;    // sample tiles
  int n_split;
  int n_mblk;         // SNP blocks of 896
  float* ABp;         // [n_split][M][2K]
  float* Tp;          // [n_mblk][N][K]
  int* err;
};

__device__ __forceinline__ void load_g_regs(const Args& a, int64_t row0, int64_t i0, bool vec16,
                                            uint4& v) {
  // thread t covers packed row (t >> 3) and 16 samples starting at 16*(t & 7)
  const int t = threadIdx.x;
  const int64_t row = row0 + (t >> 3);
  const int64_t i = i0 + (int64_t)(t & 7) * 16;
  const int64_t rows = (a.M + 3) >> 2;
  if (row < rows && vec16 && i + 16 <= a.N) {
    v = __ldg(reinterpret_cast<const uint4*>(a.G + row * a.N + i));
  } else {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t x = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int64_t ii = i + q * 4 + b;
        const uint32_t byte = (row < rows && ii < a.N) ? (uint32_t)__ldg(a.G + row * a.N + ii) : 0xFFu;
        x |= byte << (8 * b);
      }
      w[q] = x;
    }
    v = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

__device__ __forceinline__ void store_g_smem(uint8_t* gs, const uint4& v) {
  const int t = threadIdx.x;
  *reinterpret_cast<uint4*>(gs + (t >> 3) * TILE + (t & 7) * 16) = v;
}

// Q tile: thread t -> sample (t >> 1), k half (t & 1); 8 values as one 16-byte chunk.
__device__ __forceinline__ void load_q_regs(const Args& a, int64_t i0, uint4& v) {
  const int t = threadIdx.x;
  const int64_t i = i0 + (t >> 1);
  const int kh = (t & 1) * 8;
  float f[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int k = kh + q;
    f[q] = (i < a.N && k < a.K) ? __ldg(a.Q + i * a.K + k) : 0.0f;
  }
  v = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                 pack_bf16x2(f[6], f[7]));
}
__device__ __forceinline__ void store_q_smem(uint8_t* qs, const uint4& v) {
  const int t = threadIdx.x;
  *reinterpret_cast<uint4*>(qs + off_pq(t >> 1, (t & 1) * 8)) = v;
}

__global__ void __launch_bounds__(TPB, 1) em_sweep_tc_kernel(Args a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(sm + OFF_TMEM);
  const uint32_t bar_a = smem_u32(bar);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wq = warp & 3;          // TMEM lane quarter
  const int wg = warp >> 2;         // warpgroup: sample half of a tile

  const int mblk = blockIdx.x % a.n_mblk;
  const int split = blockIdx.x / a.n_mblk;
  const int64_t jb = (int64_t)mblk * SNP_BLOCK;
  const int r_eff = (int)min((int64_t)R, (a.M - jb + TILE - 1) / TILE);
  const int64_t s_first = split;
  const int64_t n_my = (a.n_stile - split + a.n_split - 1) / a.n_split;  // sample tiles of this CTA
  const bool vec16 = (a.N & 15) == 0;

  // ---- TMEM allocation (warp 0), barrier init
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_holder)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  // ---- P tiles (bf16, P and 1-P) for the CTA's SNP tiles
  for (int e = tid; e < r_eff * TILE * 2; e += TPB) {
    const int r = e / (TILE * 2), row = (e / 2) % TILE, kh = (e & 1) * 8;
    const int64_t j = jb + (int64_t)r * TILE + row;
    float p[8], c[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = kh + q;
      const bool ok = j < a.M && k < a.K;
      const float v = ok ? __ldg(a.P + j * a.K + k) : 0.0f;
      p[q] = v;
      c[q] = ok ? 1.0f - v : 0.0f;
    }
    uint8_t* pt = sm + OFF_P + r * 2 * P_TILE_BYTES;
    *reinterpret_cast<uint4*>(pt + off_pq(row, kh)) =
        make_uint4(pack_bf16x2(p[0], p[1]), pack_bf16x2(p[2], p[3]), pack_bf16x2(p[4], p[5]), pack_bf16x2(p[6], p[7]));
    *reinterpret_cast<uint4*>(pt + P_TILE_BYTES + off_pq(row, kh)) =
        make_uint4(pack_bf16x2(c[0], c[1]), pack_bf16x2(c[2], c[3]), pack_bf16x2(c[4], c[5]), pack_bf16x2(c[6], c[7]));
  }
  // first Q tile and G tile
  {
    uint4 v;
    load_q_regs(a, s_first * TILE, v);
    store_q_smem(sm + OFF_Q, v);
    load_g_regs(a, jb >> 2, s_first * TILE, vec16, v);
    store_g_smem(sm + OFF_G, v);
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_holder;
  const uint32_t s_p = smem_u32(sm + OFF_P), s_q = smem_u32(sm + OFF_Q);
  const uint32_t s_a = smem_u32(sm + OFF_A), s_b = smem_u32(sm + OFF_B);

  auto issue_h = [&](int r, int qbuf) {
    const uint32_t pa = s_p + r * 2 * P_TILE_BYTES;
    const uint64_t bq = sdesc(s_q + qbuf * P_TILE_BYTES, 128, 256);
    mma_bf16(tmem + COL_H, sdesc(pa, 128, 256), bq, ID_H, 0);
    mma_bf16(tmem + COL_HC, sdesc(pa + P_TILE_BYTES, 128, 256), bq, ID_H, 0);
  };
  if (tid == 0) {
    issue_h(0, 0);
    mma_commit(bar_a);
  }

  uint32_t phase = 0;
  bool aborted = false;
  const int64_t nsteps = n_my * r_eff;
  const float ELO = (float)E_CLAMP;
  const int jl = wq * 32 + lane;  // SNP row of this thread within the tile

  for (int64_t step = 0; step < nsteps; ++step) {
    const int64_t sidx = step / r_eff;      // index of the sample tile among this CTA's
    const int r = (int)(step % r_eff);
    const int64_t s = s_first + sidx * a.n_split;
    const int qbuf = (int)(sidx & 1), gbuf = (int)(step & 1);
    const bool ok = mbar_wait(bar_a, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) { aborted = true; break; }
    fence_after();

    // T of the previous sample tile is complete: write its partial
    if (r == 0 && sidx > 0 && wg == 0) {
      uint32_t v[16];
      tmem_ld16(tmem + ((uint32_t)(wq * 32) << 16) + COL_T, v);
      tmem_wait_ld();
      const int64_t i = (s - a.n_split) * TILE + wq * 32 + lane;
      if (i < a.N) {
        float* dst = a.Tp + ((int64_t)mblk * a.N + i) * a.K;
        #pragma unroll
        for (int k = 0; k < KP; ++k)
          if (k < a.K) dst[k] = __uint_as_float(v[k]);
      }
    }
    // prefetch the next step's G (and Q) tile into registers
    const bool has_next = step + 1 < nsteps;
    const int64_t nsidx = (step + 1) / r_eff;
    const int nr = (int)((step + 1) % r_eff);
    const int64_t ns = s_first + nsidx * a.n_split;
    uint4 gnext = make_uint4(0, 0, 0, 0), qnext = make_uint4(0, 0, 0, 0);
    if (has_next) {
      load_g_regs(a, (jb + (int64_t)nr * TILE) >> 2, ns * TILE, vec16, gnext);
      if (nr == 0) load_q_regs(a, ns * TILE, qnext);
    }

    // ---- ratios for SNP row jl, samples [64*wg, 64*wg + 64)
    {
      const int64_t jglob = jb + (int64_t)r * TILE + jl;
      const uint32_t sh = 2u * (uint32_t)(jl & 3);
      const uint8_t* gs = sm + OFF_G + gbuf * G_TILE_BYTES + (jl >> 2) * TILE;
      const uint32_t trow = tmem + ((uint32_t)(wq * 32) << 16);
#pragma unroll 1
      for (int c = 0; c < 4; ++c) {
        const int col0 = wg * 64 + c * 16;
        uint32_t hv[16], cv[16];
        tmem_ld16(trow + COL_H + col0, hv);
        tmem_ld16(trow + COL_HC + col0, cv);
        const uint4 gw = *reinterpret_cast<const uint4*>(gs + col0);
        tmem_wait_ld();
        uint32_t words[4] = {gw.x, gw.y, gw.z, gw.w};
        uint32_t ap[8], bp[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint32_t tq = (words[q] >> sh) & 0x03030303u;
          if (jglob >= a.M) tq = 0x03030303u;
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int u = q * 4 + half * 2;
            const uint32_t x = half ? (tq >> 16) : (tq & 0x0303u);
            const uint32_t sel = x * 0x22u + 0x1010u;
            const float h0 = __uint_as_float(hv[u]), h1 = __uint_as_float(hv[u + 1]);
            const float c0 = __uint_as_float(cv[u]), c1 = __uint_as_float(cv[u + 1]);
            const float rec0 = fmaxf(h0, ELO), rec1 = fmaxf(h1, ELO);
            const float omr0 = fmaxf(c0, ELO), omr1 = fmaxf(c1, ELO);
            const float r0 = rcp_approx(rec0 * omr0), r1 = rcp_approx(rec1 * omr1);
            const uint32_t ypair = pack_bf16x2(omr0 * r0, omr1 * r1);  // 1/rec
            const uint32_t xpair = pack_bf16x2(rec0 * r0, rec1 * r1);  // 1/(1-rec)
            ap[u >> 1] = mul_bf16x2(prmt(GA_LO, GA_HI, sel), ypair);
            bp[u >> 1] = mul_bf16x2(prmt(GB_LO, GB_HI, sel), xpair);
          }
        }
        *reinterpret_cast<uint4*>(sm + OFF_A + off_ab(jl, col0)) = make_uint4(ap[0], ap[1], ap[2], ap[3]);
        *reinterpret_cast<uint4*>(sm + OFF_A + off_ab(jl, col0 + 8)) = make_uint4(ap[4], ap[5], ap[6], ap[7]);
        *reinterpret_cast<uint4*>(sm + OFF_B + off_ab(jl, col0)) = make_uint4(bp[0], bp[1], bp[2], bp[3]);
        *reinterpret_cast<uint4*>(sm + OFF_B + off_ab(jl, col0 + 8)) = make_uint4(bp[4], bp[5], bp[6], bp[7]);
      }
    }
    if (has_next) {
      store_g_smem(sm + OFF_G + (gbuf ^ 1) * G_TILE_BYTES, gnext);
      if (nr == 0) store_q_smem(sm + OFF_Q + (qbuf ^ 1) * P_TILE_BYTES, qnext);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();

    if (tid == 0) {
      // A_r += a . Q_s, B_r += b . Q_s  (K = 128 samples in 8 steps of 16)
      const uint32_t acc_ab = (sidx > 0) ? 1u : 0u;
      const uint32_t sq = s_q + qbuf * P_TILE_BYTES;
#pragma unroll
      for (int ks = 0; ks < TILE / 16; ++ks) {
        const uint64_t bq = sdesc(sq + ks * 2 * 256, 256, 128);
        const uint32_t acc = (acc_ab | (ks > 0)) ? 1u : 0u;
        mma_bf16(tmem + COL_AB + 32 * r, sdesc(s_a + ks * 2 * 128, 128, 2048), bq, ID_AB, acc);
        mma_bf16(tmem + COL_AB + 32 * r + 16, sdesc(s_b + ks * 2 * 128, 128, 2048), bq, ID_AB, acc);
      }
      // T += a^T . P_r + b^T . (1 - P_r)  (K = 128 SNPs in 8 steps of 16)
      const uint32_t pa = s_p + r * 2 * P_TILE_BYTES;
#pragma unroll
      for (int ks = 0; ks < TILE / 16; ++ks) {
        const uint32_t acc = (r > 0 || ks > 0) ? 1u : 0u;
        mma_bf16(tmem + COL_T, sdesc(s_a + ks * 2 * 2048, 2048, 128), sdesc(pa + ks * 2 * 256, 256, 128), ID_T, acc);
        mma_bf16(tmem + COL_T, sdesc(s_b + ks * 2 * 2048, 2048, 128),
                 sdesc(pa + P_TILE_BYTES + ks * 2 * 256, 256, 128), ID_T, 1u);
      }
      if (has_next) issue_h(nr, (int)(nsidx & 1));
      mma_commit(bar_a);
    }
  }

  if (!aborted) {
    const bool ok = mbar_wait(bar_a, phase);
    if (__syncthreads_or(!ok)) {
      aborted = true;
    } else {
      fence_after();
      // T of the last sample tile
      if (nsteps > 0 && wg == 0) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(wq * 32) << 16) + COL_T, v);
        tmem_wait_ld();
        const int64_t s_last = s_first + (n_my - 1) * a.n_split;
        const int64_t i = s_last * TILE + wq * 32 + lane;
        if (i < a.N) {
          float* dst = a.Tp + ((int64_t)mblk * a.N + i) * a.K;
          #pragma unroll
          for (int k = 0; k < KP; ++k)
            if (k < a.K) dst[k] = __uint_as_float(v[k]);
        }
      }
      // A/B of every SNP tile: warpgroup 0 reads A, warpgroup 1 reads B
      for (int r = 0; r < r_eff && nsteps > 0; ++r) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(wq * 32) << 16) + COL_AB + 32 * r + 16 * wg, v);
        tmem_wait_ld();
        const int64_t j = jb + (int64_t)r * TILE + wq * 32 + lane;
        if (j < a.M) {
          float* dst = a.ABp + ((int64_t)split * a.M + j) * (2 * a.K) + wg * a.K;
          #pragma unroll
          for (int k = 0; k < KP; ++k)
            if (k < a.K) dst[k] = __uint_as_float(v[k]);
        }
      }
    }
  }
  if (aborted) {
    if (tid == 0) atomicExch(a.err, ADX_ERR_TIMEOUT);
    // MMAs may still be in flight: one more commit and a bounded wait before freeing TMEM
    if (tid == 0) mma_commit(bar_a);
    (void)mbar_wait(bar_a, phase);
    (void)mbar_wait(bar_a, phase ^ 1u);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
  }
}

}  // namespace tc

int tc_plan(int64_t M, int64_t N, int K, int64_t& n_stile, int& n_split, int& n_mblk) {
  if (M <= 0 || N <= 0 || K < 1 || K > tc::KP) return ADX_ERR_UNSUPPORTED;
  n_stile = ceil_div(N, tc::TILE);
  n_mblk = (int)ceil_div(M, tc::SNP_BLOCK);
  // about 8 waves of one CTA per SM (148 SMs), so the last wave is a small fraction
  int64_t sp = ceil_div(8 * 148, n_mblk);
  sp = sp < 1 ? 1 : (sp > n_stile ? n_stile : sp);
  n_split = (int)sp;
  return ADX_OK;
}

int tc_sweep(const uint8_t* G, const float* P, const float* Q, int64_t M, int64_t N, int K,
             int64_t n_stile, int n_split, int n_mblk, float* ABp, float* Tp, int* err,
             cudaStream_t st) {
  static bool attr_set[64] = {false};
  int dev = 0;
  ADX_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    ADX_CUDA_TRY(cudaFuncSetAttribute(tc::em_sweep_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      tc::SMEM_ALLOC));
    attr_set[dev] = true;
  }
  tc::Args a{G, P, Q, M, N, K, n_stile, n_split, n_mblk, ABp, Tp, err};
  tc::em_sweep_tc_kernel<<<(unsigned)(n_split * n_mblk), tc::TPB, tc::SMEM_ALLOC, st>>>(a);
  ADX_LAUNCH_CHECK();
  return ADX_OK;
}

}  // namespace adx
