// Tensor-core (tcgen05, sm_100a) form of the E-step sweep: BF16 operands, FP32 accumulation
// in tensor memory. Same statistics and the same partial-sum layout as em_sweep_kernel
// (adamixture/model/em_adam_gpu.py:46-78), for 1 <= K <= 16 (K padded to 16 in the MMAs).
//
// Per CTA: R = 7 SNP tiles of 128 SNPs (896 SNPs) and a residue class of 128-sample tiles.
// For each step (sample tile s, SNP tile r), in two half-steps of 64 samples:
//   H  = P_r  . Q_s^T      (tcgen05.mma M=128 SNPs, N=64 samples, K=16)         -> TMEM
//   Hc = (1-P_r) . Q_s^T   (the complement, so 1-h stays accurate when h -> 1)  -> TMEM
//   8 warps read H/Hc rows from TMEM and form, per entry (one reciprocal each),
//     a = g / max(h,1e-5),  b = (2-g) / max(1-h,1e-5)   (0 where missing)
//   as BF16 tiles in shared memory; after both halves
//   A_r += a . Q_s, B_r += b . Q_s   (M=128 SNPs, N=16, K=128 samples; TMEM, all sample tiles)
//   T   += a^T . P_r + b^T . (1-P_r) (M=128 samples, N=16, K=128 SNPs; TMEM, all SNP tiles)
// After the R SNP tiles of a sample tile, T (over the CTA's 896 SNPs) goes to the T partials;
// after the last sample tile, A_r/B_r go to the A/B partials of the CTA's split.
//
// Warp specialisation (9 warps): warpgroup 0 (warps 0-3) forms the ratios of the first 64
// samples of every step, warpgroup 1 (warps 4-7) those of the second 64, and warp 8 is the
// producer: it issues every MMA from one thread and streams the G tiles into shared memory
// with cp.async. H/Hc live in two TMEM buffers (one per warpgroup) and the a/b tiles in two
// shared-memory buffers (one per step parity), so while a warpgroup forms the ratios of
// its half-step the tensor pipe runs the other warpgroup's H and the A/B/T MMAs of the
// previous step. Q tiles are triple-buffered. There is no block-wide barrier in the loop:
// the warps meet only at mbarriers.
//
// TMEM (512 columns, one CTA per SM): H/Hc buffer b at [128b, 128b+128) (H first 64, Hc
// last 64) | T [256,272) | A_r,B_r [272+32r, 304+32r) for r < 7.
// Shared-memory operands use the no-swizzle canonical layout (8-row x 16-byte core
// matrices). One copy of each tile serves both of its MMA views: P_r is the K-major A of H
// and the MN-major B of T; Q_s is the K-major B of H and the MN-major B of A/B; the a/b
// tiles are the K-major A of A/B and the MN-major A of T.
//
// Synchronisation (mbarriers): hfull[w] (tcgen05.commit: H of warpgroup w's next half-step
// and every MMA issued before it are done), abready[w] (128 arrivals: warpgroup w wrote its
// a/b half and finished reading its H buffer), gfull[b] (32 arrivals from cp.async: G tile
// buffer b is loaded). Every wait is bounded and also watches a shared abort word; on a
// timeout the kernel records ADX_ERR_TIMEOUT in the status word, all warps leave their
// loops, it waits (bounded) for its MMAs in flight, frees its TMEM and returns.
#include "common.cuh"

#include <cuda_bf16.h>

namespace adx {
namespace tc {

constexpr int TPB = 288;          // 2 consumer warpgroups + 1 producer warp
constexpr int PRODUCER_WARP = 8;
constexpr int TILE = 128;      // SNPs per SNP tile, samples per sample tile
constexpr int KP = 16;         // padded K
constexpr int R = 7;           // SNP tiles per CTA
constexpr int SNP_BLOCK = R * TILE;

// shared-memory map (bytes)
constexpr int P_TILE_BYTES = TILE * KP * 2;             // 4096
constexpr int OFF_P = 0;                                // R x (P, 1-P)
constexpr int OFF_Q = OFF_P + R * 2 * P_TILE_BYTES;     // 3 buffers
constexpr int OFF_G = OFF_Q + 3 * P_TILE_BYTES;         // 2 buffers x 32 rows x 128 bytes
constexpr int G_TILE_BYTES = (TILE / 4) * TILE;         // 4096
constexpr int OFF_A = OFF_G + 2 * G_TILE_BYTES;         // 2 buffers
constexpr int AB_TILE_BYTES = TILE * TILE * 2;          // 32768
constexpr int OFF_B = OFF_A + 2 * AB_TILE_BYTES;        // 2 buffers
constexpr int OFF_BAR = OFF_B + 2 * AB_TILE_BYTES;      // 6 mbarriers
constexpr int OFF_TMEM = OFF_BAR + 48;                  // TMEM address, then the abort word
constexpr int SMEM_BYTES = OFF_TMEM + 16;
constexpr int SMEM_ALLOC = SMEM_BYTES + 1024;           // room to align the base to 1024
static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory budget");

// TMEM columns
constexpr uint32_t COL_T = 256, COL_AB = 272;
constexpr int HALF = TILE / 2;                          // samples per half-step

constexpr uint32_t WAIT_LIMIT = 1u << 26;  // ~seconds of polling before giving up

// ---------------------------------------------------------------- descriptors

// Instruction descriptor, kind::f16: BF16 A/B, FP32 D, M = 128.
__host__ __device__ constexpr uint32_t idesc(int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}
constexpr uint32_t ID_H = idesc(HALF, 0, 0);   // A = P (K-major), B = Q half (K-major)
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

// Bounded wait; returns false on timeout or when another warp has aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (it > 64) __nanosleep(32);
  }
  *abort_flag = 1;
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// Arrive on `bar` once every cp.async this thread issued before has landed (the arrival
// counts against the barrier's expected count).
__device__ __forceinline__ void cp_async_arrive(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
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

// G tile (32 packed rows x 128 samples) into shared memory by the producer warp: lane l
// copies row l. Whole 16-byte chunks go by cp.async and the lane's arrival on `bar` fires
// when they land; rows that end past N, or a sample count that is not a multiple of 16,
// take byte loads and a plain arrival.
__device__ __forceinline__ void producer_load_g(const Args& a, int64_t row0, int64_t i0, bool vec16,
                                                uint8_t* gs, uint32_t bar) {
  const int l = threadIdx.x & 31;
  const int64_t row = row0 + l;
  const int64_t rows = (a.M + 3) >> 2;
  uint8_t* dst = gs + l * TILE;
  if (row < rows && vec16 && i0 + TILE <= a.N) {
    const uint8_t* src = a.G + row * a.N + i0;
#pragma unroll
    for (int c = 0; c < TILE / 16; ++c) cp_async16(smem_u32(dst + 16 * c), src + 16 * c);
    cp_async_arrive(bar);
  } else {
    for (int c = 0; c < TILE / 4; ++c) {
      uint32_t x = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int64_t ii = i0 + c * 4 + b;
        const uint32_t byte = (row < rows && ii < a.N) ? (uint32_t)__ldg(a.G + row * a.N + ii) : 0xFFu;
        x |= byte << (8 * b);
      }
      *reinterpret_cast<uint32_t*>(dst + 4 * c) = x;
    }
    mbar_arrive(bar);
  }
}

// Q tile (128 samples x 16, bf16) by the producer warp: lane l converts samples 4l..4l+3.
__device__ __forceinline__ void producer_load_q(const Args& a, int64_t i0, uint8_t* qs) {
  const int l = threadIdx.x & 31;
#pragma unroll 1
  for (int e = 0; e < 8; ++e) {
    const int row = l * 4 + (e >> 1), kh = (e & 1) * 8;
    const int64_t i = i0 + row;
    float f[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int k = kh + q;
      f[q] = (i < a.N && k < a.K) ? __ldg(a.Q + i * a.K + k) : 0.0f;
    }
    *reinterpret_cast<uint4*>(qs + off_pq(row, kh)) =
        make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]), pack_bf16x2(f[6], f[7]));
  }
}

__global__ void __launch_bounds__(TPB, 1) em_sweep_tc_kernel(Args a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(sm + OFF_TMEM);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + OFF_TMEM + 4);
  const uint32_t bars = smem_u32(sm + OFF_BAR);
  auto HFULL = [&](int w) { return bars + 8u * (uint32_t)w; };
  auto ABREADY = [&](int w) { return bars + 16u + 8u * (uint32_t)w; };
  auto GFULL = [&](int b) { return bars + 32u + 8u * (uint32_t)b; };
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int mblk = blockIdx.x % a.n_mblk;
  const int split = blockIdx.x / a.n_mblk;
  const int64_t jb = (int64_t)mblk * SNP_BLOCK;
  const int r_eff = (int)min((int64_t)R, (a.M - jb + TILE - 1) / TILE);
  const int64_t s_first = split;
  const int64_t n_my = (a.n_stile - split + a.n_split - 1) / a.n_split;  // sample tiles of this CTA
  const bool vec16 = (a.N & 15) == 0;
  const int64_t nsteps = n_my * r_eff;
  const int64_t nhalf = 2 * nsteps;

  // ---- prologue: TMEM (producer warp), barriers, P tiles (all threads)
  if (warp == PRODUCER_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_holder)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    *abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(HFULL(0)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(HFULL(1)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(ABREADY(0)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(ABREADY(1)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 32;" ::"r"(GFULL(0)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 32;" ::"r"(GFULL(1)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
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
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_holder;
  const uint32_t s_p = smem_u32(sm + OFF_P), s_q = smem_u32(sm + OFF_Q);
  const uint32_t s_a = smem_u32(sm + OFF_A), s_b = smem_u32(sm + OFF_B);
  const float ELO = (float)E_CLAMP;

  // H/Hc of half-step u (step u/2, half u&1) into TMEM buffer u&1
  auto issue_h = [&](int64_t u) {
    const int64_t st = u >> 1;
    const int r = (int)(st % r_eff);
    const int qb = (int)((st / r_eff) % 3);
    const int h = (int)(u & 1);
    const uint32_t pa = s_p + r * 2 * P_TILE_BYTES;
    const uint64_t bq = sdesc(s_q + qb * P_TILE_BYTES + h * (HALF / 8) * 256, 128, 256);
    const uint32_t col = (uint32_t)h * 128;
    mma_bf16(tmem + col, sdesc(pa, 128, 256), bq, ID_H, 0);
    mma_bf16(tmem + col + HALF, sdesc(pa + P_TILE_BYTES, 128, 256), bq, ID_H, 0);
  };
  // A/B/T MMAs of step st (a/b buffer st&1)
  auto issue_abt = [&](int64_t st) {
    const int64_t sidx = st / r_eff;
    const int r = (int)(st % r_eff);
    const uint32_t sq = s_q + (int)(sidx % 3) * P_TILE_BYTES;
    const uint32_t ta = s_a + (int)(st & 1) * AB_TILE_BYTES, tb = s_b + (int)(st & 1) * AB_TILE_BYTES;
    const uint32_t acc_ab = (sidx > 0) ? 1u : 0u;
#pragma unroll
    for (int ks = 0; ks < TILE / 16; ++ks) {
      const uint64_t bq = sdesc(sq + ks * 2 * 256, 256, 128);
      const uint32_t acc = (acc_ab | (ks > 0)) ? 1u : 0u;
      mma_bf16(tmem + COL_AB + 32 * r, sdesc(ta + ks * 2 * 128, 128, 2048), bq, ID_AB, acc);
      mma_bf16(tmem + COL_AB + 32 * r + 16, sdesc(tb + ks * 2 * 128, 128, 2048), bq, ID_AB, acc);
    }
    const uint32_t pa = s_p + r * 2 * P_TILE_BYTES;
#pragma unroll
    for (int ks = 0; ks < TILE / 16; ++ks) {
      const uint32_t acc = (r > 0 || ks > 0) ? 1u : 0u;
      mma_bf16(tmem + COL_T, sdesc(ta + ks * 2 * 2048, 2048, 128), sdesc(pa + ks * 2 * 256, 256, 128), ID_T, acc);
      mma_bf16(tmem + COL_T, sdesc(tb + ks * 2 * 2048, 2048, 128),
               sdesc(pa + P_TILE_BYTES + ks * 2 * 256, 256, 128), ID_T, 1u);
    }
  };
  auto write_t = [&](int64_t s) {  // one warpgroup: T rows (samples) of sample tile s
    uint32_t v[16];
    tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + COL_T, v);
    tmem_wait_ld();
    const int64_t i = s * TILE + (warp & 3) * 32 + lane;
    if (i < a.N) {
      float* dst = a.Tp + ((int64_t)mblk * a.N + i) * a.K;
#pragma unroll
      for (int k = 0; k < KP; ++k)
        if (k < a.K) dst[k] = __uint_as_float(v[k]);
    }
  };

  bool aborted = false;
  if (warp == PRODUCER_WARP) {
    // ---------------------------------------------------------------- producer
    producer_load_q(a, s_first * TILE, sm + OFF_Q);
    fence_async_smem();
    __syncwarp();
    producer_load_g(a, jb >> 2, s_first * TILE, vec16, sm + OFF_G, GFULL(0));
    if (lane == 0) {
      issue_h(0);
      mma_commit(HFULL(0));
      if (nhalf > 1) {
        issue_h(1);
        mma_commit(HFULL(1));
      }
    }
    __syncwarp();
    uint32_t pab0 = 0u, pab1 = 0u;
    for (int64_t u = 0; u < nhalf; ++u) {
      const int w = (int)(u & 1);
      const int64_t st = u >> 1;
      if (!mbar_wait(ABREADY(w), w ? pab1 : pab0, abort_flag)) { aborted = true; break; }
      if (w) pab1 ^= 1u; else pab0 ^= 1u;
      fence_after();
      // the next sample tile's Q must be in shared memory before its first H is issued
      const int64_t un = u + 2;
      if (un < nhalf && (un & 1) == 0 && ((un >> 1) % r_eff) == 0) {
        const int64_t nsidx = (un >> 1) / r_eff;
        producer_load_q(a, (s_first + nsidx * a.n_split) * TILE, sm + OFF_Q + (int)(nsidx % 3) * P_TILE_BYTES);
        fence_async_smem();
        __syncwarp();
      }
      if (lane == 0) {
        if (w == 1) issue_abt(st);
        if (un < nhalf) issue_h(un);
        mma_commit(HFULL(w));
      }
      __syncwarp();
      if (w == 0 && st + 1 < nsteps) {
        const int nr = (int)((st + 1) % r_eff);
        const int64_t ns = s_first + ((st + 1) / r_eff) * a.n_split;
        producer_load_g(a, (jb + (int64_t)nr * TILE) >> 2, ns * TILE, vec16,
                        sm + OFF_G + (int)((st + 1) & 1) * G_TILE_BYTES, GFULL((int)((st + 1) & 1)));
      }
    }
  } else {
    // ---------------------------------------------------------------- consumers
    const int w = warp >> 2;           // warpgroup = half of every step
    const int wq = warp & 3;           // TMEM lane quarter
    const int jl = wq * 32 + lane;     // SNP row within the tile
    const uint32_t trow = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)w * 128;
    const uint32_t sh = 2u * (uint32_t)(jl & 3);
    uint32_t ph = 0u;
    for (int64_t u = w; u < nhalf; u += 2) {
      const int64_t st = u >> 1;
      const int64_t sidx = st / r_eff;
      const int r = (int)(st % r_eff);
      const int64_t s = s_first + sidx * a.n_split;
      if (!mbar_wait(HFULL(w), ph, abort_flag)) { aborted = true; break; }
      ph ^= 1u;
      if (!mbar_wait(GFULL((int)(st & 1)), (uint32_t)((st >> 1) & 1), abort_flag)) { aborted = true; break; }
      fence_after();
      // T of the previous sample tile: its last T MMAs were committed before this H
      if (w == 1 && r == 0 && sidx > 0) write_t(s - a.n_split);

      const int64_t jglob = jb + (int64_t)r * TILE + jl;
      const uint8_t* gs = sm + OFF_G + (int)(st & 1) * G_TILE_BYTES + (jl >> 2) * TILE + w * HALF;
      uint8_t* ta = sm + OFF_A + (int)(st & 1) * AB_TILE_BYTES;
      uint8_t* tb = sm + OFF_B + (int)(st & 1) * AB_TILE_BYTES;
      uint32_t hv[2][16], cv[2][16];
      tmem_ld16(trow, hv[0]);
      tmem_ld16(trow + HALF, cv[0]);
      tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < HALF / 16; ++c) {
        const int cur = c & 1;
        if (c + 1 < HALF / 16) {
          tmem_ld16(trow + 16 * (c + 1), hv[cur ^ 1]);
          tmem_ld16(trow + HALF + 16 * (c + 1), cv[cur ^ 1]);
        }
        const int col0 = w * HALF + 16 * c;     // sample column inside the step's tile
        const uint4 gw = *reinterpret_cast<const uint4*>(gs + 16 * c);
        const uint32_t words[4] = {gw.x, gw.y, gw.z, gw.w};
        uint32_t ap[8], bp[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint32_t tq = (words[q] >> sh) & 0x03030303u;
          if (jglob >= a.M) tq = 0x03030303u;
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int e = q * 4 + half * 2;
            const uint32_t x = half ? (tq >> 16) : (tq & 0x0303u);
            const uint32_t sel = x * 0x22u + 0x1010u;
            const float rec0 = fmaxf(__uint_as_float(hv[cur][e]), ELO);
            const float rec1 = fmaxf(__uint_as_float(hv[cur][e + 1]), ELO);
            const float omr0 = fmaxf(__uint_as_float(cv[cur][e]), ELO);
            const float omr1 = fmaxf(__uint_as_float(cv[cur][e + 1]), ELO);
            const float r0 = rcp_approx(rec0 * omr0), r1 = rcp_approx(rec1 * omr1);
            const uint32_t ypair = pack_bf16x2(omr0 * r0, omr1 * r1);  // 1/rec
            const uint32_t xpair = pack_bf16x2(rec0 * r0, rec1 * r1);  // 1/(1-rec)
            ap[e >> 1] = mul_bf16x2(prmt(GA_LO, GA_HI, sel), ypair);
            bp[e >> 1] = mul_bf16x2(prmt(GB_LO, GB_HI, sel), xpair);
          }
        }
        *reinterpret_cast<uint4*>(ta + off_ab(jl, col0)) = make_uint4(ap[0], ap[1], ap[2], ap[3]);
        *reinterpret_cast<uint4*>(ta + off_ab(jl, col0 + 8)) = make_uint4(ap[4], ap[5], ap[6], ap[7]);
        *reinterpret_cast<uint4*>(tb + off_ab(jl, col0)) = make_uint4(bp[0], bp[1], bp[2], bp[3]);
        *reinterpret_cast<uint4*>(tb + off_ab(jl, col0 + 8)) = make_uint4(bp[4], bp[5], bp[6], bp[7]);
        tmem_wait_ld();
      }
      fence_async_smem();
      fence_before();
      mbar_arrive(ABREADY(w));
    }
  }

  // ---- epilogue: wait for the last MMAs (committed to HFULL(1) as completion nhalf/2)
  if (!aborted && nhalf > 0) {
    if (!mbar_wait(HFULL(1), (uint32_t)((nhalf >> 1) & 1), abort_flag)) aborted = true;
  }
  if (__syncthreads_or(aborted)) {
    if (tid == 0) atomicExch(a.err, ADX_ERR_TIMEOUT);
    if (warp == PRODUCER_WARP) {
      // MMAs may still be in flight: one more commit and bounded waits before freeing TMEM
      volatile int never = 0;
      if (lane == 0) mma_commit(HFULL(0));
      (void)mbar_wait(HFULL(0), 0u, &never);
      (void)mbar_wait(HFULL(0), 1u, &never);
    }
  } else {
    fence_after();
    if (warp >= 4 && warp < 8) write_t(s_first + (n_my - 1) * a.n_split);
    if (warp < 8) {
      // A/B of every SNP tile: warpgroup 0 reads A, warpgroup 1 reads B
      const int wg = warp >> 2, wq = warp & 3;
      for (int r = 0; r < r_eff; ++r) {
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
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == PRODUCER_WARP) {
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
