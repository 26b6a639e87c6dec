/*
 * adamixture_b200: C ABI of the B200 (sm_100a) kernels for the ADMIXTURE Adam-EM hot path.
 *
 * Conventions
 *  - Every pointer argument except host scalars is DEVICE memory; sizes are element counts.
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy default stream.
 *    Every launch goes on `stream`; no call synchronises the device.
 *  - Every entry point returns ADX_OK (0) or an ADX_ERR_* code; adx_last_error() returns a
 *    message for the last failure on the calling host thread.
 *  - Packed genotypes: uint8 G[ceil(M/4)][N], byte (j>>2)*N + i holds SNP j of sample i in
 *    bits 2*(j&3); 0/1/2 = allele count, 3 = missing; unused bits of the last row are 0.
 *    (The reference's GPU layout, adamixture/src/utils_c/cython/snp_reader.pyx:76-120.)
 *  - P is [M][K], Q is [N][K], row-major. "precision" selects the E-step arithmetic:
 *    ADX_F64 (float64, the reference GPU path's precision), ADX_F32, and the tcgen05
 *    tensor-core form with FP32 accumulation (K <= 16) and BF16 (ADX_BF16) or FP16
 *    (ADX_F16: power-of-two-scaled operands, 8x finer rounding than BF16) operands. P/Q
 *    passed to a pass are double for ADX_F64 and float otherwise.
 *  - Calls that need scratch memory take a caller-allocated `workspace` whose size
 *    adx_*_workspace_bytes() reports; none of them allocates device memory.
 */
#ifndef ADAMIXTURE_B200_H
#define ADAMIXTURE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ADX_OK = 0,
  ADX_ERR_ARG = 1,          /* invalid size, K or pointer */
  ADX_ERR_CUDA = 2,         /* a CUDA runtime call or launch failed */
  ADX_ERR_WORKSPACE = 3,    /* workspace smaller than adx_*_workspace_bytes() */
  ADX_ERR_UNSUPPORTED = 4,  /* precision/K combination not built */
  ADX_ERR_TIMEOUT = 5,      /* a bounded in-kernel wait gave up (reported by adx_em_status) */
};

enum { ADX_F64 = 0, ADX_F32 = 1, ADX_BF16 = 2, ADX_F16 = 3 };

/* Largest K the kernels accept (the reference's GPU limit, adamixture/entry.py:299-303). */
#define ADX_MAX_K 64

const char* adx_version(void);
const char* adx_last_error(void);

/* ---------------------------------------------------------------- genotype layout */

/* Decode SNP rows [m_start, m_start+count) into out[count][N] (uint8, 3 = missing).
 * G holds packed rows starting at packed row `byte_offset` (a host-streamed slice) and
 * has `rows` packed rows. Replaces torch.ops.pack2bit.unpack2bit_gpu_chunk_uint8
 * (adamixture/src/utils_c/cuda/pack2bit.cu:15-44, 83-111, 147-160). */
int adx_unpack_u8(const uint8_t* G, int64_t rows, int64_t N, int64_t M_total, int64_t m_start,
                  int64_t count, int64_t byte_offset, uint8_t* out, void* stream);

/* Same rows decoded and centred: out = g - 2 f_j, 0 where missing (float32).
 * Replaces torch.ops.pack2bit.unpack2bit_gpu_chunk_center (pack2bit.cu:46-77, 114-141). */
int adx_unpack_center_f32(const uint8_t* G, int64_t rows, int64_t N, int64_t M_total,
                          int64_t m_start, int64_t count, int64_t byte_offset, const float* f,
                          float* out, void* stream);

/* f_j = sum_i g_ij / (2 * #observed_j), 0 when none observed (float32).
 * Replaces calculate_frequencies_gpu (adamixture/src/utils.py:781-861). */
int adx_allele_frequency(const uint8_t* G, int64_t M, int64_t N, float* f, void* stream);

/* q_bat_i = 2 * #observed SNPs of sample i (float64): the per-sample count that the
 * reference re-accumulates on every E-step (adamixture/model/em_adam_gpu.py:76, 196). */
int adx_sample_counts(const uint8_t* G, int64_t M, int64_t N, double* q_bat, void* stream);
/* Heterozygous (g = 1) genotype count per sample, float64 [N] (exact integers); with
 * adx_sample_counts it gives the warm-start network's heterozygosity feature. No
 * counterpart in the reference. */
int adx_sample_het_counts(const uint8_t* G, int64_t M, int64_t N, double* het, void* stream);

/* PLINK BED rows bed[M][ceil(N/4)] (SNP-major, LUT [2,3,1,0]) -> packed G, then the
 * reference's 0<->2 flip when the mean dosage/2 is >= 0.5. `flipped` (device int) receives
 * 1 when the flip was applied. Replaces read_bed_packed + get_mean_packed + flip_packed
 * (adamixture/src/utils_c/cython/snp_reader.pyx:76-120, 215-303;
 *  adamixture/src/snp_reader.py:747-757). workspace: adx_bed_workspace_bytes(). */
int adx_bed_workspace_bytes(int64_t M, int64_t N, size_t* bytes);
int adx_bed_to_packed(const uint8_t* bed, int64_t M, int64_t N, uint8_t* G, int* flipped,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Synthetic cohort sampler (no counterpart in the reference; used for benchmarks):
 * g = [u1 < h_q] + [u2 < h_q] with h_q = sum_k Pq[j][k] Qq[i][k] (16-bit fixed point,
 * rows of Qq sum to 2^16), u1|u2 = splitmix64((j*N+i)*0x9E3779B97F4A7C15 + key1),
 * missing when low32(splitmix64((j*N+i)*0x9E3779B97F4A7C15 + key2)) < miss_q. */
int adx_simulate_packed(const uint32_t* Pq, const uint32_t* Qq, int64_t M, int64_t N, int K,
                        uint64_t key1, uint64_t key2, uint32_t miss_q, uint8_t* G, void* stream);

/* ---------------------------------------------------------------- Adam-EM */

/* Scratch needed by adx_em_stats / adx_em_sweep / adx_em_adam_iteration for this shape.
 * Zero-fill it once after allocating: its first word is a sticky status word (the same
 * offset for every shape, so one buffer can serve several shapes). */
int adx_em_workspace_bytes(int64_t M, int64_t N, int K, int precision, size_t* bytes);

/* Read and clear the workspace's status word (ADX_OK, or ADX_ERR_TIMEOUT when a sweep's
 * bounded wait for its tensor-core work gave up). Synchronises `stream`. */
int adx_em_status(void* workspace, size_t workspace_bytes, int64_t M, int64_t N, int K,
                  int precision, int* status, void* stream);
/* Self-test of the bounded mbarrier wait the tensor-core sweep uses for every producer /
 * consumer hand-off (no counterpart in the reference): one barrier expecting one arrival;
 * arrive = 0 leaves it unarrived, so the wait must give up after `limit` polls. Writes three
 * ints to the device array `status`: the first wait's result (ADX_OK or ADX_ERR_TIMEOUT),
 * the abort word a timed-out wait raises (0/1), and a second warp's wait on the same barrier
 * (which must leave at once once the abort word is up). No GPU fault or hang either way. */
int adx_tc_wait_selftest(int arrive, uint32_t limit, int* status, void* stream);

/* One fused E-step sweep over G: A, B [M][K] and T [N][K] (float64), the sufficient
 * statistics EMAdamOptimizer.run_em_step accumulates (A_accum, B_accum, T_accum;
 * adamixture/model/em_adam_gpu.py:46-78 em_batch_math, 166-197 run_em_step).
 * P, Q are double for ADX_F64, float otherwise. */
int adx_em_stats(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
                 const void* Q, double* A, double* B, double* T, void* workspace,
                 size_t workspace_bytes, void* stream);

/* The E-step sweep alone: the same single pass over G as adx_em_stats, leaving the
 * per-block partial sums in `workspace` (for callers that time or combine the sweep). */
int adx_em_sweep(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
                 const void* Q, void* workspace, size_t workspace_bytes, void* stream);

/* The E-step sweep of an iteration with the previous iteration's log-likelihood check folded
 * in (float64, K <= 16; ADX_ERR_UNSUPPORTED otherwise): the reference checks
 * loglikelihood_gpu(P, Q) after an Adam move (adamixture/model/em_adam_gpu.py:330-353) and the
 * next E-step sweeps the same (P, Q), so this sweep leaves the partial sums of adx_em_sweep
 * and the log-likelihood of its input, which adx_em_loglik_from_sweep sums into the device
 * double *out (bit-identical to adx_loglik at ADX_F64). adx_em_adam_update then applies the
 * EM targets and the Adam move from the workspace (the second half of adx_em_adam_iteration),
 * after the caller has read the check and chosen the learning rate. */
int adx_em_sweep_loglik(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
                        const void* Q, void* workspace, size_t workspace_bytes, void* stream);
int adx_em_loglik_from_sweep(void* workspace, size_t workspace_bytes, int64_t M, int64_t N, int K,
                             int precision, double* out, void* stream);
int adx_em_adam_update(int64_t M, int64_t N, int K, int precision, double* P, double* Q, float* P32,
                       float* Q32, double* mP, double* vP, double* mQ, double* vQ, const double* q_bat,
                       double t, double lr, double beta1, double beta2, double eps, void* workspace,
                       size_t workspace_bytes, void* stream);

/* The float64 sweep (K <= 16) over SNP blocks [b0, b1) of its partition only, into the same
 * workspace partials: blocks are independent, so ranges that cover 0..n_blocks add up to
 * exactly adx_em_sweep. For callers that upload the packed matrix in pieces and sweep each
 * piece as it lands (block b holds SNPs [b*snps_per_block, (b+1)*snps_per_block), a multiple
 * of 16; each block is *ctas_per_block CTAs of one SM each, so a range fills whole waves
 * when its CTA count is a multiple of the SM count). No counterpart in the reference (it
 * sweeps fixed 8192-SNP chunks of a resident matrix, adamixture/model/em_adam_gpu.py:187-197). */
int adx_em_sweep_blocks_info(int64_t M, int64_t N, int K, int precision, int64_t* snps_per_block,
                             int* n_blocks, int* ctas_per_block);
int adx_em_sweep_blocks(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
                        const void* Q, int b0, int b1, void* workspace, size_t workspace_bytes,
                        void* stream);

/* EM targets from the statistics (em_final_update, em_adam_gpu.py:82-117):
 * P_EM = A P / max(P(A-B)+B, 1e-5); Q_EM = Q T / max(q_bat, 1e-5), rows / max(sum, 1e-5). */
int adx_em_targets(const double* P, const double* Q, const double* A, const double* B,
                   const double* T, const double* q_bat, int64_t M, int64_t N, int K,
                   double* P_EM, double* Q_EM, void* stream);

/* One Adam move toward the targets, then clamp P, Q to [1e-5, 1-1e-5] and renormalise Q
 * rows (EMAdamOptimizer.step + adam_update, em_adam_gpu.py:11-42, 201-224). `t` is the
 * step count after the increment. P32/Q32 (may be NULL) receive float copies. */
int adx_adam_step(double* P, double* Q, const double* P_EM, const double* Q_EM, double* mP,
                  double* vP, double* mQ, double* vQ, int64_t M, int64_t N, int K, double t,
                  double lr, double beta1, double beta2, double eps, float* P32, float* Q32,
                  void* stream);

/* One whole Adam-EM iteration (run_em_step + step) in two launches: the fused E-step
 * sweep, then one kernel that reduces the statistics, forms the EM targets and applies
 * the Adam move to every P and Q row. Inputs of the sweep are P32/Q32 (float) for
 * ADX_F32/ADX_BF16/ADX_F16 and P/Q (double) for ADX_F64; P32/Q32 are refreshed. */
int adx_em_adam_iteration(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                          double* P, double* Q, float* P32, float* Q32, double* mP, double* vP,
                          double* mQ, double* vQ, const double* q_bat, double t, double lr,
                          double beta1, double beta2, double eps, void* workspace,
                          size_t workspace_bytes, void* stream);

/* n_iters (1..4096) adx_em_adam_iteration calls captured once into a CUDA graph (captured on
 * a private stream; the same kernels and arguments). Iteration i of a replay takes the Adam
 * step *step_counter + i (step_counter: one device double that the graph owns for its
 * lifetime); adx_em_graph_launch(graph, t0, stream) sets it to t0, the steps already taken,
 * and replays, so the replay equals the eager iterations t0+1 .. t0+n_iters bit for bit.
 * Pointers, shapes and lr are fixed at capture: every buffer must stay allocated at the same
 * address until adx_em_graph_destroy. Replaces the per-iteration launches of the reference's
 * loop (adamixture/model/em_adam_gpu.py:330-333) between log-likelihood checks. */
int adx_em_graph_create(const uint8_t* G, int64_t M, int64_t N, int K, int precision, double* P,
                        double* Q, float* P32, float* Q32, double* mP, double* vP, double* mQ,
                        double* vQ, const double* q_bat, int n_iters, double lr, double beta1,
                        double beta2, double eps, double* step_counter, void* workspace,
                        size_t workspace_bytes, void** graph);
int adx_em_graph_launch(void* graph, double t0, void* stream);
int adx_em_graph_iterations(void* graph, int* n_iters);
int adx_em_graph_destroy(void* graph);

/* ---------------------------------------------------------------- batched float64 E-step
 * Several Adam-EM problems on one cohort in one sweep launch: n <= 64 problems, each with its
 * own packed genotypes G[p] (the same matrix, or for a cross-validation fold a copy with the
 * fold's entries hidden, e.g. by adx_cv_mask_hash), K[p] <= 16, P[p] [M][K[p]] and Q[p]
 * [N][K[p]] (device pointers, float64; the arrays of pointers and K are HOST arrays). Each
 * CTA runs the problems in order over its share of the matrix, so consecutive problems on
 * the same genotypes read them from memory once (from L2 after the first). Every problem's
 * statistics are bit-identical to the single-problem float64 sweep (adx_em_stats /
 * adx_em_adam_iteration at ADX_F64) of the same G, P and Q. The reference runs the K sweep
 * and its CV folds one after the other (adamixture/src/main.py:67-107,
 * adamixture/src/cv.py:171-267); no counterpart batches them. */
int adx_em_batch_workspace_bytes(int64_t M, int64_t N, int n, const int* K, size_t* bytes);
int adx_em_sweep_batch(int64_t M, int64_t N, int n, const int* K, const uint8_t* const* G,
                       const double* const* P, const double* const* Q, void* workspace,
                       size_t workspace_bytes, void* stream);
/* Problem p of the last batched sweep in `workspace`: mode 0 writes its A, B, T (float64);
 * mode 1 forms the EM targets and applies the Adam move to its P, Q and moments (t = step
 * count after the increment), as adx_em_adam_iteration does. */
int adx_em_batch_apply(int64_t M, int64_t N, int n, const int* K, int p, int mode, double* A, double* B,
                       double* T, const double* q_bat, double* P, double* Q, double* mP, double* vP,
                       double* mQ, double* vQ, double t, double lr, double beta1, double beta2, double eps,
                       void* workspace, size_t workspace_bytes, void* stream);

/* Shared-memory layouts ("tiles") of the float64 tensor-core sweep, chosen per device and K
 * by the autotuner (adamixture_b200/tune.py). No counterpart in the reference, whose E-step
 * has no tile choice (torch matmuls, adamixture/model/em_adam_gpu.py:46-78). A layout only
 * moves values in shared memory and sets how many CTAs share an SM, so every layout gives
 * bit-identical results; layout 0 (any K <= 16) is the default until one is set, layout 1
 * (K <= 8) puts two CTAs on an SM. The choice applies to adx_em_stats, adx_em_sweep,
 * adx_em_sweep_blocks, adx_em_sweep_loglik and adx_em_adam_iteration at ADX_F64 with
 * K <= 16, and to a batched sweep (adx_em_sweep_batch) when every problem's K has layout 1
 * selected. adx_dmma_tiles: the number of layouts for K; adx_dmma_tile_set / _get: the
 * layout of (device, K). */
int adx_dmma_tiles(int K, int* count);
int adx_dmma_tile_set(int device, int K, int tile);
int adx_dmma_tile_get(int device, int K, int* tile);

/* Binomial log-likelihood, float64 sum: sum over observed entries of
 * g log h + (2-g) log(1-h), h = clamp(P Q^T, 1e-10, 1-1e-10) (loglikelihood_gpu,
 * em_adam_gpu.py:226-279). *out is a device double. */
int adx_loglik_workspace_bytes(int64_t M, int64_t N, int K, int precision, size_t* bytes);
int adx_loglik(const uint8_t* G, int64_t M, int64_t N, int K, int precision, const void* P,
               const void* Q, double* out, void* workspace, size_t workspace_bytes,
               void* stream);

/* Allocation-free form of adx_loglik, for callers that cannot allocate device memory (a host
 * whose device memory belongs to another allocator, or a code path that cannot accept the
 * device-wide synchronisation of cudaMalloc/cudaFree). No counterpart in the reference.
 * The per-block partial sums live in a 16 KiB file-scope device array instead of a
 * workspace; every problem size fits (the plan never needs more than 1776 partials; the array holds
 * 2048, and a larger plan would be rejected with ADX_ERR_WORKSPACE).
 * The first call on a device (with it current) looks up the array's address; make it
 * before any stream capture. The address stays cached for the process: after a
 * cudaDeviceReset on that device this entry point must not be called there again.
 * Calls share the array: calls that overlap on the GPU race.
 * Allocates nothing; *out is a device double. */
int adx_loglik_noalloc(const uint8_t* G, int64_t M, int64_t N, int K, int precision,
                       const void* P, const void* Q, double* out, void* stream);

/* ---------------------------------------------------------------- initialisation
 * Shifted randomized SVD products of the centred genotypes Xc[j][i] = g - 2 f_j (0 where
 * missing; f float32 [M]), float32. They replace the decode-then-GEMM chunk loops of
 * SVD_gpu (adamixture/model/svd_gpu.py:80-87, 99-107, 133-139) and the centring unpack op
 * they call (pack2bit.cu:46-77). L <= 80. */
/* Y[M][L] = Xc B, B float32 [N][L]. */
int adx_rsvd_rows(const uint8_t* G, int64_t M, int64_t N, const float* f, const float* B, int L,
                  float* Y, void* stream);
int adx_rsvd_workspace_bytes(int64_t M, int64_t N, int L, size_t* bytes);
/* Z[N][L] = Xc' Y (accumulate != 0: Z += Xc' Y), Y float32 [M][L]; partial sums in the
 * workspace are added in a fixed order. */
int adx_rsvd_cols(const uint8_t* G, int64_t M, int64_t N, const float* f, const float* Y, int L,
                  int accumulate, float* Z, void* workspace, size_t workspace_bytes,
                  void* stream);

/* Batched bounded least squares, float64, one warp per row: X[m] = argmin over
 * lower <= x <= upper of 1/2 x'Ax - B[m]'x by block principal pivoting, A [K][K] shared.
 * Replaces bvls_kernel::batch_bvls_bpp_cuda (adamixture/src/utils_c/cuda/bvls_kernel.cu:
 * 75-164, 188-218), which ALS_gpu (adamixture/model/als_gpu.py:105,115) calls. */
int adx_bvls(const double* A, const double* B, int64_t M, int K, double lower, double upper,
             double* X, void* stream);

/* ---------------------------------------------------------------- original ADMIXTURE (BR-QN)
 * Gradient and Hessian passes over the packed genotypes, float64 (outputs overwritten):
 * Q side XtX_q [N][K][K], Xtz_q [N][K] (compute_grad_hess_Q_gpu, br_qn_gpu.py:145-179);
 * P side XtX_p [M][K][K], Xtz_p [M][K] (compute_grad_hess_P_gpu, br_qn_gpu.py:182-214).
 * Xtz is the gradient as computed there (not yet negated). */
int adx_grad_hess_q(const uint8_t* G, int64_t M, int64_t N, int K, const double* P,
                    const double* Q, double* XtX_q, double* Xtz_q, void* stream);
int adx_grad_hess_p(const uint8_t* G, int64_t M, int64_t N, int K, const double* P,
                    const double* Q, double* XtX_p, double* Xtz_p, void* stream);
/* SQP steps, float64, one warp per row; Xtz as the reference's caller passes it (negated,
 * br_qn_gpu.py:295). Q rows: simplex QP with shift from v_kk [K][K], then projection onto
 * {q >= 1e-5, sum q = 1} (sqp_kernel::sqp_solve_q_cuda, sqp_kernel.cu:262-286, 320-345).
 * P rows: box QP, then clamping to [1e-5, 1-1e-5] (sqp_solve_p_cuda, sqp_kernel.cu:
 * 288-311, 347-370). */
int adx_sqp_q(const double* XtX_q, const double* Xtz_q, const double* Q, const double* v_kk,
              int64_t N, int K, double* Q_next, void* stream);
int adx_sqp_p(const double* XtX_p, const double* Xtz_p, const double* P, int64_t M, int K,
              double* P_next, void* stream);

/* Projections of rows onto the feasible sets, float64, in place: Q rows onto
 * {q >= 1e-5, sum q = 1} (project_q_simplex, adamixture/src/utils_c/cython/sqp.pyx:112-146,
 * 330-333), P entries clamped to [1e-5, 1 - 1e-5] (project_p_box, sqp.pyx:148-151, 335-338). */
int adx_project_simplex(double* Q, int64_t N, int K, void* stream);
int adx_project_box(double* P, int64_t M, int K, void* stream);

/* ---------------------------------------------------------------- cross-validation
 * Held-out entries of a fold are hidden (set to 3) in a copy G of the packed matrix; the
 * copy must be 4-byte aligned and g_bytes (its allocation) a multiple of 4 covering it.
 * Folds as a list of flat indices j*N + i (int64; the reference's shuffled-list rule,
 * adamixture/src/cv.py:202-222, mask_entries_i32/i64 in br_qn.pyx) or by the reference's
 * hash of the flat index (cv.py:58-78, 117-147). The deviance sums (deviance_squared_sum,
 * br_qn.pyx:92-150) read the unmasked G0 and write a device double. */
int adx_cv_workspace_bytes(size_t* bytes);
int adx_cv_mask_list(uint8_t* G, size_t g_bytes, int64_t M, int64_t N, const int64_t* idx,
                     int64_t n, void* workspace, size_t workspace_bytes, void* stream);
int adx_cv_mask_hash(uint8_t* G, size_t g_bytes, const uint8_t* G0, int64_t M, int64_t N,
                     uint64_t seed, int n_folds, int fold, void* stream);
int adx_cv_deviance_list(const uint8_t* G0, int64_t M, int64_t N, int K, const double* P,
                         const double* Q, const int64_t* idx, int64_t n, double* out,
                         void* workspace, size_t workspace_bytes, void* stream);
int adx_cv_deviance_hash(const uint8_t* G0, int64_t M, int64_t N, int K, const double* P,
                         const double* Q, uint64_t seed, int n_folds, int fold, double* out,
                         void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- outputs (host)
 * Writes a float64 [rows][cols] HOST matrix as text, "%.18e" values separated by single
 * spaces, one row per line: byte for byte np.savetxt(path, X, delimiter=' '), the
 * reference's .Q/.P writer (write_outputs, adamixture/src/utils.py:252-273). threads <= 0:
 * all hardware threads. */
int adx_write_text_matrix(const char* path, const double* X, int64_t rows, int64_t cols,
                          int threads);
/* The same with "%.<decimals>f" values (0 <= decimals <= 60): byte for byte
 * np.savetxt(path, X, delimiter=' ', fmt='%.6f') at decimals = 6, the writer of the
 * projection and supervised commands (adamixture/project_entry.py:289,
 * adamixture/supervised_entry.py:386-389). */
int adx_write_text_matrix_fixed(const char* path, const double* X, int64_t rows, int64_t cols,
                                int decimals, int threads);

/* ---------------------------------------------------------------- warm-start network
 * No counterpart in the reference (a new component of this library). A per-sample network
 * 33 -> 256 -> 256 -> K (K <= 16), GELU hidden layers, output softmax(f(x) + prior) with
 * prior [B][K] optional (log of the ALS memberships, so an untrained network reproduces the
 * ALS start). Weights BF16 (uint16 bit patterns) [out][in], biases and activations float32.
 * adx_mlp_forward keeps the activations in the workspace; adx_mlp_backward (same X, same
 * workspace, right after the forward) writes the mean cross-entropy against soft targets T
 * to *loss (device float) and every weight/bias gradient (float32). adx_mlp_adam: one Adam
 * step (bias-corrected, step t >= 1) on a float32 master, refreshing its BF16 copy. */
int adx_mlp_workspace_bytes(int64_t B, int K, size_t* bytes);
int adx_mlp_forward(const float* X, const float* prior, const uint16_t* W1, const float* b1,
                    const uint16_t* W2, const float* b2, const uint16_t* W3, const float* b3,
                    int64_t B, int K, float* Q_out, void* workspace, size_t workspace_bytes,
                    void* stream);
int adx_mlp_backward(const float* X, const float* T, const uint16_t* W2, const uint16_t* W3,
                     int64_t B, int K, float* dW1, float* db1, float* dW2, float* db2,
                     float* dW3, float* db3, float* loss, void* workspace,
                     size_t workspace_bytes, void* stream);
int adx_mlp_adam(float* w, uint16_t* w_bf16, const float* g, float* m, float* v, int64_t n,
                 float lr, float beta1, float beta2, float eps, int t, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ADAMIXTURE_B200_H */
