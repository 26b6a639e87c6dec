"""Float64 numpy restatement of the reference Adam-EM GPU path. TEST INFRASTRUCTURE ONLY.

Follows the reference's ``--device gpu`` semantics (not its CPU twin): the E-step
clamps the reconstruction to [1e-5, 1-1e-5], P_EM is not clipped to the domain,
the log-likelihood clamps to [1e-10, 1-1e-10], and the priming sequence is
EM -> Adam -> (discarded EM). Every function cites the reference file:line it
restates (paths relative to the reference project root).

Sizes: meant for cohorts up to about 1e8 genotype entries (it materialises M x N
float64 temporaries per SNP chunk).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

E_CLAMP = 1e-5        # adamixture/model/em_adam_gpu.py:63
LL_CLAMP = 1e-10      # adamixture/model/em_adam_gpu.py:239
DOMAIN = 1e-5         # adamixture/model/em_adam_gpu.py:222-223


# --------------------------------------------------------------------------
# 2-bit packed genotype layout
# --------------------------------------------------------------------------

def unpack(Gp: np.ndarray, M: int, m_start: int = 0, count: int | None = None) -> np.ndarray:
    """Decode SNP rows [m_start, m_start+count) of a packed ``[ceil(M/4), N]`` matrix.

    Byte ``(j>>2)*N + i`` holds SNP j of sample i in bits ``2*(j&3)``; 3 = missing.
    Restates ``unpack2bit_chunk_kernel_uint8_SNPsPacked``
    (adamixture/src/utils_c/cuda/pack2bit.cu:15-44).
    """
    if count is None:
        count = M - m_start
    count = max(0, min(count, M - m_start))
    j = np.arange(m_start, m_start + count)
    rows = Gp[j >> 2]                      # [count, N]
    shift = ((j & 3) << 1).astype(np.uint8)[:, None]
    return ((rows >> shift) & 3).astype(np.uint8)


def pack(G: np.ndarray) -> np.ndarray:
    """Pack an unpacked ``[M, N]`` uint8 matrix (values 0..3) into ``[ceil(M/4), N]``.

    Restates ``pack_genotypes`` (adamixture/src/utils_c/cython/snp_reader.pyx:123-157):
    SNP j goes to row j>>2, bits 2*(j&3); bits of absent SNPs in the last row are 0.
    """
    M, N = G.shape
    Mb = (M + 3) // 4
    out = np.zeros((Mb, N), dtype=np.uint8)
    for k in range(4):
        rows = G[k::4].astype(np.uint8) & 3
        out[: rows.shape[0]] |= rows << (2 * k)
    return out


BED_LUT = np.array([2, 3, 1, 0], dtype=np.uint8)  # adamixture/src/utils_c/cython/snp_reader.pyx:53-58


def bed_to_packed(bed_rows: np.ndarray, N: int) -> np.ndarray:
    """PLINK BED SNP-major rows ``[M, ceil(N/4)]`` -> packed ``[ceil(M/4), N]``.

    Sample i of SNP j sits in BED byte ``i>>2`` at bits ``2*(i&3)`` and decodes with
    the LUT [2,3,1,0] (00 hom-A1 -> 2, 01 missing -> 3, 10 het -> 1, 11 hom-A2 -> 0).
    Restates ``read_bed_packed`` (adamixture/src/utils_c/cython/snp_reader.pyx:76-120).
    """
    M = bed_rows.shape[0]
    i = np.arange(N)
    codes = (bed_rows[:, i >> 2] >> ((i & 3) << 1).astype(np.uint8)) & 3
    return pack(BED_LUT[codes])


def packed_mean(Gp: np.ndarray, M: int) -> float:
    """Mean allele dosage / 2 over observed entries (adamixture/src/utils_c/cython/snp_reader.pyx:215-252)."""
    G = unpack(Gp, M)
    obs = G != 3
    cnt = 2 * int(obs.sum())
    return 0.0 if cnt == 0 else float(G[obs].astype(np.int64).sum()) / cnt


FLIP_TAB = np.array([2, 1, 0, 3], dtype=np.uint8)


def flip_packed(Gp: np.ndarray, M: int) -> np.ndarray:
    """0<->2 swap on every entry, zeroing padding bits of the last row.

    Restates ``flip_packed`` (adamixture/src/utils_c/cython/snp_reader.pyx:254-303);
    the reader applies it when ``packed_mean >= 0.5`` (adamixture/src/snp_reader.py:747-757).
    """
    G = unpack(Gp, M)
    return pack(FLIP_TAB[G])


# --------------------------------------------------------------------------
# Per-SNP / per-sample statistics
# --------------------------------------------------------------------------

def allele_frequency(G: np.ndarray) -> np.ndarray:
    """f_j = sum_i g_ij / (2 * #observed_j), 0 when nothing is observed; float32.

    Restates ``freq_batch_math`` + ``_calculate_frequencies_gpu_once``
    (adamixture/src/utils.py:781-830).
    """
    obs = G != 3
    s = (G.astype(np.float32) * obs).sum(axis=1, dtype=np.float32)
    d = obs.sum(axis=1).astype(np.float32)
    f = np.zeros(G.shape[0], dtype=np.float32)
    v = d > 0
    f[v] = s[v] / (np.float32(2.0) * d[v])
    return f


def sample_counts(G: np.ndarray) -> np.ndarray:
    """q_bat_i = 2 * #observed SNPs of sample i (em_adam_gpu.py:76, accumulated at :196)."""
    return 2.0 * (G != 3).sum(axis=0).astype(np.float64)


# --------------------------------------------------------------------------
# E-step, EM targets, Adam
# --------------------------------------------------------------------------

def em_stats(G: np.ndarray, P: np.ndarray, Q: np.ndarray, chunk: int = 8192):
    """One E-step sweep: A, B [M,K], T [N,K] and q_bat [N] (float64).

    Restates ``em_batch_math`` (adamixture/model/em_adam_gpu.py:46-78) and the chunk
    loop of ``EMAdamOptimizer.run_em_step`` (:166-197):
    rec = clamp(P Q^T, 1e-5, 1-1e-5); a = g/rec*mask; b = (2-g)/(1-rec)*mask;
    A = a Q; B = b Q; T = (a-b)^T P + sum_j b; q_bat = 2*sum_j mask.
    """
    M = G.shape[0]
    N, K = Q.shape
    A = np.zeros((M, K))
    B = np.zeros((M, K))
    T = np.zeros((N, K))
    qb = np.zeros(N)
    for s in range(0, M, chunk):
        e = min(s + chunk, M)
        g = G[s:e].astype(np.float64)
        mask = (G[s:e] != 3).astype(np.float64)
        rec = np.clip(P[s:e] @ Q.T, E_CLAMP, 1.0 - E_CLAMP)
        ta = (g / rec) * mask
        tb = ((2.0 - g) / (1.0 - rec)) * mask
        A[s:e] = ta @ Q
        B[s:e] = tb @ Q
        T += (ta - tb).T @ P[s:e]
        T += tb.sum(axis=0)[:, None]
        qb += mask.sum(axis=0) * 2.0
    return A, B, T, qb


def em_final(P, Q, A, B, T, q_bat):
    """EM targets (P_EM, Q_EM) from the sufficient statistics.

    Restates ``em_final_update`` (adamixture/model/em_adam_gpu.py:82-117), same
    operation order: P_EM = A * (P * 1/max(P(A-B)+B, 1e-5));
    Q_EM = Q*T/max(q_bat,1e-5), rows divided by max(row sum, 1e-5).
    """
    den = np.maximum((A - B) * P + B, 1e-5)
    P_EM = (1.0 / den) * P * A
    Q_EM = Q * T * (1.0 / np.maximum(q_bat, 1e-5))[:, None]
    Q_EM = Q_EM / np.maximum(Q_EM.sum(axis=1, keepdims=True), 1e-5)
    return P_EM, Q_EM


@dataclass
class Adam:
    """Adam state of ``EMAdamOptimizer`` (adamixture/model/em_adam_gpu.py:121-164)."""

    lr: float
    beta1: float
    beta2: float
    eps: float
    t: float = 0.0
    mP: np.ndarray | None = None
    vP: np.ndarray | None = None
    mQ: np.ndarray | None = None
    vQ: np.ndarray | None = None

    def init(self, P, Q):
        self.mP = np.zeros_like(P)
        self.vP = np.zeros_like(P)
        self.mQ = np.zeros_like(Q)
        self.vQ = np.zeros_like(Q)
        return self


def adam_update(param, target, m, v, t, lr, b1, b2, eps):
    """In-place Adam move toward the EM target (adamixture/model/em_adam_gpu.py:11-42)."""
    delta = target - param
    m *= b1
    m += delta * (1.0 - b1)
    v *= b2
    v += (1.0 - b2) * (delta * delta)
    m_hat = m / (1.0 - b1 ** t)
    v_hat = v / (1.0 - b2 ** t)
    param += lr * m_hat / (np.sqrt(v_hat) + eps)


def adam_step(st: Adam, P, Q, P_EM, Q_EM):
    """``EMAdamOptimizer.step`` (adamixture/model/em_adam_gpu.py:201-224)."""
    st.t += 1.0
    adam_update(P, P_EM, st.mP, st.vP, st.t, st.lr, st.beta1, st.beta2, st.eps)
    adam_update(Q, Q_EM, st.mQ, st.vQ, st.t, st.lr, st.beta1, st.beta2, st.eps)
    np.clip(P, DOMAIN, 1.0 - DOMAIN, out=P)
    np.clip(Q, DOMAIN, 1.0 - DOMAIN, out=Q)
    Q /= Q.sum(axis=1, keepdims=True)


def loglik(G: np.ndarray, P: np.ndarray, Q: np.ndarray, chunk: int = 8192) -> float:
    """Binomial log-likelihood, float64 (adamixture/model/em_adam_gpu.py:226-279).

    sum over observed entries of g*log(h) + (2-g)*log1p(-h), h clamped to
    [1e-10, 1-1e-10].
    """
    ll = 0.0
    for s in range(0, G.shape[0], chunk):
        e = min(s + chunk, G.shape[0])
        rec = np.clip(P[s:e] @ Q.T, LL_CLAMP, 1.0 - LL_CLAMP)
        g = G[s:e].astype(np.float64)
        mask = G[s:e] != 3
        term = g * np.log(rec) + (2.0 - g) * np.log1p(-rec)
        ll += float((term * mask).sum())
    return ll


@dataclass
class Trace:
    """Per-iteration record of an oracle run."""

    P: list = field(default_factory=list)
    Q: list = field(default_factory=list)
    loglik: list = field(default_factory=list)   # (iteration, L) at each check
    lr: list = field(default_factory=list)


def optimize(G, P, Q, lr=0.005, beta1=0.80, beta2=0.88, eps=1e-8, max_iter=10000,
             check=5, lr_decay=0.5, min_lr=1e-4, patience=3, tol=0.1,
             trace_iters: int = 0):
    """Adam-EM driver (adamixture/model/em_adam_gpu.py:281-356).

    Priming: EM, Adam step, then one more E-step whose result the reference discards
    (:320-322). Then ``max_iter`` Adam-EM iterations with a log-likelihood check every
    ``check`` iterations, best-checkpoint, lr decay after ``patience`` flat checks and
    a stop once lr reaches ``min_lr`` (:330-353). Returns ``(P_best, Q_best, L_best,
    trace)``; ``trace`` holds P/Q after the priming step and after each of the first
    ``trace_iters`` iterations.
    """
    P = P.astype(np.float64, copy=True)
    Q = Q.astype(np.float64, copy=True)
    st = Adam(lr, beta1, beta2, eps).init(P, Q)
    tr = Trace()
    A, B, T, qb = em_stats(G, P, Q)
    adam_step(st, P, Q, *em_final(P, Q, A, B, T, qb))
    if trace_iters:
        tr.P.append(P.copy())
        tr.Q.append(Q.copy())
    L_best = loglik(G, P, Q)
    P_best, Q_best = P.copy(), Q.copy()
    wait = 0
    for it in range(max_iter):
        A, B, T, qb = em_stats(G, P, Q)
        adam_step(st, P, Q, *em_final(P, Q, A, B, T, qb))
        if it < trace_iters:
            tr.P.append(P.copy())
            tr.Q.append(Q.copy())
        if (it + 1) % check == 0:
            L = loglik(G, P, Q)
            tr.loglik.append((it + 1, L))
            tr.lr.append(st.lr)
            if L > L_best + tol:
                L_best = L
                P_best, Q_best = P.copy(), Q.copy()
                wait = 0
            else:
                wait += 1
                if wait >= patience:
                    st.lr = max(st.lr * lr_decay, min_lr)
                    if st.lr <= min_lr:
                        break
                    wait = 0
    return P_best, Q_best, L_best, tr


def bytes_per_pass(M: int, N: int, K: int) -> int:
    """Algorithmic HBM bytes of one fused E-step pass: packed G + fp32 P, Q read and
    A, B, T written (4*K*(3M+2N))."""
    return ((M + 3) // 4) * N + 4 * K * (3 * M + 2 * N)


def entries(M: int, N: int) -> int:
    return M * N


