"""Seeded synthetic admixed cohorts (Balding-Nichols P, Dirichlet Q, binomial G).

The reference has no generator; this one follows the published benchmark recipe:

* f_j ~ Uniform(0.05, 0.95)
* P_jk ~ Beta(f_j (1-F)/F, (1-f_j)(1-F)/F)            (Balding-Nichols with F_ST = F)
* Q_i ~ Dirichlet(alpha 1_K), or a mixture of Dirichlets
* g_ij ~ Binomial(2, sum_k Q_ik P_jk), missing uniformly at random with rate ``miss``.

P and Q are drawn with numpy's ``default_rng(seed)``. Genotypes are sampled with
exact integer arithmetic so that the host sampler below and the CUDA sampler
(``adx_simulate_packed``) agree bit for bit:

* P and Q are quantised to 16-bit fixed point: ``Pq = rint(P * 2^16)`` and ``Qq`` with
  every row summing to exactly 2^16 (largest-remainder rounding). Then
  ``h_q = sum_k Pq_jk Qq_ik`` lies in [0, 2^32] and ``h = h_q / 2^32``.
* Entry (j, i) has the 64-bit counter ``c = j * N + i``. The two allele draws are
  the low and high 32 bits of ``splitmix64(c * 0x9E3779B97F4A7C15 + key1)`` and the
  missingness draw is the low 32 bits of ``splitmix64(c * 0x9E3779B97F4A7C15 + key2)``.
  ``splitmix64`` is the finaliser of Steele, Lea and Flood's SplitMix64 generator
  (OOPSLA 2014), as used by Vigna's xoshiro seeding.
* ``g = [u1 < h_q] + [u2 < h_q]``, replaced by 3 when ``u3 < rint(miss * 2^32)``.
"""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
ONE16 = 1 << 16


def splitmix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on a uint64 array (wrapping arithmetic)."""
    z = z.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z ^= z >> np.uint64(30)
        z *= _M1
        z ^= z >> np.uint64(27)
        z *= _M2
        z ^= z >> np.uint64(31)
    return z


def seed_keys(seed: int) -> tuple[int, int]:
    """The two 64-bit stream keys derived from ``seed``."""
    s = splitmix64(np.array([seed * 2 + 1], dtype=np.uint64))[0]
    t = splitmix64(np.array([seed * 2 + 2], dtype=np.uint64))[0]
    return int(s), int(t)


def quantize_P(P: np.ndarray) -> np.ndarray:
    return np.rint(np.clip(P, 0.0, 1.0) * ONE16).astype(np.uint32)


def quantize_Q(Q: np.ndarray) -> np.ndarray:
    """Rows of Q in 16-bit fixed point summing to exactly 2^16 (largest remainder)."""
    Q = np.clip(Q, 0.0, None)
    Q = Q / Q.sum(axis=1, keepdims=True)
    x = Q * ONE16
    q = np.floor(x).astype(np.int64)
    short = ONE16 - q.sum(axis=1)
    order = np.argsort(-(x - q), axis=1, kind="stable")
    K = Q.shape[1]
    for r in range(K):
        take = short > r
        q[np.nonzero(take)[0], order[take, r]] += 1
    return q.astype(np.uint32)


def sample_genotypes(Pq: np.ndarray, Qq: np.ndarray, miss_q: int, keys: tuple[int, int],
                     m_start: int = 0, m_count: int | None = None) -> np.ndarray:
    """Unpacked genotypes ``[m_count, N]`` (uint8, 3 = missing) for SNP rows from m_start."""
    M = Pq.shape[0]
    N = Qq.shape[0]
    if m_count is None:
        m_count = M - m_start
    # every product and partial sum of h_q is an integer <= 2^32, so a float64 product
    # (BLAS) is exact in any summation order
    hq = (Pq[m_start:m_start + m_count].astype(np.float64) @ Qq.T.astype(np.float64)).astype(np.uint64)
    j = np.arange(m_start, m_start + m_count, dtype=np.uint64)[:, None]
    i = np.arange(N, dtype=np.uint64)[None, :]
    k1, k2 = (np.uint64(k) for k in keys)
    with np.errstate(over="ignore"):
        c = (j * np.uint64(N) + i) * GOLDEN
        r = splitmix64(c + k1)
        r2 = splitmix64(c + k2)
    u1 = r & np.uint64(0xFFFFFFFF)
    u2 = r >> np.uint64(32)
    u3 = r2 & np.uint64(0xFFFFFFFF)
    g = (u1 < hq).astype(np.uint8) + (u2 < hq).astype(np.uint8)
    g[u3 < np.uint64(miss_q)] = 3
    return g


@dataclass
class Cohort:
    """A synthetic cohort: true parameters and the sampler's integer inputs."""

    N: int
    M: int
    K: int
    P: np.ndarray        # [M, K] float64 true allele frequencies
    Q: np.ndarray        # [N, K] float64 true ancestry proportions
    Pq: np.ndarray       # [M, K] uint32 fixed point
    Qq: np.ndarray       # [N, K] uint32 fixed point, rows sum to 2^16
    miss_q: int
    keys: tuple[int, int]

    def genotypes(self, m_start: int = 0, m_count: int | None = None) -> np.ndarray:
        return sample_genotypes(self.Pq, self.Qq, self.miss_q, self.keys, m_start, m_count)

    def genotypes_parallel(self, m_start: int, m_count: int, threads: int | None = None,
                           rows_per_task: int = 64) -> np.ndarray:
        """The same rows as ``genotypes``, sampled by several host threads (numpy releases
        the interpreter lock inside its array operations) into one ``[m_count, N]`` array."""
        import os
        from concurrent.futures import ThreadPoolExecutor

        out = np.empty((m_count, self.N), dtype=np.uint8)

        def task(s):
            n = min(rows_per_task, m_count - s)
            out[s:s + n] = self.genotypes(m_start + s, n)

        with ThreadPoolExecutor(threads or os.cpu_count() or 1) as ex:
            list(ex.map(task, range(0, m_count, rows_per_task)))
        return out

    def packed(self, block: int = 65536) -> np.ndarray:
        """Packed ``[ceil(M/4), N]`` genotypes, built on the host in SNP blocks."""
        from .packing import pack
        out = np.zeros(((self.M + 3) // 4, self.N), dtype=np.uint8)
        block = max(4, block - block % 4)
        for s in range(0, self.M, block):
            g = self.genotypes(s, min(block, self.M - s))
            out[s // 4: s // 4 + (g.shape[0] + 3) // 4] = pack(g)
        return out


def shard_keys(keys: tuple[int, int], j0: int, N: int) -> tuple[int, int]:
    """Sampler keys that make SNP rows [j0, ...) of a cohort come out of a sampler started
    at row 0: the stream of entry (j, i) is splitmix64((j N + i) * GOLDEN + key), so
    shifting the keys by j0 N GOLDEN (mod 2^64) shifts j by j0."""
    shift = (int(j0) * int(N) * int(GOLDEN)) % (1 << 64)
    return ((int(keys[0]) + shift) % (1 << 64), (int(keys[1]) + shift) % (1 << 64))


def make_cohort(N: int, M: int, K: int, F: float, alpha: float | tuple = 0.5,
                miss: float = 0.01, seed: int = 0) -> Cohort:
    """Draw the true P and Q for a cohort.

    ``alpha`` is either a Dirichlet concentration or a mixture
    ``((weight, alpha), ...)``: e.g. ``((0.7, 0.05), (0.3, 1.0))`` is 70% near-pure
    and 30% admixed samples.
    """
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.05, 0.95, size=M)
    a = f * (1.0 - F) / F
    b = (1.0 - f) * (1.0 - F) / F
    P = rng.beta(a[:, None], b[:, None], size=(M, K))
    if isinstance(alpha, (tuple, list)):
        weights = np.array([w for w, _ in alpha])
        comp = rng.choice(len(alpha), size=N, p=weights / weights.sum())
        Q = np.empty((N, K))
        for c, (_, al) in enumerate(alpha):
            sel = comp == c
            Q[sel] = rng.dirichlet(np.full(K, al), size=int(sel.sum()))
    else:
        Q = rng.dirichlet(np.full(K, float(alpha)), size=N)
    Q = np.nan_to_num(Q, nan=1.0 / K)
    miss_q = int(round(miss * 2.0 ** 32))
    return Cohort(N, M, K, P, Q, quantize_P(P), quantize_Q(Q), miss_q, seed_keys(seed))


# --------------------------------------------------------------------------
# PLINK BED writer (for CLI round trips)
# --------------------------------------------------------------------------

_BED_CODE = np.array([3, 2, 0, 1], dtype=np.uint8)  # g -> 2-bit code (inverse of LUT [2,3,1,0])


def write_bed(prefix: str | Path, G: np.ndarray) -> None:
    """Write unpacked genotypes ``[M, N]`` as ``prefix.bed/.bim/.fam`` (SNP-major).

    Every SNP goes on an autosome (chromosome ``1 + j % 22``) so the reader's default
    autosome filter keeps all of them.
    """
    prefix = str(prefix)
    M, N = G.shape
    nb = (N + 3) // 4
    codes = _BED_CODE[G]
    pad = np.zeros((M, nb * 4), dtype=np.uint8)
    pad[:, :N] = codes
    pad = pad.reshape(M, nb, 4)
    rows = (pad[:, :, 0] | (pad[:, :, 1] << 2) | (pad[:, :, 2] << 4) | (pad[:, :, 3] << 6)).astype(np.uint8)
    with open(prefix + ".bed", "wb") as fh:
        fh.write(bytes([0x6C, 0x1B, 0x01]))
        fh.write(rows.tobytes())
    with open(prefix + ".bim", "w") as fh:
        for j in range(M):
            fh.write(f"{1 + j % 22}\tsnp{j}\t0\t{j + 1}\tA\tG\n")
    with open(prefix + ".fam", "w") as fh:
        for i in range(N):
            fh.write(f"0 ind{i} 0 0 0 -9\n")
