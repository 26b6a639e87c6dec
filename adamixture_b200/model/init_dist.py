"""The initialisation (randomized SVD, then ALS) sharded over GPUs by SNP rows, one process
per GPU: the algorithms of ``svd_gpu`` and ``als_gpu`` (adamixture/model/svd_gpu.py:40-154,
adamixture/model/als_gpu.py:45-127) when each rank holds a contiguous range [j0, j1) of
whole packed rows (``em_adam_dist.shard_rows``), as the sharded Adam-EM does.

Everything indexed by SNP (the rows of the random basis, the projections, U, P, the
allele frequencies) stays on the rank that holds those SNPs; everything indexed by sample,
and every L x L or K x K matrix, is replicated. Each sum over SNPs is a local partial plus
one all-reduce:

* randomized SVD: the N x L product X' B of the prime pass and of every power iteration
  (N x L float32: 16 MB at N=200k, L=20), and the L x L Gram matrix of the final
  projection, whose eigen-decomposition gives S, V and each rank's rows of U;
* ALS: P'P (K x K), f' I_p (1 x K) and Z' I_p (k x K) for each Q update; the P update is
  local.

The random numbers are the single-process run's: every rank draws the full M x L basis and
the full M x K ALS start from the seeded generator and keeps its own rows. Replicated
values are equal on every rank (the same reduced inputs through the same deterministic
operations), so every rank takes the same branches (the SVD's relative stop, ALS's RMSE
stop) and the same collectives. The results equal the single-process run's up to the
summation order of the all-reduced sums.

The passes over the genotypes come from a backend (``CudaInitBackend``: this library's
fused randomized-SVD kernels and warp-per-row BVLS); the host logic does not depend on it,
so the multi-rank path also runs on CPU ranks with a float64 backend in the tests.
"""
from __future__ import annotations

import logging

import torch
import torch.distributed as dist

from .als_gpu import mapP, mapQ
from .svd_gpu import eigSVD_gpu

log = logging.getLogger(__name__)


class CudaInitBackend:
    """Passes over this rank's packed rows on this library's kernels (float32, as the
    single-GPU SVD) and the batched BVLS."""

    dtype = torch.float32   # the randomized SVD's working type

    def rsvd_cols(self, G, f, B, M_local):
        from .. import ops

        return ops.rsvd_cols(G, f.to(torch.float32).contiguous(), B, M_local)

    def rsvd_rows(self, G, f, Y, M_local):
        from .. import ops

        return ops.rsvd_rows(G, f.to(torch.float32).contiguous(), Y, M_local)

    def bvls(self, A, B, lower, upper):
        from .. import ops

        return ops.bvls(A, B, lower, upper)

    def frequencies(self, G, M_local):
        from .. import ops

        return ops.allele_frequency(G, M_local)


def _sum(t: torch.Tensor, group=None) -> torch.Tensor:
    """Sum over the ranks in place (nothing to do without a process group)."""
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
    return t


def eig_svd_rows(C_rows: torch.Tensor, group=None):
    """``eigSVD_gpu(C.T)`` for a tall ``C`` [M, L] whose rows are spread over the ranks:
    the L x L Gram matrix is summed over the ranks, so S and V are replicated and each rank
    gets its own rows of U. Largest first, as eigSVD_gpu."""
    cov = _sum(C_rows.transpose(0, 1) @ C_rows, group)
    D, V = torch.linalg.eigh(cov)
    S = torch.sqrt(D)
    U = (C_rows @ V) / S
    idx = torch.arange(V.shape[1] - 1, -1, -1, device=C_rows.device)
    return U[:, idx], S.flip(0), V[:, idx]


def svd_sharded(G, N: int, M: int, j0: int, j1: int, f, k: int, seed: int, power: int, tol: float,
                backend=None, group=None):
    """Rank-``k`` randomized SVD of the centred genotypes from this rank's rows [j0, j1):
    ``(U rows [j1-j0, k], S [k], V [N, k])`` -- svd_gpu.py:40-154 with the sums over SNPs
    all-reduced. ``f``: the frequencies of this rank's SNPs."""
    be = backend or CudaInitBackend()
    M_local = j1 - j0
    L = max(k + 10, 20)
    dev = f.device
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    basis = torch.randn((M, L), dtype=torch.float32, generator=gen, device=dev)
    dt = getattr(be, "dtype", torch.float32)
    proj = basis[j0:j1].to(dt).contiguous()
    del basis
    accum = _sum(be.rsvd_cols(G, f, proj, M_local), group)        # prime pass: X' Omega
    orth, _, _ = eigSVD_gpu(accum.T)
    # the shift and the stop exactly as the single-process loop computes them
    alpha = torch.tensor(0.0, device=dev)
    singular = torch.zeros(L, device=dev)
    for i in range(power):
        proj = be.rsvd_rows(G, f, orth.to(dt).contiguous(), M_local)   # this rank's rows of X orth
        accum = _sum(be.rsvd_cols(G, f, proj, M_local), group)   # X' proj
        Qm, S, _ = eigSVD_gpu(accum.sub(orth, alpha=alpha.item()).T)
        if i > 0:
            s_cur = S + alpha
            rel = torch.abs(s_cur - singular) / torch.maximum(s_cur, torch.tensor(1e-12, device=dev))
            if torch.max(rel[:k]) < tol:
                log.info(f"        Converged at iteration {i}.")
                break
            singular.copy_(s_cur)
        else:
            singular.copy_(S + alpha)
        if S[-1] > alpha:
            alpha = 0.5 * (S[-1] + alpha)
        orth = Qm
    proj = be.rsvd_rows(G, f, orth.to(dt).contiguous(), M_local)   # final projection
    u_rows, s_all, v_c = eig_svd_rows(proj, group)
    return u_rows[:, :k].contiguous(), s_all[:k].contiguous(), (orth @ v_c[:, :k]).contiguous()


def als_sharded(U_rows, S, V, f, seed: int, M: int, j0: int, j1: int, K: int, max_iter: int, tol: float,
                backend=None, group=None):
    """ALS from the sharded SVD: ``(P rows [j1-j0, K], Q [N, K])`` (float64) --
    als_gpu.py:45-127 with P'P, f' I_p and Z' I_p all-reduced. ``U_rows``, ``f``: this
    rank's rows; ``S``, ``V``: replicated."""
    be = backend or CudaInitBackend()
    dev = f.device
    dtype = torch.float64
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    Z = (U_rows * S).to(dtype)
    V = torch.as_tensor(V, device=dev, dtype=dtype)
    f_work = f.to(dtype)

    P = torch.rand((M, K), dtype=dtype, generator=gen, device=dev)[j0:j1].contiguous()
    mapP(P)

    def q_update(P):
        A_cov_P = _sum(P.T @ P, group)
        I_p = P @ torch.linalg.pinv(A_cov_P)
        f_p = _sum(f_work.reshape(1, -1) @ I_p, group)
        ZtI = _sum(Z.T @ I_p, group)
        return A_cov_P, 0.5 * (V @ ZtI) + f_p

    _, Q = q_update(P)
    mapQ(Q)
    Q0 = Q.clone()
    for i in range(max_iter):
        A_cov_Q = Q.T @ Q
        I_q = Q @ torch.linalg.pinv(A_cov_Q)
        P_free = 0.5 * (Z @ (V.T @ I_q)) + torch.outer(f_work, I_q.sum(dim=0))
        P = be.bvls(A_cov_Q.contiguous(), (P_free @ A_cov_Q).contiguous(), 0.0, 1.0)
        mapP(P)
        A_cov_P, Q_free = q_update(P)
        Q = be.bvls(A_cov_P.contiguous(), (Q_free @ A_cov_P).contiguous(), 0.0, 1.0)
        mapQ(Q)
        rmse = torch.sqrt(torch.mean((Q - Q0) ** 2))
        if bool(rmse < tol):
            log.info(f"        Convergence reached in iteration {i + 1}.")
            break
        Q0.copy_(Q)
    return P, Q


def initialize_sharded(G, N: int, M: int, j0: int, j1: int, K: int, seed: int, power: int, tol_svd: float,
                       max_als: int, tol_als: float, backend=None, group=None):
    """This rank's initial (P rows, Q) for K ancestries: frequencies of its SNPs, the sharded
    randomized SVD and ALS (the single-GPU ``initialize_k`` path, adamixture.py:182-250)."""
    be = backend or CudaInitBackend()
    f = be.frequencies(G, j1 - j0)
    U, S, V = svd_sharded(G, N, M, j0, j1, f, K, seed, power, tol_svd, be, group)
    return als_sharded(U, S, V, f, seed, M, j0, j1, K, max_als, tol_als, be, group)
