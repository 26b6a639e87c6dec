"""Shifted randomized SVD of the centred genotypes on one B200: drop-in for
``adamixture/model/svd_gpu.py``.

Same public names and signatures (``eigSVD_gpu``, ``SVD_gpu``) and the same algorithm
(svd_gpu.py:40-154): a prime pass against a Gaussian basis, ``power`` shifted power
iterations with the dynamic shift ``alpha`` and the relative singular-value stop, a final
projection, and the eigen-decomposition SVD of the small matrices. The passes over the
genotypes (decode, centre, multiply) are this library's fused kernels (``ops.rsvd_rows``
/ ``ops.rsvd_cols``), which read the packed matrix directly; the L x L eigenproblems and
the N x L / M x L products of small factors stay in torch, as in the reference.
``chunk_size`` and ``threads_per_block`` are accepted for signature compatibility.
The Gaussian basis comes from a torch generator on the genotypes' device seeded with
``seed``, as in the reference, so a CUDA run draws the reference's numbers.
"""
from __future__ import annotations

import logging
import time

import torch

from .. import ops

log = logging.getLogger(__name__)


def eigSVD_gpu(C: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """SVD of a short-wide ``C`` [L, n] through the eigendecomposition of ``C C'``
    (svd_gpu.py:11-38): returns ``U`` [n, L], ``S`` [L], ``V`` [L, L], largest first."""
    cov = C @ C.transpose(-2, -1)
    D, V = torch.linalg.eigh(cov)
    S = torch.sqrt(D)
    U = (C.transpose(-2, -1) @ V) / S
    idx = torch.arange(V.shape[1] - 1, -1, -1, device=C.device)
    return U[:, idx], S.flip(0), V[:, idx]


def _SVD_gpu_once(G, N, M, f, k, seed, power, tol, device):
    t0 = time.time()
    L = max(k + 10, 20)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    f = f.to(device=device, dtype=torch.float32).contiguous()
    proj = torch.randn((M, L), dtype=torch.float32, generator=gen, device=device)
    accum = ops.rsvd_cols(G, f, proj, M)                       # prime pass: X' Omega
    orth, _, _ = eigSVD_gpu(accum.T)
    alpha = torch.tensor(0.0, device=device)
    singular = torch.zeros(L, device=device)
    for i in range(power):
        ops.rsvd_rows(G, f, orth, M, out=proj)                 # proj = X orth
        ops.rsvd_cols(G, f, proj, M, out=accum)                # accum = X' proj
        Qm, S, _ = eigSVD_gpu(accum.sub(orth, alpha=alpha.item()).T)
        if i > 0:
            s_cur = S + alpha
            rel = torch.abs(s_cur - singular) / torch.maximum(s_cur, torch.tensor(1e-12, device=device))
            if torch.max(rel[:k]) < tol:
                log.info(f"        Converged at iteration {i}.")
                break
            singular.copy_(s_cur)
        else:
            singular.copy_(S + alpha)
        if S[-1] > alpha:
            alpha = 0.5 * (S[-1] + alpha)
        orth.copy_(Qm)
    ops.rsvd_rows(G, f, orth, M, out=proj)                     # final projection
    u_c, s_all, v_c = eigSVD_gpu(proj.T)
    S_final = s_all[:k].contiguous()
    U_final = u_c[:, :k].contiguous()
    V_final = (orth @ v_c[:, :k]).contiguous()
    log.info(f"\n    Total time for SVD={time.time() - t0:.3f}s")
    return U_final, S_final, V_final


def SVD_gpu(G: torch.Tensor, N: int, M: int, f: torch.Tensor, k: int, seed: int,
            power: int, tol: float, chunk_size: int, device: torch.device,
            threads_per_block: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Rank-``k`` randomized SVD of the centred packed genotypes: ``(U [M,k], S [k], V [N,k])``."""
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    return _SVD_gpu_once(G, N, M, f, k, seed, power, tol, G.device)
