"""ALS initialisation of P and Q from the randomized SVD on one B200: drop-in for
``adamixture/model/als_gpu.py``.

Same public names and signatures (``mapP``, ``mapQ``, ``ALS_gpu``) and the same
iteration (als_gpu.py:45-127): random P from a seeded generator on the device, Q from the
SVD factors through the pseudo-inverse of P'P, then alternating bounded least-squares
updates of P and Q in [0, 1] with the RMSE stop on Q. The batched BVLS solves are this
library's warp-per-row kernel (``ops.bvls``); the K x K pseudo-inverses and the products
of the small factors are torch (cuBLAS / cuSOLVER), as in the reference.
"""
from __future__ import annotations

import logging
import time

import torch

from .. import ops

log = logging.getLogger(__name__)


def mapP(P_in: torch.Tensor) -> None:
    """Clamp P into [1e-5, 1 - 1e-5] in place (als_gpu.py:10-21)."""
    P_in.clamp_(min=1e-5, max=1.0 - 1e-5)


def mapQ(Q_in: torch.Tensor) -> None:
    """Clamp Q into [1e-5, 1 - 1e-5] and normalise its rows in place (als_gpu.py:23-36)."""
    Q_in.clamp_(min=1e-5, max=1.0 - 1e-5)
    Q_in.div_(Q_in.sum(dim=1, keepdim=True))


def ALS_gpu(U: torch.Tensor, S: torch.Tensor, V: torch.Tensor, f: torch.Tensor,
            seed: int, M: int, K: int, max_iter: int, tol: float,
            device: torch.device) -> tuple[torch.Tensor, torch.Tensor]:
    """P [M, K] and Q [N, K] (float64) from the rank-K SVD ``U S V'`` and frequencies ``f``."""
    if torch.device(device).type != "cuda":
        raise ValueError("adamixture_b200 runs on CUDA devices only")
    t0 = time.time()
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    dtype = torch.float64
    Z = (U * S).to(dtype)
    V = torch.as_tensor(V, device=device, dtype=dtype)
    V_T, Z_T = V.T, Z.T
    f_work = f.to(dtype)

    P = torch.rand((M, K), dtype=dtype, generator=gen, device=device)
    mapP(P)
    A_cov_P = P.T @ P
    I_p = P @ torch.linalg.pinv(A_cov_P)
    f_p = f_work.reshape(1, -1) @ I_p
    Q = 0.5 * (V @ (Z_T @ I_p)) + f_p
    mapQ(Q)
    Q0 = Q.clone()

    for i in range(max_iter):
        A_cov_Q = Q.T @ Q
        I_q = Q @ torch.linalg.pinv(A_cov_Q)
        P_free = 0.5 * (Z @ (V_T @ I_q)) + torch.outer(f_work, I_q.sum(dim=0))
        P = ops.bvls(A_cov_Q.contiguous(), (P_free @ A_cov_Q).contiguous(), 0.0, 1.0)
        mapP(P)

        A_cov_P = P.T @ P
        I_p = P @ torch.linalg.pinv(A_cov_P)
        f_p = f_work.reshape(1, -1) @ I_p
        Q_free = 0.5 * (V @ (Z_T @ I_p)) + f_p
        Q = ops.bvls(A_cov_P.contiguous(), (Q_free @ A_cov_P).contiguous(), 0.0, 1.0)
        mapQ(Q)

        rmse = torch.sqrt(torch.mean((Q - Q0) ** 2))
        if rmse < tol:
            log.info(f"        Convergence reached in iteration {i + 1}.")
            break
        Q0.copy_(Q)
    log.info(f"        Total ALS time={time.time() - t0:.3f}s\n")
    return P, Q
