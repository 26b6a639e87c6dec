"""Supervised mode on one B200: drop-in for the GPU functions of
``adamixture/src/supervised.py``.

Labelled samples (y > 0, population y in 1..K) keep a near-one-hot Q row (1 - eps on their
population, eps / (K - 1) elsewhere); P starts from the labelled samples' allele
frequencies. The E-step, targets and Adam move are the unsupervised kernels; after every
update the labelled rows are snapped back (supervised.py:308-462). The SQP + ZAL form snaps
after each Q solve and after the extrapolated point (supervised.py:602-760).

Parity note: the reference's Adam-EM loop decays a local copy of the learning rate that
its optimiser never reads (supervised.py:441-451): the Adam step keeps the initial rate and
the decayed copy only drives the stop. This package does the same, so it returns the same
model.
"""
from __future__ import annotations

import logging
import time

import numpy as np
import torch

from .. import ops
from ..model.br_qn_gpu import _optimize_original_gpu_once
from ..model.em_adam_gpu import EMAdamOptimizer, loglikelihood_gpu

log = logging.getLogger(__name__)


def init_q_supervised(Q: np.ndarray, y: np.ndarray, K: int, eps: float = 1e-5) -> None:
    """Near-one-hot rows for labelled samples, unlabelled rows renormalised (in place;
    supervised.py:20-46)."""
    fill = eps / max(K - 1, 1)
    lab = np.where(y > 0)[0]
    Q[lab, :] = fill
    Q[lab, y[lab] - 1] = 1.0 - eps
    un = y == 0
    Q[un] /= Q[un].sum(axis=1, keepdims=True)


def init_p_supervised_gpu(G: torch.Tensor, y: np.ndarray, K: int, M: int, eps: float = 1e-5) -> torch.Tensor:
    """Per-population allele frequencies of the labelled samples, 0.5 where a population has
    no observed labelled genotype, clipped to [eps, 1 - eps] (supervised.py:49-109), from
    two products of the packed genotypes with the label indicator matrix."""
    N = G.shape[1]
    ind = np.zeros((N, K), dtype=np.float32)
    lab = np.where(y > 0)[0]
    ind[lab, y[lab] - 1] = 1.0
    B = torch.from_numpy(ind).to(G.device)
    zero = torch.zeros(M, dtype=torch.float32, device=G.device)
    half = torch.full((M,), 0.5, dtype=torch.float32, device=G.device)
    num = ops.rsvd_rows(G, zero, B, M).double()           # sum of g over observed labelled
    den = 2.0 * (num - ops.rsvd_rows(G, half, B, M).double())   # 2 x observed labelled
    P = torch.where(den > 0, num / den.clamp_min(1e-300), torch.full_like(num, 0.5))
    return P.clamp(eps, 1.0 - eps)


def snap_q_gpu(Q: torch.Tensor, y: np.ndarray, K: int, eps: float = 1e-5) -> None:
    """Labelled rows back to their near-one-hot value, in place (supervised.py:308-339)."""
    lab = np.where(y > 0)[0]
    if len(lab) == 0:
        return
    rows = np.full((len(lab), K), eps / max(K - 1, 1))
    rows[np.arange(len(lab)), y[lab] - 1] = 1.0 - eps
    Q[torch.from_numpy(lab).to(Q.device)] = torch.from_numpy(rows).to(Q.device, Q.dtype)


def optimize_supervised_gpu(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, y: np.ndarray,
                            lr: float, beta1: float, beta2: float, reg_adam: float,
                            max_iter: int, check: int, M: int,
                            lr_decay: float, min_lr: float, patience: int, tol_adam: float,
                            device: torch.device, chunk_size: int, threads_per_block: int,
                            precision: str | None = "f64"):
    """Supervised Adam-EM (supervised.py:342-462): ``(P_best, Q_best)``."""
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    N, K = Q.shape
    P = P.to(device=G.device, dtype=torch.float64).clone().contiguous()
    Q = Q.to(device=G.device, dtype=torch.float64).clone().contiguous()
    opt = EMAdamOptimizer(P.shape, Q.shape, lr, beta1, beta2, reg_adam, G.device, precision)
    shadows = opt.precision != "f64"
    P32 = P.float().contiguous() if shadows else None
    Q32 = Q.float().contiguous() if shadows else None
    ws = ops.Workspace.get(G.device, ops.em_workspace_bytes(M, N, K, opt.precision))

    def step():
        opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
        snap_q_gpu(Q, y, K)
        if shadows:
            Q32.copy_(Q)

    def logl():
        return loglikelihood_gpu(G, P, Q, M, N, chunk_size, G.device, threads_per_block)

    step()  # priming (the reference's following E-step changes no state)
    L_best = logl()
    P_best, Q_best = P.clone(), Q.clone()
    wait_lr = 0
    ts = time.time()
    for it in range(max_iter):
        step()
        if (it + 1) % check == 0:
            L_cur = logl()
            log.info(f"    Iteration {it + 1}, Log-likelihood: {L_cur:.1f}, Time: {time.time() - ts:.3f}s")
            ts = time.time()
            if L_cur > L_best + tol_adam:
                L_best = L_cur
                P_best.copy_(P)
                Q_best.copy_(Q)
                wait_lr = 0
            else:
                wait_lr += 1
                if wait_lr >= patience:
                    lr = max(lr * lr_decay, min_lr)   # the reference's local copy (see above)
                    if lr <= min_lr:
                        break
                    wait_lr = 0
    log.info(f"\n    Final log-likelihood (supervised): {L_best:.1f}")
    return P_best, Q_best


def optimize_supervised_original_gpu(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, y: np.ndarray,
                                     max_iter: int, K: int, M: int, N: int, tol: float, Q_hist: int,
                                     patience: int, device: torch.device, chunk_size: int,
                                     threads_per_block: int, qn_projection: str = "clamp"):
    """Supervised SQP + ZAL QN (supervised.py:602-760): ``(P_best, Q_best)``.
    ``qn_projection``: "clamp" as the reference's GPU path, "simplex" as its CPU path
    (supervised.py:556-558)."""
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    P = P.to(device=G.device, dtype=torch.float64).clone().contiguous()
    Q = Q.to(device=G.device, dtype=torch.float64).clone().contiguous()
    return _optimize_original_gpu_once(G, P, Q, max_iter, K, M, N, tol, Q_hist, patience, G.device,
                                       qn_projection=qn_projection, q_hook=lambda Qm: snap_q_gpu(Qm, y, K))
