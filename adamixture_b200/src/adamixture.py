"""Training driver of the B200 build: the GPU branches of ``adamixture/src/adamixture.py``
(``setup``, ``initialize_em_gpu``, ``initialize_k``, ``train_k``) with the same arguments
and flow -- frequencies and the randomized SVD once at K_max, then per K either SVD + ALS
or random + EM priming initialisation, followed by Adam-EM or SQP + ZAL (``original``).
Every step runs on the GPU through this library's kernels.
"""
from __future__ import annotations

import logging
import time

import numpy as np
import torch

from .. import ops
from ..model.als_gpu import ALS_gpu
from ..model.br_qn_gpu import optimize_original_gpu
from ..model.em_adam_gpu import EMAdamOptimizer, loglikelihood_gpu, optimize_parameters_gpu
from ..model.svd_gpu import SVD_gpu

log = logging.getLogger(__name__)

THREADS_PER_BLOCK = 256  # accepted for signature compatibility; kernels pick their own launch shapes


def _device(device) -> torch.device:
    d = torch.device("cuda" if device in ("gpu", "cuda") else device)
    if d.type != "cuda":
        raise ValueError("adamixture_b200 runs on CUDA devices only (use --device gpu)")
    if d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


def setup(G, N: int, M: int, K_max: int, seed: int, power: int, tol_svd: float, chunk_size: int,
          device: str, original: bool = False, init_original: str = "em", q_hist: int = 3,
          compute_svd: bool = True) -> tuple:
    """adamixture.py:23-106 (GPU branch): ``(device_obj, threads_per_block, f, U, S, V, G)``."""
    device_obj = _device(device)
    log.info(f"    Running on {str(device_obj).upper()}.\n")
    G = G.to(device_obj) if isinstance(G, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(G)).to(device_obj)
    if original and init_original == "em":
        log.info("    Skipping SVD; --original uses random + EM initialization.\n")
        return device_obj, THREADS_PER_BLOCK, None, None, None, None, G
    f = ops.allele_frequency(G, M)
    log.info("    Frequencies calculated.\n")
    U = S = V = None
    if compute_svd:
        log.info("    Running SVD on GPU...\n")
        U, S, V = SVD_gpu(G, N, M, f, K_max, seed, power, tol_svd, chunk_size, device_obj, THREADS_PER_BLOCK)
    return device_obj, THREADS_PER_BLOCK, f, U, S, V, G


def initialize_em_gpu(G, seed: int, M: int, N: int, K: int, device_obj, chunk_size: int,
                      threads_per_block: int, n_steps: int = 5):
    """Random P/Q from ``np.random.default_rng(seed)`` and ``n_steps`` plain EM steps
    (adamixture.py:140-179)."""
    rng = np.random.default_rng(seed)
    P_np = rng.random(size=(M, K), dtype=np.float64)
    Q_np = rng.random(size=(N, K), dtype=np.float64)
    np.clip(P_np, 1e-5, 1.0 - 1e-5, out=P_np)
    np.clip(Q_np, 1e-5, 1.0 - 1e-5, out=Q_np)
    Q_np /= Q_np.sum(axis=1, keepdims=True)
    P = torch.from_numpy(P_np).to(device_obj)
    Q = torch.from_numpy(Q_np).to(device_obj)
    opt = EMAdamOptimizer(P.shape, Q.shape, 0.0, 0.0, 0.0, 0.0, device_obj, precision="f64")
    t0 = time.time()
    for _ in range(n_steps):
        opt.run_em_step(G, P, Q, M, chunk_size, None)
        P.copy_(opt.P_EM)
        Q.copy_(opt.Q_EM)
    log.info(f"        Total EM initialization time={time.time() - t0:.3f}s\n")
    return P, Q


def initialize_k(G, N: int, M: int, K: int, f, seed: int, power: int, tol_svd: float, max_als: int,
                 tol_als: float, chunk_size: int, device_obj, threads_per_block: int,
                 original: bool = False, init_original: str = "em", em_init_steps: int = 5):
    """One initialisation for one K: ``(P, Q, logl)`` (adamixture.py:182-250, GPU branch)."""
    if original and init_original == "em":
        P, Q = initialize_em_gpu(G, seed, M, N, K, device_obj, chunk_size, threads_per_block, em_init_steps)
    else:
        U, S, V = SVD_gpu(G, N, M, f, K, seed, power, tol_svd, chunk_size, device_obj, threads_per_block)
        P, Q = ALS_gpu(U.contiguous(), S.contiguous(), V.contiguous(), f, seed, M, K, max_als, tol_als, device_obj)
    logl = loglikelihood_gpu(G, P, Q, M, N, chunk_size, device_obj, threads_per_block)
    log.info(f"    Initial log-likelihood for K={K}: {logl:.1f}.")
    return P, Q, logl


def train_k(G, N: int, M: int, K: int, U_max, S_max, V_max, f, seed: int, lr: float, beta1: float,
            beta2: float, reg_adam: float, max_iter: int, check: int, max_als: int, tol_als: float,
            lr_decay: float, min_lr: float, chunk_size: int, patience: int, tol_adam: float, device_obj,
            threads_per_block: int, original: bool = False, rtol: float = 1e-7, Q_hist: int = 3,
            init_original: str = "em", em_init_steps: int = 5, P_init=None, Q_init=None,
            precision: str | None = None):
    """Train one K from the shared SVD (adamixture.py:253-383, GPU branch): ``(P, Q)``."""
    if P_init is None and init_original == "mlp" and not original:
        # learned warm start, kept only if EM from it is no worse than plain EM from the
        # ALS start (both run; the better model is returned)
        from ..model import warm_start as ws

        net = ws.WarmStartMLP.load(ws.DEFAULT_WEIGHTS, device_obj)
        r = ws.warm_start_fit(net, G, N, M, K, seed, precision)
        log.info(f"    Warm start {'kept' if r['kept_warm'] else 'rejected'}: log-likelihood "
                 f"{r['loglik_warm']:.1f} (warm) vs {r['loglik_plain']:.1f} (plain).")
        return r["P"], r["Q"]
    if P_init is not None and Q_init is not None:
        P, Q = P_init, Q_init
    else:
        if original and init_original == "em":
            P, Q = initialize_em_gpu(G, seed, M, N, K, device_obj, chunk_size, threads_per_block, em_init_steps)
        else:
            log.info(f"    Running ALS on GPU ({device_obj})...")
            P, Q = ALS_gpu(U_max[:, :K].contiguous(), S_max[:K].contiguous(), V_max[:, :K].contiguous(), f,
                           seed, M, K, max_als, tol_als, device_obj)
        logl = loglikelihood_gpu(G, P, Q, M, N, chunk_size, device_obj, threads_per_block)
        log.info(f"    Initial log-likelihood for K={K}: {logl:.1f}.")
    if original:
        log.info(f"    SQP + ZAL QN running on GPU ({device_obj})...\n")
        return optimize_original_gpu(G, P, Q, max_iter, K, M, N, rtol, Q_hist, patience, device_obj,
                                     chunk_size, threads_per_block)
    log.info(f"    Adam-EM running on GPU ({device_obj})...\n")
    return optimize_parameters_gpu(G, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K, M, N, lr_decay,
                                   min_lr, patience, tol_adam, device_obj, chunk_size, threads_per_block,
                                   precision=precision)
