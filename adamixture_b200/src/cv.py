"""Cross-validation of a fitted model on one B200: drop-in for ``run_cross_validation`` of
``adamixture/src/cv.py`` (which always runs on the CPU there).

Same fold rules and score (cv.py:58-267): the observed entries are split into ``args.cv``
folds, either by the reference's shuffled list (``np.random.default_rng(seed).shuffle`` of
the observed flat indices, fold f = ``shuffled[f::v]``; used when M*N fits in int32) or
by its deterministic hash of the flat index (larger matrices); each fold's entries are
hidden, the global fit is polished by exactly 5 SQP + ZAL iterations (the CPU reference's
``polish_sqp_qn``, simplex projection of the extrapolated point), and the binomial deviance
of the held-out entries is summed. The CV index is the total over folds divided by the
number of observed entries. Hiding, polishing and scoring run on the GPU over a masked copy
of the packed matrix (``ops.cv_mask_*``, ``ops.cv_deviance_*``); only the shuffled list is
drawn on the host, with the reference's generator, so the folds are the reference's.
"""
from __future__ import annotations

import logging
from argparse import Namespace

import numpy as np
import torch

from .. import ops
from ..model.br_qn_gpu import polish_sqp_qn
from .packing import pack

log = logging.getLogger(__name__)

INT32_MAX = np.iinfo(np.int32).max


def observed_flat_indices(G: torch.Tensor, M: int, chunk: int = 1 << 15) -> np.ndarray:
    """Flat indices j*N + i of the observed entries, increasing (np.flatnonzero(G != 3))."""
    N = G.shape[1]
    out = []
    for m0 in range(0, M, chunk):
        u = ops.unpack_u8(G, m0, min(chunk, M - m0), M)
        nz = torch.nonzero(u.view(-1) != 3).view(-1)
        out.append((nz + m0 * N).cpu().numpy())
    return np.concatenate(out) if out else np.zeros(0, dtype=np.int64)


def shuffle_observed(flat: np.ndarray, seed: int) -> np.ndarray:
    """int32 observed flat indices shuffled by the reference's generator (cv.py:23-38)."""
    shuffled = np.asarray(flat).astype(np.int32, copy=True)
    np.random.default_rng(seed).shuffle(shuffled)
    return shuffled


def fold_lists(G: torch.Tensor, M: int, n_folds: int, seed: int) -> list[np.ndarray]:
    """The reference's shuffled-list folds: fold f = shuffled[f::n_folds] (cv.py:202-222)."""
    shuffled = shuffle_observed(observed_flat_indices(G, M), seed)
    return [shuffled[f::n_folds] for f in range(n_folds)]


def hash_fold_mask(flat: np.ndarray, seed: int, n_folds: int, fold: int) -> np.ndarray:
    """The reference's hash fold rule on host indices (cv.py:58-78), for checks."""
    h = flat.astype(np.uint64) + np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15)
    h ^= h >> np.uint64(30)
    h *= np.uint64(0xBF58476D1CE4E5B9)
    h ^= h >> np.uint64(27)
    h *= np.uint64(0x94D049BB133111EB)
    h ^= h >> np.uint64(31)
    return (h % np.uint64(n_folds)) == np.uint64(fold)


def run_cross_validation(args: Namespace, G, N: int, M: int, K: int, P_global, Q_global,
                         fold_rule: str = "auto", polish_iters: int = 5) -> float:
    """CV index of the fit (P_global, Q_global). ``G``: packed CUDA tensor [ceil(M/4), N], or
    the reference's unpacked uint8 array [M, N] (packed and moved to the current device).
    ``fold_rule``: "auto" (the reference's choice by size), "list" or "hash"."""
    if not isinstance(G, torch.Tensor):
        G = np.asarray(G)
        if G.shape != (M, N):
            raise ValueError(f"CV requires a genotype matrix with shape {(M, N)}, got {G.shape}.")
        G = torch.from_numpy(pack(G)).cuda()
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    dev = G.device
    P_global = torch.as_tensor(P_global, dtype=torch.float64).to(dev)
    Q_global = torch.as_tensor(Q_global, dtype=torch.float64).to(dev)
    n_folds, seed = int(args.cv), int(args.seed)
    use_hash = fold_rule == "hash" or (fold_rule == "auto" and M * N > INT32_MAX)
    if use_hash:
        n_obs = int(ops.sample_counts(G, M).sum().item()) // 2
        folds = None
    else:
        folds = fold_lists(G, M, n_folds, seed)
        n_obs = sum(len(f) for f in folds)
    if n_obs == 0:
        raise ValueError("No non-missing genotypes available for cross-validation.")
    cv_sum = 0.0
    for fold in range(n_folds):
        Gm = ops.masked_copy(G)
        if use_hash:
            ops.cv_mask_hash(Gm, G, M, seed, n_folds, fold)
        else:
            if len(folds[fold]) == 0:
                continue
            idx = torch.from_numpy(folds[fold].astype(np.int64)).to(dev)
            ops.cv_mask_list(Gm, M, idx)
        P_cv, Q_cv = polish_sqp_qn(Gm, P_global, Q_global, M, N, K, n_iters=polish_iters, Q_hist=3)
        if use_hash:
            cv_sum += ops.cv_deviance_hash(G, P_cv, Q_cv, M, seed, n_folds, fold)
        else:
            cv_sum += ops.cv_deviance_list(G, P_cv, Q_cv, M, idx)
        del Gm
    return cv_sum / float(n_obs)
