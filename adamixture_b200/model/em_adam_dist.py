"""Adam-EM sharded over GPUs by SNP rows (one process per GPU, ``torch.distributed``).

Each rank holds a contiguous range of packed genotype rows (4 SNPs per row), the matching
rows of P and its Adam moments, and a full replica of Q. One iteration:

1. the local E-step over the rank's SNPs gives A, B (its P rows) and its share of the
   Q-side statistics T (N x K);
2. one all-reduce (sum) of T -- the only per-iteration exchange (16 MB at N=200k, K=10);
3. the EM targets and the Adam move: P rows locally, Q replicated (every rank applies the
   same deterministic update to the same reduced T, so the replicas stay identical).

The per-sample observed counts q_bat are all-reduced once; the log-likelihood at each check
is a local float64 sum plus a scalar all-reduce. Control flow (priming, checks, best model,
lr decay, stop) is ``optimize_parameters_gpu``'s, on the global log-likelihood, so every
rank takes the same branches and the same collectives.

The statistics come from a backend object (``CudaBackend``: this library's kernels); the
host logic is independent of it, so the multi-rank path is also exercised on CPU ranks
with a float64 numpy backend in the tests.
"""
from __future__ import annotations

import logging

import torch
import torch.distributed as dist

log = logging.getLogger(__name__)


def shard_rows(M: int, world: int, rank: int) -> tuple[int, int]:
    """SNP range [j0, j1) of ``rank``: whole packed rows (4 SNPs), as even as possible."""
    rows = (M + 3) // 4
    r0 = rows * rank // world
    r1 = rows * (rank + 1) // world
    return min(4 * r0, M), min(4 * r1, M)


class CudaBackend:
    """E-step statistics, EM targets, Adam and log-likelihood on this library's kernels."""

    def __init__(self, precision: str | None = None):
        self.precision = precision

    def counts(self, G, M):
        from .. import ops

        return ops.sample_counts(G, M)

    def stats(self, G, P, Q, M, K):
        from .. import ops
        from .em_adam_gpu import resolve_precision

        prec = resolve_precision(K, self.precision)
        dt = ops.input_dtype(prec)
        return ops.em_stats(G, P.to(dt).contiguous(), Q.to(dt).contiguous(), M, prec)

    def targets(self, P, Q, A, B, T, q_bat):
        from .. import ops

        return ops.em_targets(P, Q, A, B, T, q_bat)

    def adam(self, P, Q, P_EM, Q_EM, st, t, lr, beta1, beta2, eps):
        from .. import ops

        ops.adam_step(P, Q, P_EM, Q_EM, st["mP"], st["vP"], st["mQ"], st["vQ"], t, lr, beta1, beta2, eps)

    def loglik(self, G, P, Q, M):
        """As the single-GPU optimiser's check: h in float64 for the float64 E-step, in
        float32 otherwise (the sum stays float64)."""
        from .. import ops
        from .em_adam_gpu import resolve_precision

        if resolve_precision(Q.shape[1], self.precision) == "f64":
            return ops.loglik_device(G, P, Q, M, "f64")
        return ops.loglik_device(G, P.float().contiguous(), Q.float().contiguous(), M, "f32")


class ShardedAdamEM:
    """One rank's state of the sharded Adam-EM: its P rows and their Adam moments, the
    replicated Q and its moments, the global sample counts."""

    def __init__(self, G, P, Q, M_local: int, K: int, beta1: float, beta2: float, reg_adam: float, lr: float,
                 group=None, backend=None):
        self.G, self.P, self.Q, self.M_local, self.K = G, P, Q, M_local, K
        self.beta1, self.beta2, self.reg_adam, self.lr = beta1, beta2, reg_adam, lr
        self.group = group
        self.be = backend or CudaBackend()
        self.q_bat = self.be.counts(G, M_local)
        dist.all_reduce(self.q_bat, group=group)
        self.st = {k: torch.zeros_like(P if k[1] == "P" else Q) for k in ("mP", "vP", "mQ", "vQ")}
        self.t = 0

    def iteration(self) -> None:
        """Local E-step, all-reduce of T, EM targets and the Adam move."""
        A, B, T = self.be.stats(self.G, self.P, self.Q, self.M_local, self.K)
        dist.all_reduce(T, group=self.group)
        P_EM, Q_EM = self.be.targets(self.P, self.Q, A, B, T, self.q_bat)
        self.t += 1
        self.be.adam(self.P, self.Q, P_EM, Q_EM, self.st, self.t, self.lr, self.beta1, self.beta2, self.reg_adam)

    def loglik(self) -> float:
        """Global log-likelihood (local float64 sum + scalar all-reduce)."""
        L = self.be.loglik(self.G, self.P, self.Q, self.M_local).reshape(1).to(torch.float64)
        dist.all_reduce(L, group=self.group)
        return float(L.item())


def optimize_parameters_dist(G, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K, M_local, N,
                             lr_decay, min_lr, patience, tol_adam, group=None, backend=None, trace=None):
    """Sharded Adam-EM: ``G``, ``P`` are this rank's SNP rows; ``Q`` is replicated (float64).
    Returns (best P rows, best Q) by the global log-likelihood, as optimize_parameters_gpu."""
    run = ShardedAdamEM(G, P, Q, M_local, K, beta1, beta2, reg_adam, lr, group, backend)
    run.iteration()  # priming
    L_best = run.loglik()
    P_best, Q_best = P.clone(), Q.clone()
    wait_lr = 0
    for it in range(max_iter):
        run.iteration()
        if (it + 1) % check == 0:
            L_cur = run.loglik()
            if trace is not None:
                trace.append((it + 1, L_cur))
            if L_cur > L_best + tol_adam:
                L_best = L_cur
                P_best.copy_(P)
                Q_best.copy_(Q)
                wait_lr = 0
            else:
                wait_lr += 1
                if wait_lr >= patience:
                    run.lr = max(run.lr * lr_decay, min_lr)
                    if run.lr <= min_lr:
                        break
                    wait_lr = 0
    return P_best, Q_best
