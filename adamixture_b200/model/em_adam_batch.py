"""Several Adam-EM fits on one cohort at once: the K sweep and its cross-validation folds.

The reference runs the K sweep one K at a time (adamixture/src/main.py:67-107) and its
cross-validation per K and fold afterwards (adamixture/src/cv.py:171-267). Here a list of
problems -- each with its own K (<= 16), start, Adam state and learning-rate schedule, and
optionally a cross-validation fold whose entries it treats as missing -- advances together:
every iteration is one launch of the batched float64 E-step sweep per tile layout in use
(one launch, or two when the autotuner runs the K <= 8 problems on the two-CTA-per-SM
layout and the others on the default one), then each problem's EM targets and Adam move. Each CTA of the sweep runs the problems in order over its share of
the matrix, so problems on the same genotypes (all full-data fits; all problems of one
fold) read them from memory once and from L2 after that.

Fold rule: entry (j, i) belongs to bucket ``h(j*N + i, seed) mod n_buckets`` with h the
reference's cross-validation hash (cv.py:58-78); fold f holds out bucket f. With
``n_buckets=10`` and folds 0..4, each fold masks 10 % of the entries. A fold's problems
share one copy of the packed matrix with the fold's entries hidden.

Every problem follows exactly the single-problem path's arithmetic and control flow
(``optimize_parameters_gpu`` at float64 for full-data problems; plain Adam-EM iterations
for fold problems), so its results are bit-identical to running it alone on the same
(masked) genotypes -- ``cross_validate(..., batched=False)`` does exactly that, through
the single-problem kernels, for comparison.
"""
from __future__ import annotations

import logging
import time
from dataclasses import dataclass, field

import torch

from .. import ops, tune
from .em_adam_gpu import EMAdamOptimizer, optimize_parameters_gpu

log = logging.getLogger(__name__)

HP = dict(lr=0.005, beta1=0.80, beta2=0.88, eps=1e-8)


@dataclass
class Problem:
    """One fit: K, its start, and the fold it holds out (-1: none)."""

    K: int
    P: torch.Tensor
    Q: torch.Tensor
    fold: int = -1
    # state
    mP: torch.Tensor | None = None
    vP: torch.Tensor | None = None
    mQ: torch.Tensor | None = None
    vQ: torch.Tensor | None = None
    q_bat: torch.Tensor | None = None
    G: torch.Tensor | None = None
    t: float = 0.0
    lr: float = HP["lr"]
    L_best: float = float("-inf")
    P_best: torch.Tensor | None = None
    Q_best: torch.Tensor | None = None
    wait: int = 0
    active: bool = True
    iterations: int = 0
    trace: list = field(default_factory=list)


def fold_copy(G: torch.Tensor, M: int, seed: int, n_buckets: int, fold: int) -> torch.Tensor:
    """A copy of the packed genotypes with bucket ``fold`` of the hash rule hidden."""
    Gm = ops.masked_copy(G)
    ops.cv_mask_hash(Gm, G, M, seed, n_buckets, fold)
    return Gm


def fold_counts(G: torch.Tensor, M: int, seed: int, n_buckets: int, fold: int) -> torch.Tensor:
    """q_bat of the genotypes with fold ``fold`` hidden: 2 x observed entries per sample."""
    return ops.sample_counts(fold_copy(G, M, seed, n_buckets, fold), M)


def _prepare(G, M, problems, seed, n_buckets):
    """Start state of every problem; each fold's masked copy and counts made once."""
    shared = {}
    for pr in problems:
        pr.P = pr.P.to(torch.float64).contiguous().clone()
        pr.Q = pr.Q.to(torch.float64).contiguous().clone()
        pr.mP, pr.vP = torch.zeros_like(pr.P), torch.zeros_like(pr.P)
        pr.mQ, pr.vQ = torch.zeros_like(pr.Q), torch.zeros_like(pr.Q)
        if pr.fold not in shared:
            Gf = G if pr.fold < 0 else fold_copy(G, M, seed, n_buckets, pr.fold)
            shared[pr.fold] = (Gf, ops.sample_counts(Gf, M))
        pr.G, pr.q_bat = shared[pr.fold]


def _iteration(M, N, live):
    """One batched sweep over the live problems, then each one's targets + Adam move. A
    batched sweep launches one tile layout, so problems whose K runs another layout (the
    autotuner's choice, ``tune.batch_groups``) go in a launch of their own."""
    for idx in tune.batch_groups([p.K for p in live], live[0].G.device):
        group = [live[i] for i in idx]
        batch = ops.EmBatch(M, N, [p.K for p in group], group[0].G.device)
        batch.sweep([p.G for p in group], [p.P for p in group], [p.Q for p in group])
        for k, pr in enumerate(group):
            pr.t += 1.0
            batch.adam(k, pr.P, pr.Q, pr.mP, pr.vP, pr.mQ, pr.vQ, pr.q_bat, pr.t, pr.lr, HP["beta1"],
                       HP["beta2"], HP["eps"])
            pr.iterations += 1


def _tune(G, M, problems):
    """The float64 sweep's layout for every K of the batch (once per shape and K)."""
    seen = set()
    for pr in problems:
        if pr.K not in seen and pr.K <= 16:
            seen.add(pr.K)
            tune.tune_dmma(pr.G, pr.P, pr.Q, M)


def optimize_batch(G, M, N, problems, seed=0, n_buckets=10, max_iter=10000, check=5, lr_decay=0.5,
                   min_lr=1e-4, patience=3, tol=0.1, fixed_iters=None):
    """Advance every problem together.

    ``fixed_iters=None``: each full-data problem runs the reference loop
    (adamixture/model/em_adam_gpu.py:281-356, as ``optimize_parameters_gpu``): priming, a
    float64 log-likelihood check every ``check`` iterations, best checkpoint, learning-rate
    decay after ``patience`` flat checks, stop at ``min_lr``; the result is its best P, Q.
    A problem leaves the batch when it stops. ``fixed_iters=n``: every problem runs exactly
    n Adam-EM iterations (the first one from the start) and keeps its last iterate.
    Returns the problems (results in ``P_best``/``Q_best``)."""
    problems = sorted(problems, key=lambda p: p.fold)   # problems on the same genotypes adjacent
    _prepare(G, M, problems, seed, n_buckets)
    _tune(G, M, problems)
    if fixed_iters is not None:
        for _ in range(int(fixed_iters)):
            _iteration(M, N, problems)
        for pr in problems:
            pr.P_best, pr.Q_best = pr.P, pr.Q
        return problems
    if any(p.fold >= 0 for p in problems):
        raise ValueError("fold problems run a fixed number of iterations (fixed_iters)")
    # priming: one iteration, then the primed point's log-likelihood is the first best
    _iteration(M, N, problems)
    for pr in problems:
        pr.L_best = float(ops.loglik_device(G, pr.P, pr.Q, M, "f64").item())
        pr.P_best, pr.Q_best = pr.P.clone(), pr.Q.clone()
    for it in range(max_iter):
        live = [p for p in problems if p.active]
        if not live:
            break
        _iteration(M, N, live)
        if (it + 1) % check:
            continue
        for pr in live:
            L = float(ops.loglik_device(G, pr.P, pr.Q, M, "f64").item())
            pr.trace.append((it + 1, L))
            if L > pr.L_best + tol:
                pr.L_best = L
                pr.P_best.copy_(pr.P)
                pr.Q_best.copy_(pr.Q)
                pr.wait = 0
            else:
                pr.wait += 1
                if pr.wait >= patience:
                    pr.lr = max(pr.lr * lr_decay, min_lr)
                    if pr.lr <= min_lr:
                        pr.active = False
                    pr.wait = 0
    return problems


def _fit_alone(G, M, N, pr, max_iter, check, lr_decay, min_lr, patience, tol):
    P, Q = optimize_parameters_gpu(G, pr.P, pr.Q, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], max_iter, check,
                                   pr.K, M, N, lr_decay, min_lr, patience, tol, G.device, 8192, 256,
                                   precision="f64")
    return P, Q


def _polish_alone(G, M, N, P0, Q0, K, fold, seed, n_buckets, n_iters):
    Gm = fold_copy(G, M, seed, n_buckets, fold)
    P, Q = P0.clone(), Q0.clone()
    opt = EMAdamOptimizer(P.shape, Q.shape, HP["lr"], HP["beta1"], HP["beta2"], HP["eps"], G.device, "f64")
    ws = ops.Workspace.get(G.device, ops.em_workspace_bytes(M, N, K, "f64"))
    for _ in range(n_iters):
        opt.fused_iteration(Gm, P, Q, None, None, M, ws)
    del Gm
    return P, Q


def cross_validate(G, M, N, Ks, starts, n_folds=5, n_buckets=10, seed=42, polish_iters=10, max_iter=300,
                   check=5, lr_decay=0.5, min_lr=1e-4, patience=3, tol=0.1, batched=True):
    """Fit every K of ``Ks`` from ``starts[K] = (P0, Q0)``, then cross-validate each fit.

    Stage 1: the full-data fits (Adam-EM to the reference's stop rule). Stage 2: for each K
    and fold f < n_folds, ``polish_iters`` Adam-EM iterations from the K's fit with bucket f
    of the hash rule held out; the fold's score is the binomial deviance of its held-out
    entries (deviance_squared_sum, adamixture/src/utils_c/cython/br_qn.pyx:92-150). The CV
    index of K is the summed deviance over its folds divided by their held-out entries.
    ``batched=True`` runs each stage's problems together (one sweep launch per iteration);
    ``batched=False`` runs them one at a time through the single-problem path.
    Returns a dict: fits {K: (P, Q)}, folds {(K, f): (P, Q)}, cv {K: index}, seconds per stage.
    """
    dev = G.device
    out = {"fits": {}, "folds": {}, "cv": {}, "seconds": {}}
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    if batched:
        probs = [Problem(K, starts[K][0], starts[K][1]) for K in Ks]
        optimize_batch(G, M, N, probs, seed, n_buckets, max_iter, check, lr_decay, min_lr, patience, tol)
        for pr in probs:
            out["fits"][pr.K] = (pr.P_best, pr.Q_best)
    else:
        for K in Ks:
            pr = Problem(K, starts[K][0], starts[K][1])
            out["fits"][K] = _fit_alone(G, M, N, pr, max_iter, check, lr_decay, min_lr, patience, tol)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    if batched:
        probs = [Problem(K, *out["fits"][K], fold=f) for f in range(n_folds) for K in Ks]
        optimize_batch(G, M, N, probs, seed, n_buckets, fixed_iters=polish_iters)
        for pr in probs:
            out["folds"][(pr.K, pr.fold)] = (pr.P_best, pr.Q_best)
    else:
        for K in Ks:
            for f in range(n_folds):
                out["folds"][(K, f)] = _polish_alone(G, M, N, *out["fits"][K], K, f, seed, n_buckets, polish_iters)
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    total_obs = float(ops.sample_counts(G, M).sum().item()) / 2.0
    held = {f: total_obs - float(fold_counts(G, M, seed, n_buckets, f).sum().item()) / 2.0 for f in range(n_folds)}
    for K in Ks:
        dev_sum = sum(ops.cv_deviance_hash(G, *out["folds"][(K, f)], M, seed, n_buckets, f) for f in range(n_folds))
        out["cv"][K] = dev_sum / sum(held.values())
    out["seconds"] = {"fits": t1 - t0, "folds": t2 - t1}
    out["held_out"] = held
    return out
