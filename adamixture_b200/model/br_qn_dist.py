"""The original ADMIXTURE algorithm (block-relaxation SQP with ZAL quasi-Newton acceleration)
sharded over GPUs by SNP rows, one process per GPU: the iteration of ``br_qn_gpu``
(adamixture/model/br_qn_gpu.py:217-382) when each rank holds a contiguous range of whole
packed rows (``em_adam_dist.shard_rows``), its rows of P and a replica of Q.

Per iteration (two SQP block updates of Q and P, the extrapolation, the acceptance test):

* Q side: the gradient/Hessian pass over the rank's SNPs gives its share of XtX_q [N,K,K]
  and Xtz_q [N,K]; one all-reduce of each (N K (K+1) doubles: 176 MB at N=200k, K=10), then
  every rank runs the same per-sample SQP solves, so the Q replicas stay identical;
* P side: the pass and the per-SNP solves are local (they need all of Q, which every rank
  has);
* ZAL: the secant system U'(U - V) alpha = U'(x0 - x1) is q x q; its P rows are summed over
  the ranks (one all-reduce of q x q and q values), its Q rows are counted once (they are
  replicated); the extrapolated point is then local (P rows) or replicated (Q);
* the log-likelihood of a candidate: a local float64 sum and one scalar all-reduce.

Every decision (acceptance, best iterate, tolerance and patience stops) is taken on
replicated values, so every rank takes the same branches and collectives. Results equal a
one-process run of the same code up to the summation order of the all-reduced sums.

The passes, solves and log-likelihood come from a backend (``CudaBrqnBackend``: this
library's kernels); the host logic does not depend on it, so the multi-rank path also runs on
CPU ranks with a float64 backend in the tests.
"""
from __future__ import annotations

import logging

import torch

from .br_qn_gpu import _mapPQ_gpu, _v_kk
from .init_dist import _sum

log = logging.getLogger(__name__)


class CudaBrqnBackend:
    """Gradient/Hessian passes over this rank's packed rows, the per-row SQP solves and the
    float64 log-likelihood on this library's kernels."""

    def grad_hess_q(self, G, P, Q, M_local):
        from .. import ops

        return ops.grad_hess_q(G, P, Q, M_local)

    def grad_hess_p(self, G, P, Q, M_local):
        from .. import ops

        return ops.grad_hess_p(G, P, Q, M_local)

    def sqp_q(self, XtX, Xtz_neg, Q, v_kk):
        from .. import ops

        N, K = Q.shape
        return ops.sqp_solve_q(XtX, Xtz_neg, Q, v_kk, N, K)

    def sqp_p(self, XtX, Xtz_neg, P):
        from .. import ops

        M, K = P.shape
        return ops.sqp_solve_p(XtX, Xtz_neg, P, M, K)

    def loglik(self, G, P, Q, M_local):
        from .. import ops

        return ops.loglik_device(G, P, Q, M_local, "f64").reshape(1)


def optimize_original_dist(G, P, Q, max_iter: int, K: int, M_local: int, N: int, tol: float, Q_hist: int,
                           patience: int, backend=None, group=None, verbose: bool = True):
    """Sharded SQP + ZAL QN from this rank's P rows and the replicated Q (float64, updated
    in place). Returns (best P rows, best Q) by the global log-likelihood."""
    be = backend or CudaBrqnBackend()
    dev, dt = P.device, torch.float64
    v_kk = _v_kk(K, dev)
    mk = M_local * K
    dim = mk + N * K
    U = torch.zeros((dim, Q_hist), dtype=dt, device=dev)
    V = torch.zeros((dim, Q_hist), dtype=dt, device=dev)
    x0, x1, x2 = (torch.empty(dim, dtype=dt, device=dev) for _ in range(3))
    P_qn, Q_qn = torch.empty_like(P), torch.empty_like(Q)

    def flat(Pm, Qm, out):
        out[:mk].copy_(Pm.ravel())
        out[mk:].copy_(Qm.ravel())

    def sqp_q(Pm, Qm):
        XtX, Xtz = be.grad_hess_q(G, Pm, Qm, M_local)
        _sum(XtX, group)
        _sum(Xtz, group)
        return be.sqp_q(XtX, Xtz.neg_(), Qm, v_kk)

    def sqp_p(Pm, Qm):
        XtX, Xtz = be.grad_hess_p(G, Pm, Qm, M_local)
        return be.sqp_p(XtX, Xtz.neg_(), Pm)

    def logl(Pm, Qm):
        return float(_sum(be.loglik(G, Pm, Qm, M_local).to(dt), group).item())

    def dot(A, B):
        """A' B over the sharded vector layout: P rows summed over the ranks, Q rows once."""
        return _sum(A[:mk].T @ B[:mk], group) + A[mk:].T @ B[mk:]

    ll_prev = -float("inf")
    ll_best = -float("inf")
    wait = 0
    P_best, Q_best = P.clone(), Q.clone()
    for it in range(1, max_iter + 1):
        Q1 = sqp_q(P, Q)
        P1 = sqp_p(P, Q1)
        Q2 = sqp_q(P1, Q1)
        P2 = sqp_p(P1, Q2)

        flat(P, Q, x0)
        flat(P1, Q1, x1)
        flat(P2, Q2, x2)
        col = (it - 1) % Q_hist
        torch.sub(x1, x0, out=U[:, col])
        torch.sub(x2, x1, out=V[:, col])
        n_cols = min(it, Q_hist)
        U_s, V_s = U[:, :n_cols], V[:, :n_cols]
        LHS = dot(U_s, U_s - V_s)
        RHS = dot(U_s, (x0 - x1).reshape(-1, 1)).reshape(-1)
        try:
            alpha = torch.linalg.solve(LHS, RHS)
        except RuntimeError:
            alpha = torch.linalg.lstsq(LHS, RHS).solution
        x_qn = x1 - V_s @ alpha
        P_qn.copy_(x_qn[:mk].view(M_local, K))
        Q_qn.copy_(x_qn[mk:].view(-1, K))
        _mapPQ_gpu(P_qn, Q_qn)

        ll_qn = logl(P_qn, Q_qn)
        if ll_qn > ll_prev:
            P.copy_(P_qn)
            Q.copy_(Q_qn)
            ll_new = ll_qn
        else:
            P.copy_(P2)
            Q.copy_(Q2)
            ll_new = logl(P2, Q2)

        best_before = ll_best
        if ll_new > ll_best:
            ll_best = ll_new
            P_best.copy_(P)
            Q_best.copy_(Q)
        if best_before != -float("inf") and ll_new <= best_before + tol:
            wait += 1
        else:
            wait = 0
        if verbose:
            log.info(f"    Iteration {it}, Log-likelihood: {ll_new:.1f}")
        if abs(ll_new - ll_prev) < tol:
            break
        if wait >= patience:
            break
        ll_prev = ll_new
    return P_best, Q_best
