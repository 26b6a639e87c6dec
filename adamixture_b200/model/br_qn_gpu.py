"""Original ADMIXTURE algorithm (block-relaxation SQP with ZAL quasi-Newton acceleration)
on one B200: drop-in for ``adamixture/model/br_qn_gpu.py``.

Same public names and signatures (``compute_grad_hess_Q_gpu``, ``compute_grad_hess_P_gpu``,
``optimize_original_gpu``) and the same iteration (br_qn_gpu.py:217-382): two SQP block
updates (Q then P, each from its gradient/Hessian pass), the ZAL secant extrapolation over
the last ``Q_hist`` updates, acceptance by log-likelihood, best-iterate tracking and the
tolerance / patience stops. The gradient/Hessian passes read the packed genotypes directly
(``ops.grad_hess_q/p``, float64), the per-row QPs run one warp per row (``ops.sqp_solve_q/p``)
and the log-likelihood is this library's reduction; the q x q secant solve and the
(M+N)K-long vector updates are torch, as in the reference. ``chunk_size``, ``unpacker``
and ``threads_per_block`` are accepted for signature compatibility.
"""
from __future__ import annotations

import logging
import time

import torch

from .. import ops
from .em_adam_gpu import loglikelihood_gpu

log = logging.getLogger(__name__)


def _mapPQ_gpu(P: torch.Tensor, Q: torch.Tensor) -> None:
    """br_qn_gpu.py:47-61."""
    torch.clamp_(P, 1e-5, 1.0 - 1e-5)
    torch.clamp_(Q, 1e-5, 1.0 - 1e-5)
    Q.div_(Q.sum(dim=1, keepdim=True))


def compute_grad_hess_Q_gpu(G, Q, P, XtX_q, Xtz_q, M, chunk_size=None, unpacker=None, dtype=None) -> None:
    """Fill ``XtX_q`` [N,K,K] and ``Xtz_q`` [N,K] (br_qn_gpu.py:145-179)."""
    ops.grad_hess_q(G, P, Q, M, XtX_q, Xtz_q)


def compute_grad_hess_P_gpu(G, Q, P, XtX_p, Xtz_p, M, chunk_size=None, unpacker=None, dtype=None) -> None:
    """Fill ``XtX_p`` [M,K,K] and ``Xtz_p`` [M,K] (br_qn_gpu.py:182-214)."""
    ops.grad_hess_p(G, P, Q, M, XtX_p, Xtz_p)


def _v_kk(K: int, device) -> torch.Tensor:
    """Right singular vectors of ones(1, K), computed on the CPU as the reference does."""
    _, _, vt = torch.linalg.svd(torch.ones((1, K), dtype=torch.float64), full_matrices=True)
    return vt.t().to(device=device, dtype=torch.float64).contiguous()


def _optimize_original_gpu_once(G, P, Q, max_iter, K, M, N, tol, Q_hist, patience, device,
                                qn_projection="clamp", verbose=True, q_hook=None):
    """``qn_projection``: how the extrapolated point returns to the feasible set -- "clamp"
    (clamp and renormalise, the GPU reference, br_qn_gpu.py:341) or "simplex" (box for P,
    simplex projection for Q, the CPU reference, adamixture/model/br_qn.py:157-158).
    ``q_hook(Q)``: applied in place to every new Q (both SQP updates and the extrapolated
    point), as supervised mode snaps labelled rows (adamixture/src/supervised.py:602-760)."""
    dt = torch.float64
    v_kk = _v_kk(K, device)
    XtX_q = torch.zeros((N, K, K), dtype=dt, device=device)
    Xtz_q = torch.zeros((N, K), dtype=dt, device=device)
    XtX_p = torch.zeros((M, K, K), dtype=dt, device=device)
    Xtz_p = torch.zeros((M, K), dtype=dt, device=device)
    dim = M * K + N * K
    U = torch.zeros((dim, Q_hist), dtype=dt, device=device)
    V = torch.zeros((dim, Q_hist), dtype=dt, device=device)
    UV = torch.zeros((dim, Q_hist), dtype=dt, device=device)
    P_qn, Q_qn = torch.empty_like(P), torch.empty_like(Q)
    x_qn = torch.empty(dim, dtype=dt, device=device)
    x0 = torch.empty(dim, dtype=dt, device=device)
    x1 = torch.empty(dim, dtype=dt, device=device)
    x2 = torch.empty(dim, dtype=dt, device=device)
    mk = M * K

    def flat(Pm, Qm, out):
        out[:mk].copy_(Pm.ravel())
        out[mk:].copy_(Qm.ravel())

    def sqp_q(Pm, Qm):
        ops.grad_hess_q(G, Pm, Qm, M, XtX_q, Xtz_q)
        Xtz_q.neg_()
        Qn = ops.sqp_solve_q(XtX_q, Xtz_q, Qm, v_kk, N, K)
        if q_hook is not None:
            q_hook(Qn)
        return Qn

    def sqp_p(Pm, Qm):
        ops.grad_hess_p(G, Pm, Qm, M, XtX_p, Xtz_p)
        Xtz_p.neg_()
        return ops.sqp_solve_p(XtX_p, Xtz_p, Pm, M, K)

    def logl(Pm, Qm):
        return loglikelihood_gpu(G, Pm, Qm, M, N, 0, device, 0)

    ll_prev = -float("inf")
    ll_best = -float("inf")
    wait = 0
    P_best, Q_best = torch.empty_like(P), torch.empty_like(Q)
    for it in range(1, max_iter + 1):
        t_it = time.time()
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
        torch.sub(U_s, V_s, out=UV[:, :n_cols])
        LHS = U_s.T @ UV[:, :n_cols]
        torch.sub(x0, x1, out=x_qn)
        RHS = U_s.T @ x_qn
        try:
            alpha = torch.linalg.solve(LHS, RHS)
        except RuntimeError:
            alpha = torch.linalg.lstsq(LHS, RHS).solution
        torch.matmul(V_s, alpha, out=x_qn)
        torch.sub(x1, x_qn, out=x_qn)
        P_qn.copy_(x_qn[:mk].view(M, K))
        Q_qn.copy_(x_qn[mk:].view(-1, K))
        if qn_projection == "simplex":
            ops.project_box_(P_qn)
            ops.project_simplex_(Q_qn)
        else:
            _mapPQ_gpu(P_qn, Q_qn)
        if q_hook is not None:
            q_hook(Q_qn)

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
            log.info(f"    Iteration {it}, Log-likelihood: {ll_new:.1f}, Time: {time.time() - t_it:.3f}s")
        if abs(ll_new - ll_prev) < tol:
            if verbose:
                log.info(f"    Converged at iteration {it}.")
            break
        if wait >= patience:
            if verbose:
                log.info(f"    Converged at iteration {it} after {wait} iterations without improvement.")
            break
        ll_prev = ll_new
    if verbose:
        log.info(f"\n    Final log-likelihood: {ll_best:.1f}")
    return P_best, Q_best


def optimize_original_gpu(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, max_iter: int,
                          K: int, M: int, N: int, tol: float, Q_hist: int,
                          patience: int, device: torch.device, chunk_size: int,
                          threads_per_block: int) -> tuple[torch.Tensor, torch.Tensor]:
    """SQP + ZAL QN from ``(P, Q)`` (float64, copied); returns the best ``(P, Q)``."""
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    P_w = P.to(device=G.device, dtype=torch.float64).clone().contiguous()
    Q_w = Q.to(device=G.device, dtype=torch.float64).clone().contiguous()
    return _optimize_original_gpu_once(G, P_w, Q_w, max_iter, K, M, N, tol, Q_hist, patience, G.device)


def polish_sqp_qn(G: torch.Tensor, P_init, Q_init, M: int, N: int, K: int,
                  n_iters: int = 3, Q_hist: int = 3) -> tuple[torch.Tensor, torch.Tensor]:
    """Exactly ``n_iters`` SQP + ZAL iterations from a warm start with early stopping off
    (tol 0, patience n_iters + 1) and the CPU reference's simplex projection of the
    extrapolated point: adamixture/model/br_qn.py:50-70, on the GPU."""
    P = torch.as_tensor(P_init, dtype=torch.float64).to(G.device).clone().contiguous()
    Q = torch.as_tensor(Q_init, dtype=torch.float64).to(G.device).clone().contiguous()
    return _optimize_original_gpu_once(G, P, Q, n_iters, K, M, N, 0.0, Q_hist, n_iters + 1, G.device,
                                       qn_projection="simplex", verbose=False)
