"""Projection of new samples onto a fitted P on one B200: drop-in for the GPU functions of
``adamixture/src/projection.py`` (``optimize_projection_gpu``,
``optimize_projection_original_gpu``).

P stays fixed; only Q is optimised. Adam-EM form (projection.py:178-321): the E-step is
this library's fused sweep (``ops.em_stats``, whose P-side statistics are discarded), Q's
EM target is formed from T and q_bat as in ``em_final_update``, and Q takes the Adam step,
clamp and row normalisation, with the priming step, log-likelihood checks every ``check``
iterations, best-Q tracking and lr decay of the reference. Original form
(projection.py:505-640): two SQP updates of Q per iteration from the Q-side gradient/Hessian
pass, ZAL extrapolation on Q, acceptance by log-likelihood and the tolerance / patience
stops.
"""
from __future__ import annotations

import logging
import time

import torch

from .. import ops
from ..model.br_qn_gpu import _v_kk
from ..model.em_adam_gpu import adam_update, loglikelihood_gpu, resolve_precision

log = logging.getLogger(__name__)


def _q_target(Q, T, q_bat):
    """Q's EM target (em_adam_gpu.py:82-117, Q side): Q*T / max(q_bat, 1e-5), rows
    normalised by max(sum, 1e-5)."""
    Qt = Q * T / torch.clamp(q_bat, min=1e-5).unsqueeze(1)
    return Qt / torch.clamp(Qt.sum(dim=1, keepdim=True), min=1e-5)


def optimize_projection_gpu(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor,
                            lr: float, beta1: float, beta2: float, reg_adam: float,
                            max_iter: int, check: int, M: int,
                            lr_decay: float, min_lr: float, patience: int, tol_adam: float,
                            device: torch.device, chunk_size: int, threads_per_block: int,
                            precision: str | None = "f64") -> torch.Tensor:
    """Q [N, K] maximising the likelihood with P fixed (Adam-EM on Q)."""
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    N, K = Q.shape
    prec = resolve_precision(K, precision)
    dt = ops.input_dtype(prec)
    P = P.to(device=G.device, dtype=torch.float64).contiguous()
    Q = Q.to(device=G.device, dtype=torch.float64).clone().contiguous()
    P_in = P.to(dt).contiguous()
    m_Q, v_Q = torch.zeros_like(Q), torch.zeros_like(Q)
    t_tensor = torch.tensor(0.0, device=G.device, dtype=torch.float64)

    q_bat = ops.sample_counts(G, M)

    def em_q():
        _, _, T = ops.em_stats(G, P_in, Q.to(dt).contiguous(), M, prec)
        return _q_target(Q, T, q_bat)

    def adam_q(Qt):
        t_tensor.add_(1.0)
        adam_update(Q, Qt, m_Q, v_Q, t_tensor, lr, beta1, beta2, reg_adam)
        torch.clamp_(Q, 1e-5, 1.0 - 1e-5)
        Q.div_(Q.sum(dim=1, keepdim=True))

    def logl():
        return loglikelihood_gpu(G, P, Q, M, N, chunk_size, G.device, threads_per_block)

    adam_q(em_q())
    em_q()  # the reference's priming runs a second E-step whose result is unused
    L_best = logl()
    Q_best = Q.clone()
    wait_lr = 0
    ts = time.time()
    for it in range(max_iter):
        adam_q(em_q())
        if (it + 1) % check == 0:
            L_cur = logl()
            log.info(f"    Iteration {it + 1}, Log-likelihood: {L_cur:.1f}, Time: {time.time() - ts:.3f}s")
            ts = time.time()
            if L_cur > L_best + tol_adam:
                L_best = L_cur
                Q_best.copy_(Q)
                wait_lr = 0
            else:
                wait_lr += 1
                if wait_lr >= patience:
                    lr = max(lr * lr_decay, min_lr)
                    if lr <= min_lr:
                        log.info("    Convergence reached.")
                        break
                    wait_lr = 0
    log.info(f"\n    Final log-likelihood (projection): {L_best:.1f}")
    return Q_best


def optimize_projection_original_gpu(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor,
                                     max_iter: int, K: int, M: int, N: int, tol: float, Q_hist: int,
                                     patience: int, device: torch.device, chunk_size: int,
                                     threads_per_block: int) -> torch.Tensor:
    """Q [N, K] with P fixed by SQP + ZAL quasi-Newton on Q."""
    if not G.is_cuda:
        raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")
    dt = torch.float64
    P = P.to(device=G.device, dtype=dt).contiguous()
    Q = Q.to(device=G.device, dtype=dt).clone().contiguous()
    v_kk = _v_kk(K, G.device)
    XtX_q = torch.zeros((N, K, K), dtype=dt, device=G.device)
    Xtz_q = torch.zeros((N, K), dtype=dt, device=G.device)
    dim = N * K
    U = torch.zeros((dim, Q_hist), dtype=dt, device=G.device)
    V = torch.zeros((dim, Q_hist), dtype=dt, device=G.device)
    UV = torch.zeros((dim, Q_hist), dtype=dt, device=G.device)
    Q_qn = torch.empty_like(Q)

    def sqp_q(Qm):
        ops.grad_hess_q(G, P, Qm, M, XtX_q, Xtz_q)
        Xtz_q.neg_()
        return ops.sqp_solve_q(XtX_q, Xtz_q, Qm, v_kk, N, K)

    def logl(Qm):
        return loglikelihood_gpu(G, P, Qm, M, N, chunk_size, G.device, threads_per_block)

    ll_prev = ll_best = -float("inf")
    wait = 0
    Q_best = torch.empty_like(Q)
    for it in range(1, max_iter + 1):
        t_it = time.time()
        Q1 = sqp_q(Q)
        Q2 = sqp_q(Q1)
        x0, x1, x2 = Q.reshape(-1), Q1.reshape(-1), Q2.reshape(-1)
        col = (it - 1) % Q_hist
        torch.sub(x1, x0, out=U[:, col])
        torch.sub(x2, x1, out=V[:, col])
        n_cols = min(it, Q_hist)
        U_s, V_s = U[:, :n_cols], V[:, :n_cols]
        torch.sub(U_s, V_s, out=UV[:, :n_cols])
        LHS = U_s.T @ UV[:, :n_cols]
        RHS = U_s.T @ (x0 - x1)
        try:
            alpha = torch.linalg.solve(LHS, RHS)
        except RuntimeError:
            alpha = torch.linalg.lstsq(LHS, RHS).solution
        Q_qn.copy_((x1 - V_s @ alpha).view(N, K))
        torch.clamp_(Q_qn, 1e-5, 1.0 - 1e-5)
        Q_qn.div_(Q_qn.sum(dim=1, keepdim=True))
        ll_qn = logl(Q_qn)
        if ll_qn > ll_prev:
            Q.copy_(Q_qn)
            ll_new = ll_qn
        else:
            Q.copy_(Q2)
            ll_new = logl(Q2)
        best_before = ll_best
        if ll_new > ll_best:
            ll_best = ll_new
            Q_best.copy_(Q)
        if best_before != -float("inf") and ll_new <= best_before + tol:
            wait += 1
        else:
            wait = 0
        log.info(f"    Iteration {it}, Log-likelihood: {ll_new:.1f}, Time: {time.time() - t_it:.3f}s")
        if abs(ll_new - ll_prev) < tol or wait >= patience:
            break
        ll_prev = ll_new
    log.info(f"\n    Final log-likelihood (projection): {ll_best:.1f}")
    return Q_best
