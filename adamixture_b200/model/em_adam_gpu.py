"""Adam-EM on one B200: drop-in for ``adamixture/model/em_adam_gpu.py``.

Same public names and signatures as the reference module:
``adam_update``, ``em_final_update``, ``EMAdamOptimizer`` (``run_em_step``, ``step``),
``loglikelihood_gpu``, ``optimize_parameters_gpu``. P and Q stay float64 tensors on the
device, as in the reference. The per-chunk torch/cuBLAS work of the reference is replaced
by one fused CUDA sweep over the packed genotypes per iteration; ``chunk_size`` and
``threads_per_block`` are accepted for signature compatibility and have no effect on
the arithmetic.

E-step arithmetic (``precision``): ``"f64"`` reproduces the reference's float64 path;
``"f32"`` forms ratios and partial sums in float32 (float64 cross-block sums);
``"bf16"`` and ``"f16"`` are the tensor-core forms (BF16 or power-of-two-scaled FP16
operands, FP32 accumulation; K <= 16); ``"mixed"`` runs tensor-core sweeps until the
first plateau and float32 sweeps after it. ``set_precision`` sets the default
(environment: ``ADX_PRECISION``); the default policy ("auto") is ``"f16"`` for
8 <= K <= 16 and ``"f32"`` otherwise (float32 ratios below K = 8, as specified). FP16
rather than BF16: at the same cost per iteration, its 11-bit operands let Adam converge
in float32's number of iterations, where BF16's 8-bit operands need about twice as many.
``"f16"`` can be asked for at any K <= 16: the tensor-core sweep is also the faster one
below K = 8 (1.6x at K=2 on N=10k x M=200k).
"""
from __future__ import annotations

import logging
import os
import time

import torch

from .. import ops, tune
from .._lib import AdxError

log = logging.getLogger(__name__)

_PRECISION = os.environ.get("ADX_PRECISION", "auto")
# runs of fused iterations between log-likelihood checks replay a captured CUDA graph
USE_GRAPHS = os.environ.get("ADX_GRAPHS", "1") != "0"


def set_precision(p: str) -> None:
    """Default E-step arithmetic: "f64", "f32", "bf16", "f16", "mixed" or "auto"."""
    global _PRECISION
    if p not in ("auto", "mixed"):
        ops.precision_code(p)
    _PRECISION = p


TC_MIN_K, TC_MAX_K = 8, 16


def resolve_precision(K: int, precision: str | None = None) -> str:
    """The E-step arithmetic for this K. "auto": tensor cores (scaled FP16 operands, FP32
    accumulation) for 8 <= K <= 16, float32 otherwise. "mixed" resolves to the first
    phase's arithmetic here (the optimiser switches to float32 at the first plateau)."""
    p = precision or _PRECISION
    if p in ("auto", "mixed"):
        return "f16" if TC_MIN_K <= K <= TC_MAX_K else "f32"
    if p in ("bf16", "f16") and K > TC_MAX_K:
        raise ValueError(f"the tensor-core E-step supports K <= {TC_MAX_K} (got K={K}); use 'f32'")
    return p


def _require_cuda(*ts):
    for t in ts:
        if isinstance(t, torch.Tensor) and not t.is_cuda:
            raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU tensor)")


def adam_update(param, param_target, m, v, t_tensor, lr, beta1, beta2, reg_adam):
    """In-place Adam move toward the EM target (em_adam_gpu.py:11-42). ``param`` and
    ``param_target`` are either P-shaped or Q-shaped; Q rows are NOT renormalised here
    (``EMAdamOptimizer.step`` does that, as in the reference)."""
    delta = param_target - param
    m.mul_(beta1).add_(delta, alpha=1 - beta1)
    v.mul_(beta2).addcmul_(delta, delta, value=1 - beta2)
    m_hat = m / (1 - beta1 ** t_tensor)
    v_hat = v / (1 - beta2 ** t_tensor)
    param.add_(lr * m_hat / (torch.sqrt(v_hat) + reg_adam))
    return param


def em_final_update(P, Q, A_accum, B_accum, T_accum, q_bat, P_target, Q_target):
    """EM targets from the statistics (em_adam_gpu.py:82-117), one CUDA launch."""
    _require_cuda(P, Q)
    return ops.em_targets(P, Q, A_accum, B_accum, T_accum, q_bat, P_target, Q_target)


class EMAdamOptimizer:
    """Adam state + EM buffers (em_adam_gpu.py:121-224), same constructor and methods."""

    def __init__(self, P_shape, Q_shape, lr, beta1, beta2, reg_adam, device, precision=None):
        self.device = torch.device(device)
        self.lr = lr
        self.beta1 = beta1
        self.beta2 = beta2
        self.reg_adam = reg_adam
        self.dtype = torch.float64
        self.precision = resolve_precision(int(Q_shape[1]), precision)
        self.t = torch.tensor(0.0, device=self.device, dtype=self.dtype)
        self._t = 0
        z = lambda s: torch.zeros(s, dtype=self.dtype, device=self.device)  # noqa: E731
        self.m_P, self.v_P = z(P_shape), z(P_shape)
        self.m_Q, self.v_Q = z(Q_shape), z(Q_shape)
        self.A_accum, self.B_accum = z(P_shape), z(P_shape)
        self.T_accum = z(Q_shape)
        self.q_bat = z(Q_shape[0])
        self.P_EM, self.Q_EM = z(P_shape), z(Q_shape)
        self._qbat_key = None

    def _sample_counts(self, G, M):
        key = (G.data_ptr(), tuple(G.shape), M)
        if self._qbat_key != key:
            self.q_bat.copy_(ops.sample_counts(G, M))
            self._qbat_key = key
        return self.q_bat

    def _operands(self, P, Q):
        dt = ops.input_dtype(self.precision)
        if P.dtype == dt:
            return P.contiguous(), Q.contiguous()
        return P.to(dt).contiguous(), Q.to(dt).contiguous()

    def run_em_step(self, G, P, Q, M, chunk_size, unpacker=None):
        """One E-step sweep -> EM targets ``(P_EM, Q_EM)`` (em_adam_gpu.py:166-199)."""
        _require_cuda(G, P, Q)
        Pin, Qin = self._operands(P, Q)
        A, B, T = ops.em_stats(G, Pin, Qin, M, self.precision)
        self.A_accum.copy_(A)
        self.B_accum.copy_(B)
        self.T_accum.copy_(T)
        self._sample_counts(G, M)
        return ops.em_targets(P, Q, self.A_accum, self.B_accum, self.T_accum, self.q_bat,
                              self.P_EM, self.Q_EM)

    def step(self, P, Q, P_target, Q_target, P32=None, Q32=None):
        """Adam move, clamp to [1e-5, 1-1e-5], renormalise Q rows (em_adam_gpu.py:201-224)."""
        self._t += 1
        self.t.fill_(float(self._t))
        ops.adam_step(P, Q, P_target, Q_target, self.m_P, self.v_P, self.m_Q, self.v_Q,
                      self._t, self.lr, self.beta1, self.beta2, self.reg_adam, P32, Q32)

    def can_fold_check(self, K: int) -> bool:
        """Whether this arithmetic has the sweep with the log-likelihood check folded in."""
        return self.precision == "f64" and K <= 16

    def sweep_with_loglik(self, G, P, Q, M, workspace):
        """The E-step sweep of the next iteration, which also returns (as a device scalar) the
        float64 log-likelihood of its input (P, Q): the check the reference runs after the
        previous iteration's move, bit-identical to ``loglikelihood_gpu``. Follow it with
        ``apply_update``."""
        self._sample_counts(G, M)
        ops.em_sweep_loglik(G, P, Q, M, workspace)
        return ops.em_loglik_from_sweep(workspace, M, Q.shape[0], Q.shape[1])

    def apply_update(self, P, Q, P32, Q32, M, workspace):
        """EM targets + Adam move from the last ``sweep_with_loglik`` (at ``self.lr``)."""
        self._t += 1
        ops.em_adam_update(P, Q, P32, Q32, self.m_P, self.v_P, self.m_Q, self.v_Q, self.q_bat, M, self._t,
                           self.lr, self.beta1, self.beta2, self.reg_adam, self.precision, workspace)

    def fused_iteration(self, G, P, Q, P32, Q32, M, workspace=None):
        """``run_em_step`` + ``step`` in two launches, without materialising A/B/T."""
        self._sample_counts(G, M)
        self._t += 1
        ops.em_adam_iteration(G, P, Q, P32, Q32, self.m_P, self.v_P, self.m_Q, self.v_Q,
                              self.q_bat, M, self._t, self.lr, self.beta1, self.beta2,
                              self.reg_adam, self.precision, workspace)


class _IterationGraphs:
    """Runs of fused Adam-EM iterations (between two log-likelihood checks) as replays of a
    captured CUDA graph (``ops.EmGraph``), one graph per (run length, learning rate,
    arithmetic), built on first use; the replays equal the eager iterations bit for bit.
    A run of one iteration, or ``enabled=False``, runs eagerly. ``ws`` must be a workspace of
    the optimiser's own (``ops.em_workspace``)."""

    def __init__(self, opt, G, P, Q, P32, Q32, M, ws, enabled=None):
        self.opt, self.G, self.P, self.Q, self.P32, self.Q32, self.M, self.ws = opt, G, P, Q, P32, Q32, M, ws
        self.enabled = USE_GRAPHS if enabled is None else enabled
        self.cache = {}

    def run(self, n: int) -> None:
        opt = self.opt
        if n <= 0:
            return
        if not self.enabled or n < 2:
            for _ in range(n):
                opt.fused_iteration(self.G, self.P, self.Q, self.P32, self.Q32, self.M, self.ws)
            return
        key = (n, opt.lr, opt.precision, self.ws.data_ptr())
        g = self.cache.get(key)
        if g is None:
            q_bat = opt._sample_counts(self.G, self.M)
            try:
                g = ops.EmGraph(self.G, self.P, self.Q, self.P32, self.Q32, opt.m_P, opt.v_P, opt.m_Q, opt.v_Q,
                                q_bat, self.M, n, opt.lr, opt.beta1, opt.beta2, opt.reg_adam, opt.precision,
                                self.ws)
            except AdxError as e:
                # the capture itself failed (nothing ran): the same iterations, launched one by one
                log.warning(f"    CUDA graph capture unavailable ({e}); launching iterations one by one.")
                self.enabled = False
                self.run(n)
                return
            self.cache[key] = g
        g.launch(opt._t)
        opt._t += n

    def close(self) -> None:
        for g in self.cache.values():
            g.close()
        self.cache.clear()


def logl_batch_math(g_chunk, p_batch, Q):
    """Reference per-chunk log-likelihood in float64 torch (em_adam_gpu.py:226-248); kept
    for API compatibility; the library computes the sum with ``loglikelihood_gpu``."""
    rec = torch.clamp(p_batch @ Q.T, 1e-10, 1.0 - 1e-10).to(torch.float64)
    g = g_chunk.to(torch.float64)
    return ((g * torch.log(rec) + (2.0 - g) * torch.log1p(-rec)) * (g_chunk != 3)).sum()


def loglikelihood_gpu(G, P, Q, M, N, batch_size, device, threads_per_block, precision="f64") -> float:
    """Binomial log-likelihood, float64 sum over the packed genotypes (em_adam_gpu.py:250-279).

    ``precision`` selects how h = PQ^T is formed: "f64" (the reference's arithmetic) or
    "f32" (float32 dot products; the per-entry factors and the sum stay float64)."""
    _require_cuda(G, P, Q)
    dt = torch.float64 if precision == "f64" else torch.float32
    out = ops.loglik_device(G, P.to(dt).contiguous(), Q.to(dt).contiguous(), M, precision)
    return float(out.item())


def _optimize_parameters_gpu_once(G, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K, M, N,
                                  lr_decay, min_lr, patience, tol_adam, device, chunk_size,
                                  threads_per_block, precision=None, trace=None, fold_checks=True):
    """Adam-EM with lr decay (em_adam_gpu.py:281-356), fused iterations.

    Same control flow as the reference: priming (E-step + Adam step), log-likelihood of
    the primed point as the first best, then ``max_iter`` iterations with a check every
    ``check`` iterations. The reference's second priming E-step, whose result it never
    uses (:322), is skipped: it changes no state. ``trace`` (a list) receives
    ``(iteration, loglik, seconds since the start)`` at each check (host clock after the
    check's read-back, so the device work up to it is included). ``precision="mixed"``: tensor-core sweeps
    until the first plateau (``patience`` checks without a new best), float32 sweeps after
    it, with the same Adam state and learning rate.
    """
    mixed = (precision or _PRECISION) == "mixed"
    opt = EMAdamOptimizer(P.shape, Q.shape, lr, beta1, beta2, reg_adam, device, precision)
    prec = opt.precision
    ll_prec = "f64" if prec == "f64" else "f32"
    dt = ops.input_dtype(prec)
    P32 = P.to(torch.float32).contiguous() if dt == torch.float32 else None
    Q32 = Q.to(torch.float32).contiguous() if dt == torch.float32 else None
    ws = ops.em_workspace(M, N, K, prec, G.device)
    if prec == "f64" and K <= 16:
        tune.tune_dmma(G, P, Q, M, workspace=ws)

    def loglik():
        if ll_prec == "f64":
            L = float(ops.loglik_device(G, P, Q, M, "f64").item())
        else:
            L = float(ops.loglik_device(G, P32, Q32, M, "f32").item())
        st = ops.em_status(ws, M, N, K, prec)
        if st:
            raise RuntimeError(f"E-step sweep reported status {st} (a bounded wait timed out)")
        return L

    ts = time.time()
    t_start = time.perf_counter()
    opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
    log.info(f"    Performed priming iteration... ({time.time() - ts:.1f}s)\n")
    if fold_checks and not mixed and opt.can_fold_check(K):
        return _loop_folded_checks(G, P, Q, M, N, K, opt, ws, max_iter, check, lr_decay, min_lr, patience,
                                   tol_adam, trace, t_start)
    L_best = loglik()
    P_best, Q_best = P.clone(), Q.clone()
    wait_lr = 0
    ts = time.time()
    graphs = _IterationGraphs(opt, G, P, Q, P32, Q32, M, ws)
    it = 0   # iterations done
    try:
        while it < max_iter:
            # the fused iterations up to the next check (or the end), replayed from a graph
            n = min(check - it % check, max_iter - it)
            graphs.run(n)
            it += n
            if it % check:
                continue
            L_cur = loglik()
            if trace is not None:
                trace.append((it, L_cur, time.perf_counter() - t_start))
            log.info(f"    Iteration {it}, Log-likelihood: {L_cur:.1f}, Time: {time.time() - ts:.3f}s")
            ts = time.time()
            if L_cur > L_best + tol_adam:
                L_best = L_cur
                P_best.copy_(P)
                Q_best.copy_(Q)
                wait_lr = 0
            else:
                wait_lr += 1
                if wait_lr >= patience and mixed and prec != "f32":
                    # mixed precision: the first plateau ends the tensor-core phase; the same Adam
                    # state continues with float32 sweeps (same float32 P/Q shadows)
                    prec = opt.precision = "f32"
                    ws = graphs.ws = ops.em_workspace(M, N, K, prec, G.device)
                    log.info("    Plateau in the tensor-core phase: continuing with float32 E-steps.")
                    wait_lr = 0
                    continue
                if wait_lr >= patience:
                    old = opt.lr
                    opt.lr = max(opt.lr * lr_decay, min_lr)
                    log.info(f"    Plateau reached ({wait_lr} checks without beating best). "
                             f"Reducing lr: {old:.3e} → {opt.lr:.3e}")
                    if opt.lr <= min_lr:
                        log.info("        Convergence reached.")
                        break
                    wait_lr = 0
    finally:
        graphs.close()
    log.info(f"\n    Final log-likelihood: {L_best:.1f}")
    return P_best, Q_best


def _loop_folded_checks(G, P, Q, M, N, K, opt, ws, max_iter, check, lr_decay, min_lr, patience, tol_adam, trace,
                        t_start):
    """The reference loop after the priming step (em_adam_gpu.py:318-353) with every
    log-likelihood check folded into the next iteration's sweep (float64, K <= 16).

    The check after iteration ``it`` (1-based ``it`` a multiple of ``check``) scores the
    (P, Q) that iteration ``it + 1`` sweeps, so that sweep returns it; the decisions (best
    checkpoint of the current P, Q, learning-rate decay, stop) are taken before that
    iteration's move is applied, and a stop leaves the move unapplied -- the same states,
    values and control flow as checking after the move. The first best is the log-likelihood
    of the primed (P, Q), which the first iteration's sweep returns. A check due after the
    last iteration runs on its own."""
    state = {"L_best": None, "P_best": None, "Q_best": None, "wait": 0}

    def decide(L, it):
        """The reference's decisions on check value L of iteration ``it``; False = stop."""
        st = ops.em_status(ws, M, N, K, opt.precision)
        if st:
            raise RuntimeError(f"E-step sweep reported status {st} (a bounded wait timed out)")
        if state["L_best"] is None:
            state["L_best"], state["P_best"], state["Q_best"] = L, P.clone(), Q.clone()
            return True
        if trace is not None:
            trace.append((it, L, time.perf_counter() - t_start))
        log.info(f"    Iteration {it}, Log-likelihood: {L:.1f}")
        if L > state["L_best"] + tol_adam:
            state["L_best"] = L
            state["P_best"].copy_(P)
            state["Q_best"].copy_(Q)
            state["wait"] = 0
            return True
        state["wait"] += 1
        if state["wait"] >= patience:
            old = opt.lr
            opt.lr = max(opt.lr * lr_decay, min_lr)
            log.info(f"    Plateau reached ({state['wait']} checks without beating best). "
                     f"Reducing lr: {old:.3e} → {opt.lr:.3e}")
            if opt.lr <= min_lr:
                log.info("        Convergence reached.")
                return False
            state["wait"] = 0
        return True

    need = True   # the next sweep's input needs its log-likelihood (first: the primed point)
    stopped = False
    graphs = _IterationGraphs(opt, G, P, Q, None, None, M, ws)
    it = 0        # iterations done
    try:
        while it < max_iter:
            if need:
                L = float(opt.sweep_with_loglik(G, P, Q, M, ws).item())
                if not decide(L, it):
                    stopped = True
                    break
                opt.apply_update(P, Q, None, None, M, ws)
                need = False
                it += 1
            else:
                # the plain iterations up to the next check (or the end), replayed from a graph
                n = min(check - it % check, max_iter - it)
                graphs.run(n)
                it += n
            if it % check == 0:
                need = True
    finally:
        graphs.close()
    if need and not stopped:
        decide(float(ops.loglik_device(G, P, Q, M, "f64").item()), max_iter)
    log.info(f"\n    Final log-likelihood: {state['L_best']:.1f}")
    return state["P_best"], state["Q_best"]


MAX_UPLOAD_PIECES = 4


def upload_pieces(n_blocks: int, ctas_per_block: int, sms: int, max_pieces: int = MAX_UPLOAD_PIECES):
    """Block ranges of the pieces in which a host matrix is uploaded and swept.

    Each piece's sweep is one launch of ``ctas_per_block`` CTAs per block, one CTA per SM,
    so a launch takes as long as its CTA count rounded up to whole waves of ``sms``. The
    pieces are the most (up to ``max_pieces``) whose waves add up to the full sweep's, the
    larger ones last: piece i gets w_i waves and the blocks that fit in them. More pieces
    let the sweep start sooner after the upload starts; a piece that would leave part of a
    wave idle would make the sweeps slower than the full sweep. Returns [(b0, b1), ...]."""
    waves = -(-n_blocks * ctas_per_block // sms)
    for q in range(min(max_pieces, waves, n_blocks), 1, -1):
        w = [waves // q + (1 if i >= q - waves % q else 0) for i in range(q)]
        fit = [wi * sms // ctas_per_block for wi in w]
        if min(fit) < 1 or sum(fit) < n_blocks:
            continue
        out, b = [], 0
        for f in fit:
            if b < n_blocks:
                out.append((b, min(n_blocks, b + f)))
                b += f
        return out
    return [(0, n_blocks)]


def _upload_and_prime(G_host, P, Q, M, K, opt, device):
    """Copy the packed matrix from host memory to ``device`` in pieces of whole SNP blocks
    (``upload_pieces``) on a copy stream and run the priming iteration's float64 sweep and
    sample counts on each piece as it lands, then the priming move: the copy overlaps the
    sweep. The partial sums are the full sweep's, so the primed (P, Q) equal those of
    uploading first and priming after. Returns the device matrix and the workspace."""
    N = Q.shape[0]
    G = torch.empty(G_host.shape, dtype=torch.uint8, device=device)
    ws = ops.em_workspace(M, N, K, "f64", G.device)
    spb, nb, cpb = ops.em_sweep_blocks_info(M, N, K)
    sms = torch.cuda.get_device_properties(G.device).multi_processor_count
    rows_pb = spb // 4                                  # packed rows per block
    main = torch.cuda.current_stream(G.device)
    copy = torch.cuda.Stream(G.device)
    copy.wait_stream(main)
    q = torch.zeros(N, dtype=torch.float64, device=G.device)
    rows = G.shape[0]
    pieces = []
    with torch.cuda.stream(copy):
        for b0, b1 in upload_pieces(nb, cpb, sms):
            r0, r1 = b0 * rows_pb, min(rows, b1 * rows_pb)
            G[r0:r1].copy_(G_host[r0:r1], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy)
            pieces.append((b0, b1, r0, r1, ev))
    for b0, b1, r0, r1, ev in pieces:
        main.wait_event(ev)
        ops.em_sweep_blocks(G, P, Q, M, b0, b1, ws)
        # per-sample observed counts of the piece's SNPs (exact integers: any order)
        q += ops.sample_counts(G[r0:r1], min(M, 4 * r1) - 4 * r0)
    G.record_stream(copy)
    opt.q_bat.copy_(q)
    opt._qbat_key = (G.data_ptr(), tuple(G.shape), M)
    opt.apply_update(P, Q, None, None, M, ws)
    return G, ws


def optimize_parameters_gpu(G, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K, M, N,
                            lr_decay, min_lr, patience, tol_adam, device, chunk_size,
                            threads_per_block, precision=None, trace=None):
    """Adam-EM on the GPU (em_adam_gpu.py:359-385). The reference's OOM retry halves the
    chunk size; the fused sweep has no per-chunk temporaries, so there is nothing to
    retry: the only allocations are P/Q-sized buffers and the partial-sum workspace.

    ``G`` may also be a packed matrix in (pinned) host memory, with P and Q on the host or
    the device: in float64 with K <= 16 it is then uploaded to ``device`` in pieces, each
    piece swept by the priming iteration as it lands (the copy overlaps the sweep); the
    iterations are the same as for a resident matrix."""
    if not G.is_cuda:
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("adamixture_b200 runs on CUDA devices only (got a CPU device)")
        P = P.to(dev, torch.float64).contiguous().clone()
        Q = Q.to(dev, torch.float64).contiguous().clone()
        opt_prec = resolve_precision(K, precision)
        if opt_prec == "f64" and K <= 16 and (precision or _PRECISION) != "mixed":
            return _optimize_streamed(G, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K, M, N, lr_decay,
                                      min_lr, patience, tol_adam, dev, trace)
        G = G.to(dev)
    _require_cuda(G, P, Q)
    P = P.to(torch.float64).contiguous().clone()
    Q = Q.to(torch.float64).contiguous().clone()
    return _optimize_parameters_gpu_once(G, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K,
                                         M, N, lr_decay, min_lr, patience, tol_adam, device,
                                         chunk_size, threads_per_block, precision, trace)


def _optimize_streamed(G_host, P, Q, lr, beta1, beta2, reg_adam, max_iter, check, K, M, N, lr_decay, min_lr,
                       patience, tol_adam, device, trace):
    """``optimize_parameters_gpu`` from a host matrix, float64: the upload overlaps the
    priming sweep, then the reference loop with folded checks."""
    opt = EMAdamOptimizer(P.shape, Q.shape, lr, beta1, beta2, reg_adam, device, "f64")
    ts = time.time()
    t_start = time.perf_counter()
    G, ws = _upload_and_prime(G_host, P, Q, M, K, opt, device)
    log.info(f"    Performed priming iteration... ({time.time() - ts:.1f}s)\n")
    # the priming sweep ran the default layout; the loop's sweeps run the tuned one (the
    # tuning sweeps overwrite only partial sums that the loop's first sweep rewrites)
    tune.tune_dmma(G, P, Q, M, workspace=ws)
    return _loop_folded_checks(G, P, Q, M, N, K, opt, ws, max_iter, check, lr_decay, min_lr, patience, tol_adam,
                               trace, t_start)

