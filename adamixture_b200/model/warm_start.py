"""Learned warm start of Q (and P from one M-step) for Adam-EM; a new component of this
build with no counterpart in the reference.

Per sample, a small network maps 33 features to the K-way membership:

* the sample's ALS memberships Q_als (the reference's initialisation, adamixture/model/
  als_gpu.py, itself a function of the randomized-SVD factors), zero-padded to 16;
* its first 16 randomized-SVD scores V S, each standardised over the samples (signs fixed
  by the largest-magnitude SNP loading, as the reference's tests canonicalise U/V);
* its heterozygosity (heterozygous / observed genotypes).

The output is ``softmax(f(x) + log Q_als)``: a residual on the ALS start (with the last
layer initialised to zero, an untrained network returns Q_als; padded columns carry a
large negative prior). Training targets are the converged Q of plain EM started from the
same ALS init on seeded synthetic cohorts, so the labels of target and input agree. The
network is trained and run on this library's kernels (``adx_mlp_forward``,
``adx_mlp_backward``, ``adx_mlp_adam``: BF16 weights, FP32 accumulation).

``P`` of the warm start is one M-step from ``Q0``: by default the P target of one EM step
from (P_als, Q0) (this library's E-step and targets); the alternative ``m_step_P`` takes
the membership-weighted allele frequencies ``P_jk = sum_i g_ji Q_ik / (2 sum_i obs_ji
Q_ik)`` from two products of the packed genotypes (``ops.rsvd_rows``), which measured far
worse (it discards the ALS P). Plain EM from the ALS start stays the fallback and the
yardstick: ``warm_start_fit`` keeps the warm run only if its converged log-likelihood is no
worse than the plain run's (within 1e-6 relative).
"""
from __future__ import annotations

import logging
import math
import time
from pathlib import Path

import numpy as np
import torch

from .. import _lib, ops
from .als_gpu import ALS_gpu
from .em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu
from .svd_gpu import SVD_gpu

log = logging.getLogger(__name__)

D_IN, H, KMAX = 33, 256, 16
N_SCORES = 16
PAD_PRIOR = -30.0


def _bf16_bits(w: torch.Tensor) -> torch.Tensor:
    return w.to(torch.bfloat16).contiguous()


class WarmStartMLP:
    """Weights (fp32 masters + BF16 copies), Adam state and the kernel calls."""

    SHAPES = {"W1": (H, D_IN), "b1": (H,), "W2": (H, H), "b2": (H,), "W3": (KMAX, H), "b3": (KMAX,)}

    def __init__(self, device, seed: int = 0):
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        w = {
            "W1": torch.randn(H, D_IN, generator=g) * math.sqrt(2.0 / D_IN),
            "b1": torch.zeros(H),
            "W2": torch.randn(H, H, generator=g) * math.sqrt(2.0 / H),
            "b2": torch.zeros(H),
            "W3": torch.zeros(KMAX, H),   # residual on the prior: starts as the identity map
            "b3": torch.zeros(KMAX),
        }
        self.w = {k: v.to(self.device, torch.float32).contiguous() for k, v in w.items()}
        self._refresh_bf16()
        self.m = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.t = 0
        self._ws = None

    def _refresh_bf16(self):
        self.wb = {k: _bf16_bits(self.w[k]) for k in ("W1", "W2", "W3")}

    def _workspace(self, B: int) -> torch.Tensor:
        n = _lib.query_size("adx_mlp_workspace_bytes", B, KMAX)
        if self._ws is None or self._ws.numel() < n:
            self._ws = torch.empty(n, dtype=torch.uint8, device=self.device)
        return self._ws

    def forward(self, X: torch.Tensor, prior: torch.Tensor) -> torch.Tensor:
        """Q [B, 16] (float32) for features X [B, 33] and prior [B, 16]."""
        B = X.shape[0]
        ws = self._workspace(B)
        out = torch.empty((B, KMAX), dtype=torch.float32, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.call("adx_mlp_forward", X.data_ptr(), prior.data_ptr(), self.wb["W1"].data_ptr(), self.w["b1"].data_ptr(),
                  self.wb["W2"].data_ptr(), self.w["b2"].data_ptr(), self.wb["W3"].data_ptr(),
                  self.w["b3"].data_ptr(), B, KMAX, out.data_ptr(), ws.data_ptr(), ws.numel(), st)
        return out

    def gradients(self, X: torch.Tensor, prior: torch.Tensor, T: torch.Tensor) -> float:
        """Forward + backward on one batch; gradients land in ``self.g``; returns the loss."""
        B = X.shape[0]
        self.forward(X, prior)
        ws = self._workspace(B)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        g = self.g
        _lib.call("adx_mlp_backward", X.data_ptr(), T.data_ptr(), self.wb["W2"].data_ptr(), self.wb["W3"].data_ptr(),
                  B, KMAX, g["W1"].data_ptr(), g["b1"].data_ptr(), g["W2"].data_ptr(), g["b2"].data_ptr(),
                  g["W3"].data_ptr(), g["b3"].data_ptr(), loss.data_ptr(), ws.data_ptr(), ws.numel(), st)
        return loss

    def step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.t += 1
        st = torch.cuda.current_stream(self.device).cuda_stream
        for k in self.w:
            wb = self.wb.get(k)
            _lib.call("adx_mlp_adam", self.w[k].data_ptr(), None if wb is None else wb.data_ptr(),
                      self.g[k].data_ptr(), self.m[k].data_ptr(), self.v[k].data_ptr(), self.w[k].numel(),
                      float(lr), float(beta1), float(beta2), float(eps), self.t, st)

    def loss(self, X: torch.Tensor, prior: torch.Tensor, T: torch.Tensor, batch: int = 16384) -> float:
        """Mean cross-entropy of the current weights on a data set (forward passes only)."""
        tot = 0.0
        for s in range(0, X.shape[0], batch):
            p = self.forward(X[s:s + batch].contiguous(), prior[s:s + batch].contiguous())
            tot += float(-(T[s:s + batch] * torch.log(p.clamp_min(1e-30))).sum())
        return tot / X.shape[0]

    def train(self, X: torch.Tensor, prior: torch.Tensor, T: torch.Tensor, epochs: int = 30,
              batch: int = 4096, lr: float = 1e-3, seed: int = 0, val=None) -> list[float]:
        """Minibatch Adam on (X, prior, T); returns the mean training loss per epoch. With
        ``val = (Xv, prior_v, Tv)`` (held-out cohorts), the weights kept at the end are
        those of the epoch with the lowest validation loss -- the untrained start, which
        returns the prior, included -- so the network departs from the ALS start only as
        far as that generalises; ``self.val_history`` records the validation losses."""
        n = X.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        hist = []
        best = None
        if val is not None:
            self.val_history = [self.loss(*val)]
            best = (self.val_history[0], {k: v.clone() for k, v in self.w.items()})
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g, device=self.device)
            tot, cnt = torch.zeros((), device=self.device), 0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                loss = self.gradients(X[idx].contiguous(), prior[idx].contiguous(), T[idx].contiguous())
                self.step(lr)
                tot += loss[0] * idx.numel()
                cnt += idx.numel()
            hist.append(float(tot) / cnt)
            if val is not None:
                vl = self.loss(*val)
                self.val_history.append(vl)
                if vl < best[0]:
                    best = (vl, {k: v.clone() for k, v in self.w.items()})
        if best is not None:
            for k in self.w:
                self.w[k].copy_(best[1][k])
            self._refresh_bf16()
        return hist

    def save(self, path) -> None:
        np.savez_compressed(path, **{k: v.cpu().numpy() for k, v in self.w.items()})

    @classmethod
    def load(cls, path, device) -> "WarmStartMLP":
        net = cls(device)
        with np.load(path) as z:
            for k in net.w:
                net.w[k].copy_(torch.from_numpy(z[k]))
        net._refresh_bf16()
        return net


# ---------------------------------------------------------------- features and M-step

def canonical_scores(U: torch.Tensor, S: torch.Tensor, V: torch.Tensor) -> torch.Tensor:
    """V S with each column's sign fixed by its largest-magnitude SNP loading."""
    piv = torch.argmax(torch.abs(U), dim=0)
    sign = torch.sign(U[piv, torch.arange(U.shape[1], device=U.device)])
    sign[sign == 0] = 1
    return V * S * sign


def sample_features(G, M: int, U, S, V, Q_als: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(X [N, 33] float32, prior [N, 16] float32) for the network."""
    N, K = Q_als.shape
    dev = Q_als.device
    sc = canonical_scores(U, S, V)[:, :N_SCORES].float()
    sc = (sc - sc.mean(0)) / sc.std(0).clamp_min(1e-12)
    if sc.shape[1] < N_SCORES:
        sc = torch.cat([sc, torch.zeros((N, N_SCORES - sc.shape[1]), device=dev)], 1)
    obs = ops.sample_counts(G, M) / 2.0
    het = (ops.sample_het_counts(G, M) / obs.clamp_min(1.0)).float().unsqueeze(1)
    q = torch.zeros((N, KMAX), dtype=torch.float32, device=dev)
    q[:, :K] = Q_als.float()
    X = torch.cat([q, sc, het], 1).contiguous()
    prior = torch.full((N, KMAX), PAD_PRIOR, dtype=torch.float32, device=dev)
    prior[:, :K] = torch.log(Q_als.float().clamp_min(1e-5))
    return X, prior.contiguous()


def m_step_P(G, Q: torch.Tensor, M: int) -> torch.Tensor:
    """P_jk = sum_i g Q_ik / (2 sum_i obs Q_ik), clamped (float64 [M, K])."""
    Qf = Q.float().contiguous()
    zero = torch.zeros(M, dtype=torch.float32, device=Q.device)
    half = torch.full((M,), 0.5, dtype=torch.float32, device=Q.device)
    num = ops.rsvd_rows(G, zero, Qf, M).double()          # sum over observed of g Q
    shifted = ops.rsvd_rows(G, half, Qf, M).double()      # sum over observed of (g - 1) Q
    den = 2.0 * (num - shifted)                            # 2 sum over observed of Q
    return (num / den.clamp_min(1e-12)).clamp(1e-5, 1.0 - 1e-5)


def em_m_step_P(G, P: torch.Tensor, Q: torch.Tensor, M: int) -> torch.Tensor:
    """P of one EM step from (P, Q): the E-step statistics at (P, Q), then the P target of
    em_final_update (adamixture/model/em_adam_gpu.py:82-117), float64."""
    A, B, T = ops.em_stats(G, P.contiguous(), Q.contiguous(), M, "f64")
    q_bat = ops.sample_counts(G, M)
    P_EM, _ = ops.em_targets(P.contiguous(), Q.contiguous(), A, B, T, q_bat)
    return P_EM


def predict(net: WarmStartMLP, G, M: int, U, S, V, Q_als: torch.Tensor, P_als: torch.Tensor | None = None,
            p_rule: str = "em") -> tuple[torch.Tensor, torch.Tensor]:
    """Warm start (P0, Q0), float64. ``p_rule``: "em" -- P of one EM step from (P_als, Q0);
    "freq" -- the membership-weighted allele frequencies of ``m_step_P``."""
    K = Q_als.shape[1]
    X, prior = sample_features(G, M, U, S, V, Q_als)
    Q0 = net.forward(X, prior)[:, :K].double().clamp(1e-5, 1.0 - 1e-5)
    Q0 = Q0 / Q0.sum(1, keepdim=True)
    if p_rule == "em" and P_als is not None:
        return em_m_step_P(G, P_als.double(), Q0, M), Q0
    return m_step_P(G, Q0, M), Q0


# ---------------------------------------------------------------- training data and runs

HP = dict(lr=0.005, beta1=0.80, beta2=0.88, reg_adam=1e-8, check=5, lr_decay=0.5, min_lr=1e-4,
          patience=3, tol=0.1)


def init_als(G, N, M, K, seed=42, power=5, tol_svd=0.1):
    f = ops.allele_frequency(G, M)
    U, S, V = SVD_gpu(G, N, M, f, max(K, N_SCORES), seed, power, tol_svd, 8192, G.device, 256)
    P, Q = ALS_gpu(U[:, :K].contiguous(), S[:K].contiguous(), V[:, :K].contiguous(), f, seed, M, K, 1000, 1e-4,
                   G.device)
    return U, S, V, P, Q


def run_em(G, N, M, K, P0, Q0, precision=None, max_iter=10000):
    """Plain Adam-EM to convergence with the reference's settings; (P, Q, loglik, trace)."""
    trace: list = []
    P, Q = optimize_parameters_gpu(G, P0.clone(), Q0.clone(), HP["lr"], HP["beta1"], HP["beta2"], HP["reg_adam"],
                                   max_iter, HP["check"], K, M, N, HP["lr_decay"], HP["min_lr"], HP["patience"],
                                   HP["tol"], G.device, 8192, 256, precision=precision, trace=trace)
    return P, Q, loglikelihood_gpu(G, P, Q, M, N, 8192, G.device, 256), trace


def simulate(N, M, K, F, seed, device, alpha=0.5, miss=0.01):
    from ..src.simulate import make_cohort

    coh = make_cohort(N, M, K, F, alpha, miss, seed)
    Pq = torch.from_numpy(coh.Pq.astype(np.int32)).to(device)
    Qq = torch.from_numpy(coh.Qq.astype(np.int32)).to(device)
    return ops.simulate_packed(Pq, Qq, coh.miss_q, coh.keys), coh


def training_set(cohorts, device, precision=None):
    """(X, prior, T) pooled over seeded cohorts given as (N, M, K, F, seed) tuples."""
    Xs, Ps, Ts = [], [], []
    for (N, M, K, F, seed) in cohorts:
        G, _ = simulate(N, M, K, F, seed, device)
        U, S, V, P0, Q0 = init_als(G, N, M, K, seed)
        _, Q_em, _, _ = run_em(G, N, M, K, P0, Q0, precision)
        X, prior = sample_features(G, M, U, S, V, Q0)
        T = torch.zeros((N, KMAX), dtype=torch.float32, device=device)
        T[:, :K] = Q_em.float()
        Xs.append(X), Ps.append(prior), Ts.append(T)
        del G
    return torch.cat(Xs), torch.cat(Ps), torch.cat(Ts)


def iterations_to_reach(trace, target: float, rel: float = 1e-6):
    """First traced iteration whose log-likelihood is within ``rel`` of ``target``."""
    for it, L, *_ in trace:
        if L >= target - rel * abs(target):
            return it
    return None


def warm_start_fit(net: WarmStartMLP, G, N: int, M: int, K: int, seed: int = 42, precision=None) -> dict:
    """Plain EM from the ALS start and EM from the network's warm start on the same data;
    the warm result is kept only if its log-likelihood is no worse than the plain one's
    (within 1e-6 relative). Returns both runs' log-likelihoods, wall times and iterations
    to reach the plain run's converged log-likelihood."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    U, S, V, P_als, Q_als = init_als(G, N, M, K, seed)
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t0
    t0 = time.perf_counter()
    P_p, Q_p, L_p, tr_p = run_em(G, N, M, K, P_als, Q_als, precision)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0 + t_init
    t0 = time.perf_counter()
    P_w0, Q_w0 = predict(net, G, M, U, S, V, Q_als, P_als)
    torch.cuda.synchronize()
    t_pred = time.perf_counter() - t0
    P_w, Q_w, L_w, tr_w = run_em(G, N, M, K, P_w0, Q_w0, precision)
    torch.cuda.synchronize()
    t_warm = time.perf_counter() - t0 + t_init
    keep = L_w >= L_p - 1e-6 * abs(L_p)
    target = max(e[1] for e in tr_p) if tr_p else None

    def seconds_to(trace, extra):
        for it, L, sec in trace:
            if L >= target - 1e-6 * abs(target):
                return sec + extra
        return None

    return {
        "loglik_plain": L_p, "loglik_warm": L_w, "kept_warm": bool(keep),
        "seconds_plain": t_plain, "seconds_warm": t_warm, "seconds_init": t_init, "seconds_predict": t_pred,
        # wall time from the start of initialisation to the first check within 1e-6 of the
        # plain run's converged log-likelihood
        "seconds_to_target_plain": seconds_to(tr_p, t_init) if tr_p else None,
        "seconds_to_target_warm": seconds_to(tr_w, t_init + t_pred) if tr_p else None,
        # traced values share the runs' log-likelihood arithmetic: compare within it
        "iters_plain": iterations_to_reach(tr_p, max(e[1] for e in tr_p)) if tr_p else None,
        "iters_warm_to_plain": iterations_to_reach(tr_w, max(e[1] for e in tr_p)) if tr_p else None,
        "loglik_init_als": loglikelihood_gpu(G, P_als, Q_als, M, N, 8192, G.device, 256),
        "loglik_init_warm": loglikelihood_gpu(G, P_w0, Q_w0, M, N, 8192, G.device, 256),
        "loglik_init_als_P_warm_Q": loglikelihood_gpu(G, P_als, Q_w0, M, N, 8192, G.device, 256),
        "P": P_w if keep else P_p, "Q": Q_w if keep else Q_p,
    }


DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "warm_start_weights.npz"


def train_default(device, out=DEFAULT_WEIGHTS, n_train: int = 50, n_val: int = 5, size=(20_000, 50_000),
                  epochs: int = 30, seed: int = 0) -> dict:
    """Train the shipped weights: 50 seeded synthetic cohorts of N=20,000 x M=50,000 (K in
    6..10, F in 0.02..0.15, Dirichlet(0.5) memberships, 1% missing) fitted by plain EM from
    the ALS start; 5 more cohorts select the epoch. Reproducible from the seeds
    (``python bench.py --config c5 --train`` runs it and evaluates the result)."""
    rng = np.random.default_rng(seed)
    N, M = size
    spec = [(N, M, int(rng.integers(6, 11)), float(rng.uniform(0.02, 0.15)), 5000 + c)
            for c in range(n_train + n_val)]
    X, P, T = training_set(spec[:n_train], device)
    Xv, Pv, Tv = training_set(spec[n_train:], device)
    net = WarmStartMLP(device, seed)
    hist = net.train(X, P, T, epochs=epochs, batch=2048, lr=5e-4, val=(Xv, Pv, Tv))
    if out is not None:
        net.save(out)
    return {"train_loss": hist, "val_loss": net.val_history, "cohorts": spec}
