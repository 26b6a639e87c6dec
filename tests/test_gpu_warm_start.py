"""The warm-start network on the GPU: forward and gradients of the CUDA kernels against
the float64 oracle (oracle/mlp.py) with the same BF16 weights and the kernels' BF16
rounding of every product's inputs (gradients within 5e-3 of each tensor's largest
magnitude, outputs within 1e-4: float32 accumulation over 256-wide layers and a batch sum,
and float32 activations that differ from the oracle's float64 ones in their last bits
rounding to a neighbouring BF16 value),
the untrained network reproducing its prior, training lowering the loss, the one-step
M-step against numpy, and a warm-started fit on a held-out cohort (network trained on
seeded cohorts by these kernels), whose result is never worse than plain EM."""
import numpy as np
import pytest
import torch

from oracle import em_oracle as orc
from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws(cuda):
    from adamixture_b200.model import warm_start

    return warm_start


def _rand_batch(B, K, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(B, 33)).astype(np.float32)
    q = rng.dirichlet(np.ones(K), B)
    prior = np.full((B, 16), -30.0, dtype=np.float32)
    prior[:, :K] = np.log(q)
    T = np.zeros((B, 16), dtype=np.float32)
    T[:, :K] = rng.dirichlet(np.ones(K) * 0.5, B)
    return X, prior, T


def test_forward_and_gradients_vs_oracle(ws):
    net = ws.WarmStartMLP("cuda", seed=3)
    # give the last layer non-zero weights so every gradient path is exercised
    net.w["W3"].copy_(torch.randn(16, 256, generator=torch.Generator().manual_seed(5)) * 0.05)
    net.w["b1"].copy_(torch.linspace(-0.5, 0.5, 256))
    net._refresh_bf16()
    X, prior, T = _rand_batch(300, 6, 0)
    Xd, Pd, Td = (torch.from_numpy(a).cuda() for a in (X, prior, T))
    Q = net.forward(Xd, Pd).cpu().numpy()
    W = {k: net.wb[k].float().cpu().numpy().astype(np.float64) for k in ("W1", "W2", "W3")}
    b = {k: net.w[k].cpu().numpy().astype(np.float64) for k in ("b1", "b2", "b3")}
    cache = omlp.forward(X.astype(np.float64), prior, W["W1"], b["b1"], W["W2"], b["b2"], W["W3"], b["b3"])
    # a float32 activation next to a BF16 rounding boundary can round one BF16 step away
    # from the oracle's float64 one: a few outputs move by up to ~1e-4
    np.testing.assert_allclose(Q, cache["p"], atol=1e-4)
    loss = float(net.gradients(Xd, Pd, Td)[0])
    loss0, g0 = omlp.backward(X.astype(np.float64), T.astype(np.float64), W["W2"], W["W3"], cache)
    assert abs(loss - loss0) <= 5e-5 * abs(loss0)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        got = net.g[k].cpu().numpy()
        scale = np.abs(g0[k]).max()
        assert np.abs(got - g0[k]).max() <= 5e-3 * scale, (k, np.abs(got - g0[k]).max(), scale)


def test_untrained_network_returns_its_prior_and_training_lowers_the_loss(ws):
    net = ws.WarmStartMLP("cuda", seed=1)
    X, prior, T = _rand_batch(4096, 5, 1)
    Xd, Pd, Td = (torch.from_numpy(a).cuda() for a in (X, prior, T))
    Q = net.forward(Xd, Pd).cpu().numpy()
    np.testing.assert_allclose(Q[:, :5], np.exp(prior[:, :5]), atol=1e-6)
    hist = net.train(Xd, Pd, Td, epochs=20, batch=512, lr=2e-3)
    assert hist[-1] < 0.9 * hist[0], hist


def test_m_step_P_vs_numpy(ws, synth):
    M = int(synth["M"])
    G = orc.unpack(synth["packed"], M)
    Q = synth["Q0"]
    P = ws.m_step_P(torch.from_numpy(synth["packed"]).cuda(), torch.from_numpy(Q).cuda(), M).cpu().numpy()
    obs = (G != 3).astype(np.float64)
    num = np.where(G != 3, G, 0).astype(np.float64) @ Q
    den = 2.0 * obs @ Q
    np.testing.assert_allclose(P, np.clip(num / den, 1e-5, 1 - 1e-5), rtol=2e-5, atol=1e-7)


def test_warm_started_fit_on_a_held_out_cohort(ws):
    dev = torch.device("cuda")
    cohorts = [(3000, 6000, 4, F, 100 + s) for s, F in enumerate((0.03, 0.06, 0.1, 0.15))]
    X, prior, T = ws.training_set(cohorts, dev)
    net = ws.WarmStartMLP(dev, seed=0)
    hist = net.train(X, prior, T, epochs=40, batch=2048, lr=1e-3)
    assert hist[-1] < hist[0]
    G, _ = ws.simulate(4000, 8000, 4, 0.08, 999, dev)
    r = ws.warm_start_fit(net, G, 4000, 8000, 4)
    print({k: v for k, v in r.items() if k not in ("P", "Q")})
    # the fallback rule: the returned model is never worse than plain EM's
    L = ws.loglikelihood_gpu(G, r["P"], r["Q"], 8000, 4000, 8192, dev, 256)
    assert L >= r["loglik_plain"] - 1e-6 * abs(r["loglik_plain"])


def test_shipped_network_gain_on_a_held_out_cohort(ws):
    # What the shipped network (trained on 50 cohorts of N=20,000 x M=50,000, K 6..10, seeds
    # 5000..5054) gains over the reference's ALS start on a cohort it has not seen (seed 7777):
    # iterations and seconds to the first check within 1e-6 relative of plain EM's converged
    # log-likelihood, printed. The warm run must reach that log-likelihood, and the fallback
    # keeps the returned model no worse than plain EM's. Measured: 50 against 55 iterations
    # here (0.30 against 0.29 s with the prediction); on two held-out cohorts of config 5
    # (N=100,000 x M=300,000, K=8; bench.py --config c5) 100 against 110 and 95 against 90
    # iterations: no consistent gain.
    dev = torch.device("cuda")
    net = ws.WarmStartMLP.load(ws.DEFAULT_WEIGHTS, dev)
    N, M, K = 20_000, 50_000, 8
    G, _ = ws.simulate(N, M, K, 0.05, 7777, dev)
    r = ws.warm_start_fit(net, G, N, M, K)
    print("held-out gain: iterations", r["iters_plain"], "->", r["iters_warm_to_plain"],
          "seconds to target", r["seconds_to_target_plain"], "->", r["seconds_to_target_warm"])
    assert r["iters_warm_to_plain"] is not None
    L = ws.loglikelihood_gpu(G, r["P"], r["Q"], M, N, 8192, dev, 256)
    assert L >= r["loglik_plain"] - 1e-6 * abs(r["loglik_plain"])
