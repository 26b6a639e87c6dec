"""GPU checks of the tensor-core (tcgen05, FP32 accumulation) E-step with BF16 or FP16
operands.

The statistics are compared with the float64 oracle / reference per statistic, as the
max abs error relative to the largest magnitude and the relative Frobenius error: at the
BF16 bar (operands rounded to 8 significant bits) max <= 2e-2, Frobenius <= 4e-3; at the
FP16 bar (11 significant bits, power-of-two-scaled operands) max <= 5e-3, Frobenius <= 1e-3.
The converged log-likelihood is within 1e-4 relative of the reference's float64 run.
"""
import numpy as np
import pytest
import torch

from oracle import em_oracle as orc

pytestmark = pytest.mark.gpu


def dev_t(x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t if dtype is None else t.to(dtype)


BARS = {"bf16": (2e-2, 4e-3), "f16": (5e-3, 1e-3)}


def check_stats(got, ref, name, prec="bf16"):
    g = got.cpu().numpy()
    scale = np.abs(ref).max()
    mx = np.abs(g - ref).max() / scale
    fro = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    print(prec, name, f"max {mx:.2e} fro {fro:.2e}")
    bmx, bfro = BARS[prec]
    assert mx <= bmx and fro <= bfro, (prec, name, mx, fro)
    return mx, fro


@pytest.fixture(scope="module")
def ops(cuda):
    from adamixture_b200 import ops as _ops

    return _ops


@pytest.fixture(params=["bf16", "f16"])
def prec(request):
    return request.param


@pytest.mark.parametrize("N,M,K", [(130, 130, 8), (1001, 523, 8), (1030, 900, 10),
                                   (257, 1800, 16), (300, 1000, 1), (64, 2000, 12)])
def test_tc_stats_vs_oracle(ops, prec, N, M, K):
    rng = np.random.default_rng(N + M + K)
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    P = np.clip(rng.beta(0.8, 0.8, size=(M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    A0, B0, T0, _ = orc.em_stats(G, P, Q)
    A, B, T = ops.em_stats(dev_t(orc.pack(G)), dev_t(P, torch.float32), dev_t(Q, torch.float32), M, prec)
    for got, ref, nm in ((A, A0, "A"), (B, B0, "B"), (T, T0, "T")):
        check_stats(got, ref, nm, prec)


@pytest.mark.parametrize("name", ["demo", "synth", "edge"])
def test_tc_stats_vs_reference(ops, prec, name, request):
    d = request.getfixturevalue(name)
    M = int(d["M"])
    A, B, T = ops.em_stats(dev_t(d["packed"]), dev_t(d["P0"], torch.float32),
                           dev_t(d["Q0"], torch.float32), M, prec)
    for got, nm in ((A, "A"), (B, "B"), (T, "T")):
        check_stats(got, d[nm], nm, prec)


def test_tc_many_tiles_and_splits(ops, prec):
    # several SNP blocks of 896, sample splits, ragged last tiles, N a multiple of 16
    rng = np.random.default_rng(2)
    N, M, K = 3 * 1024 + 16, 2 * 896 + 300, 10
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    P = np.clip(rng.beta(0.8, 0.8, size=(M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    A0, B0, T0, _ = orc.em_stats(G, P, Q)
    A, B, T = ops.em_stats(dev_t(orc.pack(G)), dev_t(P, torch.float32), dev_t(Q, torch.float32), M, prec)
    for got, ref, nm in ((A, A0, "A"), (B, B0, "B"), (T, T0, "T")):
        check_stats(got, ref, nm, prec)


def test_tc_extreme_frequencies(ops, prec):
    # P at the domain bounds, pure Q rows: h near 1e-5 and near 1-1e-5, where the
    # complement MMA keeps 1-h accurate
    rng = np.random.default_rng(9)
    N, M, K = 256, 512, 8
    P = rng.choice([1e-5, 1 - 1e-5, 0.5], size=(M, K))
    Q = np.full((N, K), 1e-5)
    Q[np.arange(N), rng.integers(0, K, N)] = 1 - (K - 1) * 1e-5
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    A0, B0, T0, _ = orc.em_stats(G, P, Q)
    A, B, T = ops.em_stats(dev_t(orc.pack(G)), dev_t(P, torch.float32), dev_t(Q, torch.float32), M, prec)
    for got, ref, nm in ((A, A0, "A"), (B, B0, "B"), (T, T0, "T")):
        check_stats(got, ref, nm, prec)


def test_tc_status_word_clear(ops, prec, synth):
    M, N, K = int(synth["M"]), int(synth["N"]), int(synth["K"])
    ws = ops.Workspace.get(torch.device("cuda"), ops.em_workspace_bytes(M, N, K, prec))
    ops.em_sweep(dev_t(synth["packed"]), dev_t(synth["P0"], torch.float32),
                 dev_t(synth["Q0"], torch.float32), M, prec, ws)
    assert ops.em_status(ws, M, N, K, prec) == 0


def test_bounded_wait_gives_up_and_reports(ops):
    # the wait the sweep uses at every producer/consumer hand-off, on a barrier nothing
    # arrives at: it gives up after its poll limit, reports a timeout and raises the abort
    # word, which a second waiting warp honours at once; with the arrival both complete
    assert ops.tc_wait_selftest(False, 2000) == [5, 1, 5]
    assert ops.tc_wait_selftest(True, 2000) == [0, 0, 0]


def test_optimiser_raises_on_a_sweep_timeout(ops, synth, monkeypatch):
    # a sweep that timed out leaves ADX_ERR_TIMEOUT in its workspace's status word; the
    # optimiser's next check must raise (here the word is set by hand in the optimiser's own
    # workspace), and the read clears it
    from adamixture_b200.model.em_adam_gpu import optimize_parameters_gpu

    M, N, K = int(synth["M"]), int(synth["N"]), int(synth["K"])
    G = dev_t(synth["packed"])
    made = []
    plain = ops.em_workspace

    def with_timeout_status(*args, **kw):
        ws = plain(*args, **kw)
        ws[:4].copy_(torch.tensor([5, 0, 0, 0], dtype=torch.uint8))
        made.append(ws)
        return ws

    monkeypatch.setattr(ops, "em_workspace", with_timeout_status)
    with pytest.raises(RuntimeError, match="status 5"):
        optimize_parameters_gpu(G, dev_t(synth["P0"]), dev_t(synth["Q0"]), 0.005, 0.80, 0.88, 1e-8, 10, 5, K,
                                M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 512, precision="f16")
    assert len(made) == 1 and ops.em_status(made[0], M, N, K, "f16") == 0


@pytest.mark.parametrize("name", ["demo", "synth"])
def test_tc_converged_loglik(ops, prec, name, request):
    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu

    d = request.getfixturevalue(name)
    M, N, K = int(d["M"]), int(d["N"]), int(d["K"])
    G = dev_t(d["packed"])
    P, Q = optimize_parameters_gpu(G, dev_t(d["P0"]), dev_t(d["Q0"]), 0.005, 0.80, 0.88, 1e-8,
                                   10000, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 512,
                                   precision=prec)
    L = loglikelihood_gpu(G, P, Q, M, N, 8192, G.device, 512)
    ref = float(d["conv_loglik"])
    print(name, prec, "converged loglik", L, "reference", ref, "rel", abs(L - ref) / abs(ref))
    # FP16 operands (the default): the 1e-6 relative bar of the converged fit (measured
    # 1.2e-7 on demo, 7.4e-9 on synth). BF16 operands round 8x coarser; their bar is set
    # at the measured gap (4.1e-6 on demo, 3.6e-7 on synth) with headroom, not at 1e-6.
    bar = 1e-6 if prec == "f16" else 1e-5
    assert abs(L - ref) <= bar * abs(ref)


@pytest.mark.parametrize("name", ["demo", "synth"])
def test_mixed_precision_reaches_the_float32_fit(ops, name, request):
    # BF16 tensor-core sweeps to the first plateau, float32 after it: the converged
    # log-likelihood matches the plain float32 run's within 1e-6 relative
    import time

    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu

    d = request.getfixturevalue(name)
    M, N, K = int(d["M"]), int(d["N"]), int(d["K"])
    G = dev_t(d["packed"])
    out = {}
    for prec in ("f32", "mixed"):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        P, Q = optimize_parameters_gpu(G, dev_t(d["P0"]), dev_t(d["Q0"]), 0.005, 0.80, 0.88, 1e-8, 10000, 5, K,
                                       M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 512, precision=prec)
        torch.cuda.synchronize()
        out[prec] = (loglikelihood_gpu(G, P, Q, M, N, 8192, G.device, 512), time.perf_counter() - t0)
    print(name, "f32", out["f32"], "mixed", out["mixed"])
    L32, Lm = out["f32"][0], out["mixed"][0]
    assert abs(Lm - L32) <= 1e-6 * abs(L32)


@pytest.mark.parametrize("K", [1, 2, 3, 5])
def test_f16_converged_fit_at_small_k(ops, K):
    # the default E-step for every K <= 16: its converged log-likelihood against this
    # library's float64 fit (the reference's arithmetic) from the same start
    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu
    from adamixture_b200.src.simulate import make_cohort

    N, M = 1500, 6000
    coh = make_cohort(N, M, K, F=0.1, alpha=0.5, miss=0.01, seed=70 + K)
    G = dev_t(orc.pack(coh.genotypes()))
    rng = np.random.default_rng(K)
    P0 = rng.uniform(0.2, 0.8, (M, K))
    Q0 = rng.dirichlet(np.ones(K), N)
    out = {}
    for prec in ("f64", "f16"):
        P, Q = optimize_parameters_gpu(G, dev_t(P0), dev_t(Q0), 0.005, 0.80, 0.88, 1e-8, 10000, 5, K, M, N,
                                       0.5, 1e-4, 3, 0.1, G.device, 8192, 512, precision=prec)
        out[prec] = loglikelihood_gpu(G, P, Q, M, N, 8192, G.device, 512)
    rel = (out["f16"] - out["f64"]) / abs(out["f64"])
    print("K", K, "f64", out["f64"], "f16", out["f16"], "rel", rel)
    assert abs(rel) <= 1e-5
