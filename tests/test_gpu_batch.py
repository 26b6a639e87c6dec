"""The batched float64 E-step (the K sweep and its cross-validation folds in one launch)
against the single-problem path.

Bars: every problem's statistics are bit-identical to the single-problem float64 sweep on
the same genotypes with the problem's fold hidden; whole batched fits and fold polishes are
bit-identical to running each problem alone (so within the 1e-12 the batch is held to);
each fold of the 10-bucket hash rule holds out 10 % of the observed entries.
"""
import numpy as np
import pytest
import torch

from oracle import em_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops(cuda):
    from adamixture_b200 import ops as _ops

    return _ops


def _cohort(N, M, K, seed):
    from adamixture_b200.src.simulate import make_cohort

    coh = make_cohort(N, M, K, F=0.08, alpha=0.5, miss=0.01, seed=seed)
    return torch.from_numpy(orc.pack(coh.genotypes())).cuda()


def _start(M, N, K, seed):
    rng = np.random.default_rng(seed)
    P0 = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q0 = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
    Q0 /= Q0.sum(1, keepdims=True)
    return torch.from_numpy(P0).cuda(), torch.from_numpy(Q0).cuda()


@pytest.mark.parametrize("N,M", [(1000, 777), (2048, 301)])
def test_batched_stats_equal_single_problem_sweeps(ops, N, M):
    from adamixture_b200.model.em_adam_batch import fold_copy

    G = _cohort(N, M, 4, N + M)
    Ks = [2, 5, 10, 16, 3, 12]
    folds = [-1, 0, 3, -1, 9, 4]
    seed = 42
    starts = [_start(M, N, K, 10 + i) for i, K in enumerate(Ks)]
    Gs = [G if f < 0 else fold_copy(G, M, seed, 10, f) for f in folds]
    batch = ops.EmBatch(M, N, Ks, G.device)
    batch.sweep(Gs, [s[0] for s in starts], [s[1] for s in starts])
    for p, (K, f) in enumerate(zip(Ks, folds)):
        A, B, T = batch.stats(p)
        A1, B1, T1 = ops.em_stats(Gs[p], starts[p][0], starts[p][1], M, "f64")
        for got, ref in ((A, A1), (B, B1), (T, T1)):
            assert torch.equal(got, ref), (K, f, float((got - ref).abs().max()))
        # and against the float64 oracle on the masked genotypes
        Gu = orc.unpack(Gs[p].cpu().numpy(), M)
        A0, B0, T0, _ = orc.em_stats(Gu, starts[p][0].cpu().numpy(), starts[p][1].cpu().numpy())
        for got, ref in ((A, A0), (B, B0), (T, T0)):
            err = np.abs(got.cpu().numpy() - ref).max() / np.abs(ref).max()
            assert err <= 1e-12, (K, f, err)


def test_fold_rule_holds_out_ten_percent(ops):
    from adamixture_b200.model.em_adam_batch import fold_counts

    N, M = 3000, 2000
    G = _cohort(N, M, 3, 5)
    total = float(ops.sample_counts(G, M).sum().item()) / 2
    for f in range(5):
        held = total - float(fold_counts(G, M, 42, 10, f).sum().item()) / 2
        assert abs(held / total - 0.1) < 0.005, (f, held / total)


def test_batched_cross_validation_equals_sequential(ops):
    from adamixture_b200.model.em_adam_batch import cross_validate

    N, M = 1500, 3000
    G = _cohort(N, M, 4, 7)
    Ks = [2, 3, 4, 6, 9]
    starts = {K: _start(M, N, K, 100 + K) for K in Ks}
    kw = dict(n_folds=5, n_buckets=10, seed=42, polish_iters=6, max_iter=80)
    b = cross_validate(G, M, N, Ks, starts, batched=True, **kw)
    s = cross_validate(G, M, N, Ks, starts, batched=False, **kw)
    for K in Ks:
        for x, y in zip(b["fits"][K], s["fits"][K]):
            assert float((x - y).abs().max()) <= 1e-12, K
        for f in range(5):
            for x, y in zip(b["folds"][(K, f)], s["folds"][(K, f)]):
                assert float((x - y).abs().max()) <= 1e-12, (K, f)
        assert abs(b["cv"][K] - s["cv"][K]) <= 1e-12 * abs(s["cv"][K]), K
    print("cv index", b["cv"], "seconds batched", b["seconds"], "sequential", s["seconds"])
