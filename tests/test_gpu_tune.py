"""The float64 sweep's tile layouts and their autotuner (adamixture_b200/tune.py).

Bar: a layout changes where values sit in shared memory and how many CTAs share an SM,
never the arithmetic or its order, so every statistic, partial sum and log-likelihood is
bit-identical across layouts (ragged shapes included: N not a multiple of the 256-sample
sub-tile or of 8, M not a multiple of the 16-SNP chunk or of 4); the tuner picks a valid
layout, records it in the library and in its cache, and the fits it tunes equal untuned
fits bit for bit.
"""
import numpy as np
import pytest
import torch

from oracle import em_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture()
def tune(cuda):
    from adamixture_b200 import tune as _tune

    before = {k: _tune.get_tile(k, 0) for k in range(1, 17)}
    yield _tune
    for k, t in before.items():
        _tune.set_tile(k, t, 0)


def _cohort(N, M, K, seed, miss=0.02):
    rng = np.random.default_rng(seed)
    g = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.35 - miss, miss]).astype(np.uint8)
    P = np.clip(rng.beta(0.8, 0.8, size=(M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    G = torch.from_numpy(orc.pack(g)).cuda()
    return G, torch.from_numpy(P).cuda(), torch.from_numpy(Q).cuda()


SHAPES = [(1037, 3005), (256, 16), (2048, 777), (9, 5)]


@pytest.mark.parametrize("K", [1, 2, 3, 4, 5, 7, 8])
@pytest.mark.parametrize("N,M", SHAPES)
def test_layouts_give_bit_identical_statistics(tune, K, N, M):
    from adamixture_b200 import ops

    assert tune.tiles(K) == 2
    G, P, Q = _cohort(N, M, K, seed=17 * K + N)
    out = {}
    for tile in (0, 1):
        tune.set_tile(K, tile, 0)
        assert tune.get_tile(K, 0) == tile
        out[tile] = ops.em_stats(G, P, Q, M, "f64")
    for a, b, nm in zip(out[0], out[1], "ABT"):
        assert torch.equal(a, b), (nm, float((a - b).abs().max()))
    # and the float64 oracle agrees with both (the statistics are right, not just equal)
    A0, B0, T0, _ = orc.em_stats(orc.unpack(G.cpu().numpy(), M), P.cpu().numpy(), Q.cpu().numpy())
    for got, ref in zip(out[1], (A0, B0, T0)):
        err = float(np.abs(got.cpu().numpy() - ref).max() / max(np.abs(ref).max(), 1e-300))
        assert err <= 1e-11, err


@pytest.mark.parametrize("K", [3, 8])
def test_layouts_give_bit_identical_folded_checks_and_block_ranges(tune, K):
    from adamixture_b200 import ops

    N, M = 1537, 4099
    G, P, Q = _cohort(N, M, K, seed=5 + K)
    ll, parts, ranges = {}, {}, {}
    spb, n_blocks, _ = ops.em_sweep_blocks_info(M, N, K)
    for tile in (0, 1):
        tune.set_tile(K, tile, 0)
        ws = ops.em_workspace(M, N, K, "f64", G.device)
        ops.em_sweep_loglik(G, P, Q, M, ws)
        ll[tile] = float(ops.em_loglik_from_sweep(ws, M, N, K).item())
        parts[tile] = ws.clone()
        ws2 = ops.em_workspace(M, N, K, "f64", G.device)
        cut = max(1, n_blocks // 3)
        ops.em_sweep_blocks(G, P, Q, M, 0, cut, ws2)
        ops.em_sweep_blocks(G, P, Q, M, cut, n_blocks, ws2)
        ranges[tile] = ws2
    assert ll[0] == ll[1]
    assert torch.equal(parts[0], parts[1])
    assert torch.equal(ranges[0], ranges[1])
    assert ll[0] == float(ops.loglik_device(G, P, Q, M, "f64").item())


def test_batch_launches_follow_the_layouts(tune):
    from adamixture_b200 import ops

    N, M = 1100, 2003
    Ks = [2, 5, 8, 10]
    data = [_cohort(N, M, k, seed=40 + k) for k in Ks]
    G = data[0][0]
    ref = [ops.em_stats(G, P, Q, M, "f64") for _, P, Q in data]
    for tiles in ((0, 0, 0, 0), (1, 1, 1, 0), (1, 0, 1, 0)):
        for k, t in zip(Ks, tiles):
            tune.set_tile(k, t, 0)
        groups = tune.batch_groups(Ks, 0)
        assert sorted(i for g in groups for i in g) == list(range(len(Ks)))
        assert len(groups) == len(set(tiles))
        for idx in groups:
            batch = ops.EmBatch(M, N, [Ks[i] for i in idx], G.device)
            batch.sweep([G] * len(idx), [data[i][1] for i in idx], [data[i][2] for i in idx])
            for p, i in enumerate(idx):
                for a, b in zip(batch.stats(p), ref[i]):
                    assert torch.equal(a, b)
    # a batch of K <= 8 problems whose layouts are all 1 runs layout 1 in one launch
    for k in Ks[:3]:
        tune.set_tile(k, 1, 0)
    batch = ops.EmBatch(M, N, Ks[:3], G.device)
    batch.sweep([G] * 3, [d[1] for d in data[:3]], [d[2] for d in data[:3]])
    for p in range(3):
        for a, b in zip(batch.stats(p), ref[p]):
            assert torch.equal(a, b)


def test_tuner_picks_records_and_caches(tune, tmp_path, monkeypatch):
    import json

    monkeypatch.setenv("ADX_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(tune, "_LOADED", False)
    monkeypatch.setattr(tune, "_CACHE", {})
    N, M, K = 4096, 6000, 4
    G, P, Q = _cohort(N, M, K, seed=3)
    t = tune.tune_dmma(G, P, Q, M)
    assert t in (0, 1) and tune.get_tile(K, 0) == t
    (key, rec), = tune.choices().items()
    assert f"K={K}" in key and rec["tile"] == t and set(rec["ms"]) == {"0", "1"}
    assert json.loads((tmp_path / "tune.json").read_text())[key]["tile"] == t
    # a cache hit sets the recorded layout without timing again
    tune.set_tile(K, 1 - t, 0)
    assert tune.tune_dmma(G, P, Q, M) == t and tune.get_tile(K, 0) == t
    # K > 8 has one layout: nothing to tune
    G2, P2, Q2 = _cohort(512, 300, 10, seed=4)
    assert tune.tune_dmma(G2, P2, Q2, 300) == 0


def test_tuned_fit_equals_untuned_fit(tune, monkeypatch):
    from adamixture_b200.model.em_adam_gpu import optimize_parameters_gpu

    N, M, K = 2000, 5000, 6
    G, P, Q = _cohort(N, M, K, seed=9)
    args = dict(lr=0.005, beta1=0.80, beta2=0.88, reg_adam=1e-8, max_iter=12, check=5, K=K, M=M, N=N,
                lr_decay=0.5, min_lr=1e-6, patience=3, tol_adam=0.1, device=G.device, chunk_size=4096,
                threads_per_block=256, precision="f64")
    monkeypatch.setenv("ADX_AUTOTUNE", "0")
    tune.set_tile(K, 0, 0)
    P0, Q0 = optimize_parameters_gpu(G, P, Q, **args)
    monkeypatch.setenv("ADX_AUTOTUNE", "1")
    tune.set_tile(K, 1, 0)   # whichever the tuner keeps, the fit is the same
    P1, Q1 = optimize_parameters_gpu(G, P, Q, **args)
    assert torch.equal(P0, P1) and torch.equal(Q0, Q1)


def test_invalid_layouts_are_rejected(tune):
    from adamixture_b200 import _lib

    assert tune.tiles(9) == 1 and tune.tiles(16) == 1 and tune.tiles(1) == 2
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        tune.set_tile(10, 1, 0)
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        tune.set_tile(3, 2, 0)
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        tune.tiles(17)
