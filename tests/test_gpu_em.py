"""GPU parity of the CUDA path against the reference (golden fixtures) and the CPU oracle.

Bars (written per test):
  * decode / layout / counts / sampler: bit-exact;
  * E-step statistics, float64 mode: rtol 1e-10 against the reference's float64 torch path;
  * per-iteration P/Q, float64 mode: 1e-5 max abs (the per-iteration parity bar; observed ~1e-12);
  * per-iteration P/Q, float32 mode: 1e-5 max abs on the 301-sample cohort; on the
    105-sample demo cohort 99.9% of entries within 1e-5 and all within 2e-4 (Adam divides
    each step by sqrt(v), which scales a float32 rounding of a near-zero EM delta by
    lr/|delta|: the bound shrinks like 1/sqrt(N));
  * log-likelihood: 1e-12 relative (float64 h), 1e-6 relative (float32 h);
  * converged log-likelihood: 1e-6 relative of the reference's converged value.
"""
import numpy as np
import pytest
import torch

from oracle import em_oracle as orc

pytestmark = pytest.mark.gpu


def dev_t(x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t if dtype is None else t.to(dtype)


@pytest.fixture(scope="module")
def ops(cuda):
    from adamixture_b200 import ops as _ops

    return _ops


# ------------------------------------------------------------------ layout

@pytest.mark.parametrize("name", ["demo", "edge", "synth"])
def test_unpack_bit_exact(ops, name, request):
    d = request.getfixturevalue(name)
    M = int(d["M"])
    G = dev_t(d["packed"])
    full = ops.unpack_u8(G, 0, M, M).cpu().numpy()
    assert np.array_equal(full, orc.unpack(d["packed"], M))
    # chunked with host-streamed slices (byte_offset), odd chunk sizes
    for start, count in ((0, 1), (3, 9), (5, 8192), (M - 3, 100)):
        bs = start // 4
        be = (min(M, start + count) + 3) // 4
        part = ops.unpack_u8(G[bs:be].contiguous(), start, count, M, bs).cpu().numpy()
        assert np.array_equal(part, orc.unpack(d["packed"], M, start, count))


def test_unpack_center(ops, demo):
    M = int(demo["M"])
    G = dev_t(demo["packed"])
    f = dev_t(demo["freq"])
    out = ops.unpack_center(G, f, 17, 999, M).cpu().numpy()
    g = orc.unpack(demo["packed"], M, 17, 999).astype(np.float32)
    exp = np.where(g == 3, np.float32(0), g - np.float32(2) * demo["freq"][17:17 + 999, None])
    np.testing.assert_array_equal(out, exp)


def test_allele_frequency(ops, demo, edge):
    for d in (demo, edge):
        M = int(d["M"])
        f = ops.allele_frequency(dev_t(d["packed"]), M).cpu().numpy()
        np.testing.assert_array_equal(f, orc.allele_frequency(orc.unpack(d["packed"], M)))
    np.testing.assert_allclose(ops.allele_frequency(dev_t(demo["packed"]), int(demo["M"])).cpu().numpy(),
                               demo["freq"], rtol=1e-6)


@pytest.mark.parametrize("name", ["demo", "edge", "synth"])
def test_sample_counts(ops, name, request):
    d = request.getfixturevalue(name)
    M = int(d["M"])
    q = ops.sample_counts(dev_t(d["packed"]), M).cpu().numpy()
    np.testing.assert_array_equal(q, d["q_bat"])


def test_bed_to_packed_matches_reference_reader(ops, demo):
    N, M = int(demo["N"]), int(demo["M"])
    G = ops.bed_to_packed(dev_t(demo["bed_rows"]), N, M).cpu().numpy()
    assert np.array_equal(G, demo["packed"])


def test_bed_flip_rule(ops):
    from adamixture_b200.src import packing

    rng = np.random.default_rng(5)
    for N, M in ((7, 13), (64, 33)):
        G = rng.choice([0, 1, 2, 3], size=(M, N), p=[0.05, 0.15, 0.7, 0.1]).astype(np.uint8)  # mean > .5
        nb = (N + 3) // 4
        codes = np.array([3, 2, 0, 1], dtype=np.uint8)[G]
        pad = np.zeros((M, nb * 4), np.uint8)
        pad[:, :N] = codes
        pad = pad.reshape(M, nb, 4)
        rows = pad[..., 0] | (pad[..., 1] << 2) | (pad[..., 2] << 4) | (pad[..., 3] << 6)
        exp = orc.bed_to_packed(rows, N)
        assert orc.packed_mean(exp, M) >= 0.5
        exp = orc.flip_packed(exp, M)
        got = ops.bed_to_packed(dev_t(rows), N, M).cpu().numpy()
        assert np.array_equal(got, exp)
        assert np.array_equal(packing.bed_rows_to_packed(rows, N), orc.bed_to_packed(rows, N))


def test_simulator_matches_host_sampler(ops, synth):
    Pq = dev_t(synth["Pq"].astype(np.int32))
    Qq = dev_t(synth["Qq"].astype(np.int32))
    keys = tuple(int(k) for k in synth["keys"])
    G = ops.simulate_packed(Pq, Qq, int(synth["miss_q"]), keys).cpu().numpy()
    assert np.array_equal(G, synth["packed"])


# ------------------------------------------------------------------ E-step

@pytest.mark.parametrize("name", ["demo", "edge", "synth"])
def test_em_stats_f64_matches_reference(ops, name, request):
    d = request.getfixturevalue(name)
    M = int(d["M"])
    A, B, T = ops.em_stats(dev_t(d["packed"]), dev_t(d["P0"]), dev_t(d["Q0"]), M, "f64")
    np.testing.assert_allclose(A.cpu().numpy(), d["A"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(B.cpu().numpy(), d["B"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(T.cpu().numpy(), d["T"], rtol=1e-10, atol=1e-9)
    q = ops.sample_counts(dev_t(d["packed"]), M)
    P_EM, Q_EM = ops.em_targets(dev_t(d["P0"]), dev_t(d["Q0"]), A, B, T, q)
    np.testing.assert_allclose(P_EM.cpu().numpy(), d["P_EM"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(Q_EM.cpu().numpy(), d["Q_EM"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", ["demo", "edge", "synth"])
def test_em_stats_f32_close_to_reference(ops, name, request):
    d = request.getfixturevalue(name)
    M = int(d["M"])
    A, B, T = ops.em_stats(dev_t(d["packed"]), dev_t(d["P0"], torch.float32),
                           dev_t(d["Q0"], torch.float32), M, "f32")
    for got, ref in ((A, d["A"]), (B, d["B"]), (T, d["T"])):
        got = got.cpu().numpy()
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 2e-5 * scale


@pytest.mark.parametrize("K", [1, 2, 3, 5, 7, 8, 10, 13, 16, 17, 33, 64])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_em_stats_random_shapes_vs_oracle(ops, K, prec):
    rng = np.random.default_rng(K)
    N, M = 1001 + K, 523 + 7 * K
    G = rng.integers(0, 4, size=(M, N)).astype(np.uint8)
    P = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q = rng.random((N, K))
    Q /= Q.sum(1, keepdims=True)
    A0, B0, T0, _ = orc.em_stats(G, P, Q)
    dt = torch.float64 if prec == "f64" else torch.float32
    A, B, T = ops.em_stats(dev_t(orc.pack(G)), dev_t(P, dt), dev_t(Q, dt), M, prec)
    tol = 1e-11 if prec == "f64" else 3e-5
    for got, ref in ((A, A0), (B, B0), (T, T0)):
        err = np.abs(got.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err <= tol, err


def test_em_stats_large_tile_counts(ops):
    # several sample sub-tiles and splits, a ragged last SNP block and sample tile
    rng = np.random.default_rng(1)
    N, M, K = 5 * 1024 + 3, 4 * 4096 + 5, 4
    coh_G = rng.integers(0, 4, size=(M, N)).astype(np.uint8)
    P = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.ones(K), size=N)
    A0, B0, T0, _ = orc.em_stats(coh_G, P, Q)
    A, B, T = ops.em_stats(dev_t(orc.pack(coh_G)), dev_t(P), dev_t(Q), M, "f64")
    np.testing.assert_allclose(A.cpu().numpy(), A0, rtol=1e-10)
    np.testing.assert_allclose(B.cpu().numpy(), B0, rtol=1e-10)
    np.testing.assert_allclose(T.cpu().numpy(), T0, rtol=1e-10)


def test_em_stats_f64_mma_tiles(ops):
    # the float64 tensor-core sweep (K <= 16) with 8-byte genotype loads (N a multiple of 8),
    # many sample sub-tiles per split, and SNP blocks that end inside a staged group
    rng = np.random.default_rng(2)
    for N, M, K in ((4096, 3001, 10), (2048 + 8, 517, 16), (1024, 129, 1)):
        G = rng.integers(0, 4, size=(M, N)).astype(np.uint8)
        P = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
        Q = rng.dirichlet(np.ones(K), size=N)
        A0, B0, T0, _ = orc.em_stats(G, P, Q)
        A, B, T = ops.em_stats(dev_t(orc.pack(G)), dev_t(P), dev_t(Q), M, "f64")
        for got, ref in ((A, A0), (B, B0), (T, T0)):
            err = np.abs(got.cpu().numpy() - ref).max() / np.abs(ref).max()
            assert err <= 1e-12, (N, M, K, err)


# ------------------------------------------------------------------ iterations

def _trace(d, precision, n):
    """Reference loop (priming + n iterations) through the fused CUDA iteration."""
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer

    M = int(d["M"])
    G = dev_t(d["packed"])
    P = dev_t(d["P0"]).clone()
    Q = dev_t(d["Q0"]).clone()
    P32, Q32 = P.float(), Q.float()
    opt = EMAdamOptimizer(P.shape, Q.shape, 0.005, 0.80, 0.88, 1e-8, G.device, precision)
    snaps = []
    for it in range(n + 1):
        opt.fused_iteration(G, P, Q, P32, Q32, M)
        snaps.append((P.cpu().numpy().copy(), Q.cpu().numpy().copy()))
    return snaps


@pytest.mark.parametrize("name", ["demo", "synth", "edge"])
def test_per_iteration_f64_within_1e5(ops, name, request):
    d = request.getfixturevalue(name)
    n = int(d["trace_iters"].max())
    snaps = _trace(d, "f64", n)
    for s, t in enumerate(d["trace_iters"]):
        assert np.abs(snaps[t][0] - d["trace_P"][s]).max() <= 1e-5
        assert np.abs(snaps[t][1] - d["trace_Q"][s]).max() <= 1e-5


def test_unfused_api_matches_fused(ops, synth):
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer

    M = int(synth["M"])
    G = dev_t(synth["packed"])
    P = dev_t(synth["P0"]).clone()
    Q = dev_t(synth["Q0"]).clone()
    opt = EMAdamOptimizer(P.shape, Q.shape, 0.005, 0.80, 0.88, 1e-8, G.device, "f64")
    for _ in range(3):
        P_EM, Q_EM = opt.run_em_step(G, P, Q, M, 8192)
        opt.step(P, Q, P_EM, Q_EM)
    fused = _trace(synth, "f64", 2)[-1]
    np.testing.assert_allclose(P.cpu().numpy(), fused[0], atol=1e-13)
    np.testing.assert_allclose(Q.cpu().numpy(), fused[1], atol=1e-13)


def test_per_iteration_f32_synth_within_1e5(ops, synth):
    n = int(synth["trace_iters"].max())
    snaps = _trace(synth, "f32", n)
    for s, t in enumerate(synth["trace_iters"]):
        assert np.abs(snaps[t][0] - synth["trace_P"][s]).max() <= 1e-5
        assert np.abs(snaps[t][1] - synth["trace_Q"][s]).max() <= 1e-5


def test_per_iteration_f32_demo(ops, demo):
    n = int(demo["trace_iters"].max())
    snaps = _trace(demo, "f32", n)
    for s, t in enumerate(demo["trace_iters"]):
        for k in (0, 1):
            err = np.abs(snaps[t][k] - (demo["trace_P"], demo["trace_Q"])[k][s])
            assert err.max() <= 2e-4
            assert np.quantile(err, 0.999) <= 1e-5


@pytest.mark.parametrize("name", ["demo", "synth", "edge"])
def test_loglik(ops, name, request):
    d = request.getfixturevalue(name)
    M = int(d["M"])
    G = dev_t(d["packed"])
    ref = float(d["loglik0"])
    l64 = float(ops.loglik_device(G, dev_t(d["P0"]), dev_t(d["Q0"]), M, "f64").item())
    l32 = float(ops.loglik_device(G, dev_t(d["P0"], torch.float32), dev_t(d["Q0"], torch.float32), M, "f32").item())
    assert abs(l64 - ref) <= 1e-12 * abs(ref)
    assert abs(l32 - ref) <= 1e-6 * abs(ref)


@pytest.mark.parametrize("N,M,K", [(1024, 777, 10), (1026, 501, 8), (4000, 333, 3), (2048, 130, 16),
                                   (512, 64, 24), (1000, 97, 64)])
def test_loglik_load_paths(ops, N, M, K):
    # N a multiple of the samples per thread: one word load per packed quad; otherwise, or
    # with G one byte off alignment, byte loads. Same sums either way, and against the oracle.
    rng = np.random.default_rng(N + M + K)
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    P = np.clip(rng.beta(0.8, 0.8, size=(M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    ref = orc.loglik(G, P, Q)
    Gp = orc.pack(G)
    Gd = dev_t(Gp)
    flat = torch.empty(Gp.size + 1, dtype=torch.uint8, device=Gd.device)
    flat[1:] = Gd.reshape(-1)
    Gmis = flat[1:].view(Gp.shape)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-6)):
        dt = torch.float64 if prec == "f64" else torch.float32
        Pd, Qd = dev_t(P, dt), dev_t(Q, dt)
        a = float(ops.loglik_device(Gd, Pd, Qd, M, prec).item())
        b = float(ops.loglik_device(Gmis, Pd, Qd, M, prec).item())
        assert a == b, (prec, a, b)
        assert abs(a - ref) <= tol * abs(ref), (prec, a, ref)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("name", ["demo", "synth"])
def test_converged_loglik_within_1e6(ops, name, prec, request):
    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu, optimize_parameters_gpu

    d = request.getfixturevalue(name)
    M, N, K = int(d["M"]), int(d["N"]), int(d["K"])
    G = dev_t(d["packed"])
    P, Q = optimize_parameters_gpu(G, dev_t(d["P0"]), dev_t(d["Q0"]), 0.005, 0.80, 0.88, 1e-8,
                                   10000, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 512,
                                   precision=prec)
    L = loglikelihood_gpu(G, P, Q, M, N, 8192, G.device, 512)
    ref = float(d["conv_loglik"])
    assert abs(L - ref) <= 1e-6 * abs(ref), (L, ref)
    Qn = Q.cpu().numpy()
    np.testing.assert_allclose(Qn.sum(1), 1.0, atol=1e-12)
    # the reference clamps to [1e-5, 1-1e-5] after the Adam move and then renormalises
    # rows whose sum an Adam move does not preserve, so entries can end a little under
    # 1e-5 (em_adam_gpu.py:222-224)
    assert Qn.min() > 0.5e-5 and P.min().item() >= 1e-5 - 1e-15


def test_cpu_tensors_rejected(ops, demo):
    from adamixture_b200.model.em_adam_gpu import loglikelihood_gpu

    with pytest.raises(ValueError, match="CUDA"):
        loglikelihood_gpu(torch.from_numpy(demo["packed"]), torch.zeros(3, 2), torch.zeros(3, 2),
                          3, 3, 8192, torch.device("cpu"), 1)


def test_reference_op_names(ops, demo):
    ops.register_reference_ops()
    M = int(demo["M"])
    G = dev_t(demo["packed"])
    out = torch.ops.pack2bit.unpack2bit_gpu_chunk_uint8(G, 100, 8192, M, 0, 512)
    assert np.array_equal(out.cpu().numpy(), orc.unpack(demo["packed"], M, 100, 8192))


@pytest.mark.parametrize("name", ["demo", "synth"])
def test_sweep_with_folded_check_equals_separate_check(ops, name, request):
    # the float64 sweep that also returns the log-likelihood of its input: the check equals
    # loglikelihood_gpu bit for bit, and its partial sums give the fused iteration's move
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer, loglikelihood_gpu

    d = request.getfixturevalue(name)
    M, N = int(d["M"]), int(d["N"])
    G = dev_t(d["packed"])
    runs = []
    for folded in (True, False):
        P, Q = dev_t(d["P0"]).clone(), dev_t(d["Q0"]).clone()
        opt = EMAdamOptimizer(P.shape, Q.shape, 0.005, 0.80, 0.88, 1e-8, G.device, "f64")
        ws = torch.zeros(ops.em_workspace_bytes(M, N, Q.shape[1], "f64"), dtype=torch.uint8, device=G.device)
        checks = []
        for it in range(7):
            if folded and it % 3 == 0:
                checks.append(float(opt.sweep_with_loglik(G, P, Q, M, ws).item()))
                opt.apply_update(P, Q, None, None, M, ws)
            else:
                if not folded and it % 3 == 0:
                    checks.append(loglikelihood_gpu(G, P, Q, M, N, 8192, G.device, 256))
                opt.fused_iteration(G, P, Q, None, None, M, ws)
        runs.append((P.cpu().numpy(), Q.cpu().numpy(), checks))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    assert runs[0][2] == runs[1][2], (runs[0][2], runs[1][2])


@pytest.mark.parametrize("name", ["demo", "synth"])
def test_optimiser_with_folded_checks_equals_the_reference_loop(ops, name, request):
    # the float64 optimiser folds each check into the next sweep; the returned model, the
    # check trace and the stop point equal those of the loop that checks after each move
    from adamixture_b200.model.em_adam_gpu import _optimize_parameters_gpu_once

    d = request.getfixturevalue(name)
    M, N, K = int(d["M"]), int(d["N"]), int(d["K"])
    G = dev_t(d["packed"])
    out = []
    for fold in (True, False):
        tr = []
        P, Q = _optimize_parameters_gpu_once(G, dev_t(d["P0"]).clone(), dev_t(d["Q0"]).clone(), 0.005, 0.80, 0.88,
                                             1e-8, 10000, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 512,
                                             precision="f64", trace=tr, fold_checks=fold)
        out.append((P.cpu().numpy(), Q.cpu().numpy(), [(it, L) for it, L, _ in tr]))
    assert out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def _ranges(nb):
    """An irregular cover of [0, nb) by consecutive block ranges."""
    cuts = sorted(c for c in {0, 1, nb // 3, 2 * nb // 3 + 1, nb} if c <= nb)
    return [(a, b) for a, b in zip(cuts, cuts[1:]) if a < b]


@pytest.mark.parametrize("N,M,K", [(105, 1000, 3), (2000, 9001, 7), (777, 40_003, 16), (3000, 5, 2)])
def test_block_range_sweeps_equal_the_full_sweep(ops, N, M, K):
    # the float64 sweep over ranges of its SNP blocks, each reading only its own packed rows:
    # the ranges of one workspace add up to the full sweep's workspace bit for bit
    rng = np.random.default_rng(N + M + K)
    g = rng.integers(0, 3, size=(M, N), dtype=np.uint8)
    g[rng.random((M, N)) < 0.02] = 3
    G = dev_t(orc.pack(g))
    P = dev_t(np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5))
    Q = rng.random((N, K))
    Q = dev_t(Q / Q.sum(1, keepdims=True))
    spb, nb, cpb = ops.em_sweep_blocks_info(M, N, K)
    assert spb % 16 == 0 and nb == -(-M // spb) and cpb * nb <= 1776
    nbytes = ops.em_workspace_bytes(M, N, K, "f64")
    full = torch.zeros(nbytes, dtype=torch.uint8, device=G.device)
    ops.em_sweep(G, P, Q, M, "f64", full)
    parts = torch.zeros_like(full)
    Gp = torch.full_like(G, 0xFF)        # rows outside the swept ranges hold junk (all missing)
    for b0, b1 in reversed(_ranges(nb)):
        r0, r1 = b0 * spb // 4, min(G.shape[0], b1 * spb // 4)
        Gp[r0:r1] = G[r0:r1]
        ops.em_sweep_blocks(Gp, P, Q, M, b0, b1, parts)
    assert torch.equal(full, parts)
    with pytest.raises(Exception, match="b0 < b1"):
        ops.em_sweep_blocks(G, P, Q, M, 0, nb + 1, parts)


@pytest.mark.parametrize("name", ["demo", "synth"])
def test_optimiser_from_host_matrix_equals_resident(ops, name, request, monkeypatch):
    # a packed matrix in pinned host memory is uploaded in pieces that the priming sweep
    # consumes as they land; the fit equals the one from the device-resident matrix exactly
    from adamixture_b200.model import em_adam_gpu as em

    d = request.getfixturevalue(name)
    M, N, K = int(d["M"]), int(d["N"]), int(d["K"])
    monkeypatch.setattr(em, "upload_pieces", lambda nb, cpb, sms: _ranges(nb))   # several pieces
    out = []
    for host in (True, False):
        G = torch.from_numpy(d["packed"]).pin_memory() if host else dev_t(d["packed"])
        P0 = torch.from_numpy(d["P0"]) if host else dev_t(d["P0"])
        Q0 = torch.from_numpy(d["Q0"]) if host else dev_t(d["Q0"])
        tr = []
        P, Q = em.optimize_parameters_gpu(G, P0, Q0, 0.005, 0.80, 0.88, 1e-8, 60, 5, K, M, N, 0.5, 1e-4, 3, 0.1,
                                          torch.device("cuda", 0), 8192, 512, precision="f64", trace=tr)
        out.append((P.cpu().numpy(), Q.cpu().numpy(), [(it, L) for it, L, _ in tr]))
    assert out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "bf16"])
def test_graph_replay_equals_eager_iterations(ops, synth, prec):
    # fused iterations captured once into a CUDA graph (adx_em_graph_create) and replayed at
    # steps t0+1..t0+n: P, Q and the Adam moments equal the eager iterations bit for bit
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer

    d = synth
    M, N = int(d["M"]), int(d["N"])
    G = dev_t(d["packed"])
    runs = []
    for graphed in (False, True):
        P, Q = dev_t(d["P0"]).clone(), dev_t(d["Q0"]).clone()
        P32, Q32 = (P.float(), Q.float()) if prec != "f64" else (None, None)
        opt = EMAdamOptimizer(P.shape, Q.shape, 0.005, 0.80, 0.88, 1e-8, G.device, prec)
        ws = ops.em_workspace(M, N, Q.shape[1], prec, G.device)
        opt.fused_iteration(G, P, Q, P32, Q32, M, ws)            # step 1, eager in both runs
        if graphed:
            g = ops.EmGraph(G, P, Q, P32, Q32, opt.m_P, opt.v_P, opt.m_Q, opt.v_Q, opt.q_bat, M, 4, opt.lr,
                            opt.beta1, opt.beta2, opt.reg_adam, prec, ws)
            g.launch(1)                                            # steps 2..5
            g.launch(5)                                            # steps 6..9
            opt._t = 9
            g.close()
            with pytest.raises(RuntimeError):
                g.launch(9)
        else:
            for _ in range(8):
                opt.fused_iteration(G, P, Q, P32, Q32, M, ws)
        opt.fused_iteration(G, P, Q, P32, Q32, M, ws)            # step 10
        runs.append([x.cpu().numpy() for x in (P, Q, opt.m_P, opt.v_P, opt.m_Q, opt.v_Q)])
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name,prec", [("demo", "f64"), ("synth", "f64"), ("synth", "f32"), ("synth", "mixed")])
def test_optimiser_with_graphs_equals_eager(ops, name, prec, request, monkeypatch):
    # the optimiser replays the iterations between checks from captured graphs; the fit, the
    # check trace and the stop point equal those of the eager loop
    from adamixture_b200.model import em_adam_gpu as em

    d = request.getfixturevalue(name)
    M, N, K = int(d["M"]), int(d["N"]), int(d["K"])
    G = dev_t(d["packed"])
    out = []
    for graphs in (False, True):
        monkeypatch.setattr(em, "USE_GRAPHS", graphs)
        tr = []
        P, Q = em._optimize_parameters_gpu_once(G, dev_t(d["P0"]).clone(), dev_t(d["Q0"]).clone(), 0.005, 0.80,
                                                0.88, 1e-8, 10000, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192,
                                                512, precision=prec, trace=tr)
        out.append((P.cpu().numpy(), Q.cpu().numpy(), [(it, L) for it, L, _ in tr]))
    assert out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_graph_rejects_bad_arguments(ops, synth):
    M, N = int(synth["M"]), int(synth["N"])
    G = dev_t(synth["packed"])
    P, Q = dev_t(synth["P0"]).clone(), dev_t(synth["Q0"]).clone()
    z = [torch.zeros_like(x) for x in (P, P, Q, Q)]
    q = torch.ones(N, dtype=torch.float64, device=G.device)
    ws = ops.em_workspace(M, N, Q.shape[1], "f64", G.device)
    with pytest.raises(Exception, match="n_iters"):
        ops.EmGraph(G, P, Q, None, None, *z, q, M, 0, 0.005, 0.8, 0.88, 1e-8, "f64", ws)
    with pytest.raises(ValueError, match="workspace"):
        ops.EmGraph(G, P, Q, None, None, *z, q, M, 3, 0.005, 0.8, 0.88, 1e-8, "f64", ws[:100])


@pytest.mark.parametrize("N,M,K", [(1, 1, 1), (1, 37, 5), (7, 1, 16), (9, 3, 10), (8, 16, 4), (255, 17, 12)])
def test_degenerate_shapes_vs_oracle(ops, N, M, K):
    # one sample, one SNP, fewer samples than a warp's 32 or a sub-tile's 256, a single
    # packed row: statistics (both float64 forms' shapes route to the float64 MMA sweep for
    # K <= 16) and the float64 log-likelihood against the oracle
    rng = np.random.default_rng(N * 1000 + M * 10 + K)
    G = rng.integers(0, 4, size=(M, N)).astype(np.uint8)
    P = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q = rng.random((N, K))
    Q /= Q.sum(1, keepdims=True)
    A0, B0, T0, _ = orc.em_stats(G, P, Q)
    Gd = dev_t(orc.pack(G))
    A, B, T = ops.em_stats(Gd, dev_t(P), dev_t(Q), M, "f64")
    for got, ref in ((A, A0), (B, B0), (T, T0)):
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got.cpu().numpy() - ref).max() <= 1e-12 * scale
    L0 = orc.loglik(G, P, Q)
    L = float(ops.loglik_device(Gd, dev_t(P), dev_t(Q), M, "f64").item())
    assert abs(L - L0) <= 1e-12 * max(abs(L0), 1.0), (L, L0)


def test_all_missing_matrix(ops):
    # every entry missing: zero statistics and log-likelihood, and an Adam-EM iteration
    # leaves P and Q finite and inside their bounds
    from adamixture_b200.model.em_adam_gpu import EMAdamOptimizer

    N, M, K = 300, 70, 6
    G = dev_t(orc.pack(np.full((M, N), 3, dtype=np.uint8)))
    rng = np.random.default_rng(3)
    P = dev_t(np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5))
    Q = rng.random((N, K))
    Q = dev_t(Q / Q.sum(1, keepdims=True))
    A, B, T = ops.em_stats(G, P, Q, M, "f64")
    assert float(A.abs().max()) == 0.0 and float(B.abs().max()) == 0.0 and float(T.abs().max()) == 0.0
    assert float(ops.loglik_device(G, P, Q, M, "f64").item()) == 0.0
    opt = EMAdamOptimizer(P.shape, Q.shape, 0.005, 0.80, 0.88, 1e-8, G.device, "f64")
    for _ in range(3):
        opt.fused_iteration(G, P, Q, None, None, M)
    for x in (P, Q):
        assert bool(torch.isfinite(x).all()) and float(x.min()) >= 0.0 and float(x.max()) <= 1.0


def test_optimiser_without_graph_capture_runs_eagerly(ops, synth, monkeypatch):
    # a capture the library reports as failed (here a stand-in that raises the library's
    # error) leaves the optimiser on one-by-one launches of the same iterations
    from adamixture_b200 import _lib
    from adamixture_b200.model import em_adam_gpu as em

    def refuse(*args, **kw):
        raise _lib.AdxError("adx_em_graph_create: CUDA error: capture refused")

    M, N, K = int(synth["M"]), int(synth["N"]), int(synth["K"])
    G = dev_t(synth["packed"])
    out = []
    for patch in (False, True):
        if patch:
            monkeypatch.setattr(ops, "EmGraph", refuse)
        P, Q = em._optimize_parameters_gpu_once(G, dev_t(synth["P0"]).clone(), dev_t(synth["Q0"]).clone(), 0.005,
                                                0.80, 0.88, 1e-8, 40, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192,
                                                512, precision="f32")
        out.append((P.cpu().numpy(), Q.cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
