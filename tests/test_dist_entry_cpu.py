"""The multi-GPU command's host logic (adamixture_b200.dist_entry) on CPU ranks.

* The sharded BED read: for 1-4 ranks, with and without the flip and with a chromosome
  filter, the ranks' packed rows concatenate to exactly the single reader's matrix
  (``read_bed_packed``), so the flip decision is the global one.
* A whole run (sharded init, then Adam-EM or SQP + ZAL QN, outputs gathered on rank 0) with
  two gloo ranks on float64 backends that restate the kernels (the oracle's) against the
  same run with one rank: P and Q within 1e-9, and rank 0 writes the reference's .Q/.P files.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import em_oracle as orc


def _cohort(N, M, K, seed, high=False, split=False):
    rng = np.random.default_rng(seed)
    P = 0.3 * rng.beta(0.6, 0.6, size=(M, K))
    if high:
        P = 1.0 - P                # mostly the second allele: the reader flips
    if split:
        # low frequencies in the first half, very high in the second: the file's mean is above
        # 1/2 (it flips) while the first half's alone is below (it would not)
        P[: M // 2] = 0.3 * rng.beta(0.6, 0.6, size=(M // 2, K))
        P[M // 2:] = 1.0 - 0.05 * rng.beta(0.6, 0.6, size=(M - M // 2, K))
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    G = rng.binomial(2, np.clip(P @ Q.T, 0, 1)).astype(np.uint8)
    G[rng.random(G.shape) < 0.02] = 3
    return G


@pytest.mark.parametrize("high", [False, True])
@pytest.mark.parametrize("chrom", [None, ["3", "7", "12"]])
def test_shards_concatenate_to_the_single_reader(tmp_path, high, chrom):
    from adamixture_b200.dist_entry import read_bed_shard
    from adamixture_b200.src.packing import read_bed_packed
    from adamixture_b200.src.simulate import write_bed

    G = _cohort(37, 203, 3, 5, high)
    write_bed(tmp_path / "c", G)
    whole, N, M = read_bed_packed(tmp_path / "c.bed", specific_chrom=chrom)
    whole = whole.numpy()
    for world in (1, 2, 3, 4):
        parts = [read_bed_shard(tmp_path / "c.bed", r, world, specific_chrom=chrom) for r in range(world)]
        assert all(p[1] == N and p[2] == M for p in parts)
        # no process group here: each shard decides the flip on its own mean, which agrees with
        # the file's for these cohorts (mean dosage / 2 near 0.15 or 0.85); the two-rank test
        # below covers the global decision
        assert abs(orc.packed_mean(whole, M) - 0.5) > 0.2
        np.testing.assert_array_equal(np.concatenate([p[0] for p in parts]), whole)
        assert parts[0][3] == 0 and parts[-1][4] == M


class _OracleShard:
    def __init__(self):
        from tests.test_dist_brqn_cpu import OracleBrqnBackend
        from tests.test_dist_cpu import OracleBackend
        from tests.test_dist_init_cpu import NumpyInitBackend

        self.init, self.em, self.brqn = NumpyInitBackend(), OracleBackend(), OracleBrqnBackend()

    def prepare(self, Gp, M_local):
        return orc.unpack(Gp, M_local)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, prefix, out, algorithm):
    import torch.distributed as dist

    from adamixture_b200.dist_entry import parse_args, read_bed_shard, run

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # under the process group the flip follows the whole file's mean
        Gp, N, M, j0, j1 = read_bed_shard(prefix + ".bed", rank, world)
        np.save(os.path.join(out, f"shard{rank}.npy"), Gp)
        args = parse_args(["--k", "3", "--data_path", prefix + ".bed", "--save_dir", out, "--name", "run",
                           "--algorithm", algorithm, "--max_iter", "10" if algorithm == "adamem" else "3",
                           "--max_als", "20", "--power", "4"])
        res = run(args, backends=_OracleShard())
        if rank == 0:
            np.savez(os.path.join(out, "res.npz"), P=res[0], Q=res[1])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("algorithm", ["adamem", "brqn"])
def test_two_rank_run_matches_one_rank(tmp_path, algorithm):
    from adamixture_b200.src.packing import read_bed_packed
    from adamixture_b200.src.simulate import write_bed

    G = _cohort(48, 301, 3, 9, split=True)
    prefix = str(tmp_path / "c")
    write_bed(prefix, G)
    from adamixture_b200.src.packing import pack
    half = pack(G[:150])
    assert orc.packed_mean(half, 150) < 0.5 < orc.packed_mean(pack(G), 301)
    outs = {}
    for world in (1, 2):
        out = tmp_path / f"w{world}"
        out.mkdir()
        mp.start_processes(_rank, args=(world, _free_port(), prefix, str(out), algorithm), nprocs=world,
                           join=True, start_method="spawn")
        outs[world] = out
    whole, N, M = read_bed_packed(prefix + ".bed")
    cat = np.concatenate([np.load(outs[2] / f"shard{r}.npy") for r in range(2)])
    np.testing.assert_array_equal(cat, whole.numpy())   # rank 0's half flipped with the file, not alone
    r1, r2 = np.load(outs[1] / "res.npz"), np.load(outs[2] / "res.npz")
    assert r1["P"].shape == (M, 3) and r1["Q"].shape == (N, 3)
    np.testing.assert_allclose(r2["P"], r1["P"], atol=1e-9)
    np.testing.assert_allclose(r2["Q"], r1["Q"], atol=1e-9)
    Qf = np.loadtxt(outs[2] / "run.3.Q")
    Pf = np.loadtxt(outs[2] / "run.3.P")
    np.testing.assert_allclose(Qf, r2["Q"], rtol=1e-15)
    np.testing.assert_allclose(Pf, r2["P"], rtol=1e-15)


@pytest.mark.parametrize("bad", [["--k", "0"], ["--k", "65"], ["--k", "3", "--device", "cpu"],
                                 ["--k", "3", "--lr", "-1"]])
def test_bad_options_are_rejected(bad):
    from adamixture_b200.dist_entry import parse_args

    with pytest.raises(SystemExit):
        parse_args(bad + ["--data_path", "x.bed", "--save_dir", "o", "--name", "r"])
