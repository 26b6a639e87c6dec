"""The SNP-sharded initialisation (randomized SVD + ALS, adamixture_b200.model.init_dist)
with two gloo ranks on the CPU against the same code in one process, on a float64 backend
that restates the passes over the genotypes (the oracle's centred products and BVLS).

Bars: the gathered P rows and the replicated Q equal the one-process run's within 1e-9
(the all-reduced sums differ from one sum only in float64 rounding), the replicas of Q are
identical across the ranks, and the singular values are those of the centred matrix
(np.linalg.svd) within 1e-2 relative (a randomized SVD of a cohort with a flat spectrum).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import em_oracle as orc
from oracle import solvers as sol

K, SEED, POWER, TOL_SVD, MAX_ALS, TOL_ALS = 6, 42, 6, 1e-4, 20, 1e-4


class NumpyInitBackend:
    dtype = torch.float64

    def rsvd_cols(self, G, f, B, M_local):
        return torch.from_numpy(sol.rsvd_cols(G, f.numpy(), B.numpy()))

    def rsvd_rows(self, G, f, Y, M_local):
        return torch.from_numpy(sol.rsvd_rows(G, f.numpy(), Y.numpy()))

    def bvls(self, A, B, lower, upper):
        return torch.from_numpy(sol.bvls_bpp(A.numpy(), B.numpy(), lower, upper))

    def frequencies(self, G, M_local):
        return torch.from_numpy(orc.allele_frequency(G).astype(np.float64))


def _cohort():
    from tests.conftest import GOLDEN

    with np.load(GOLDEN / "synth.npz") as z:
        M = int(z["M"])
        return orc.unpack(z["packed"], M), M


def _run(G, M, j0, j1):
    from adamixture_b200.model.init_dist import initialize_sharded

    N = G.shape[1]
    return initialize_sharded(np.ascontiguousarray(G[j0:j1]), N, M, j0, j1, K, SEED, POWER, TOL_SVD, MAX_ALS,
                              TOL_ALS, backend=NumpyInitBackend())


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    from adamixture_b200.model.em_adam_dist import shard_rows

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        G, M = _cohort()
        j0, j1 = shard_rows(M, world, rank)
        P, Q = _run(G, M, j0, j1)
        np.savez(os.path.join(out, f"r{rank}.npz"), P=P.numpy(), Q=Q.numpy(), j0=j0, j1=j1)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def one_process():
    G, M = _cohort()
    P, Q = _run(G, M, 0, M)
    return G, M, P.numpy(), Q.numpy()


def test_one_process_svd_matches_the_exact_singular_values(one_process):
    from adamixture_b200.model.init_dist import svd_sharded

    G, M, _, _ = one_process
    f = NumpyInitBackend().frequencies(G, M)
    U, S, V = svd_sharded(G, G.shape[1], M, 0, M, f, K, SEED, POWER, TOL_SVD, NumpyInitBackend())
    exact = np.linalg.svd(sol.centred(G, f.numpy()), compute_uv=False)[:K]
    np.testing.assert_allclose(S.numpy(), exact, rtol=1e-2)
    # U and V orthonormal
    np.testing.assert_allclose(U.numpy().T @ U.numpy(), np.eye(K), atol=1e-9)
    np.testing.assert_allclose(V.numpy().T @ V.numpy(), np.eye(K), atol=1e-6)


def test_two_rank_sharded_initialisation_matches_one_process(tmp_path, one_process):
    G, M, P1, Q1 = one_process
    mp.start_processes(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(2)]
    assert int(parts[0]["j0"]) == 0 and int(parts[1]["j1"]) == M
    P = np.concatenate([p["P"] for p in parts])
    np.testing.assert_allclose(P, P1, atol=1e-9)
    for p in parts:
        np.testing.assert_allclose(p["Q"], Q1, atol=1e-9)
    np.testing.assert_array_equal(parts[0]["Q"], parts[1]["Q"])   # replicas identical
    assert np.all(P >= 0.0) and np.all(P <= 1.0)
    np.testing.assert_allclose(parts[0]["Q"].sum(1), 1.0, atol=1e-12)
