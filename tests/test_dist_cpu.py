"""The SNP-sharded Adam-EM host logic with two gloo ranks on the CPU: each rank runs
optimize_parameters_dist on its rows of the synthetic cohort with a float64 numpy
statistics backend (the oracle's E-step, targets and Adam), exchanging T, the sample counts
and the log-likelihood through torch.distributed; the gathered P rows and the replicated Q
match the single-process oracle run (the shards' T sums differ from the full sum only in
float64 rounding)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import em_oracle as orc


class OracleBackend:
    def counts(self, G, M):
        return torch.from_numpy(orc.sample_counts(G))

    def stats(self, G, P, Q, M, K):
        A, B, T, _ = orc.em_stats(G, P.numpy(), Q.numpy())
        return torch.from_numpy(A), torch.from_numpy(B), torch.from_numpy(T)

    def targets(self, P, Q, A, B, T, q_bat):
        Pe, Qe = orc.em_final(P.numpy(), Q.numpy(), A.numpy(), B.numpy(), T.numpy(), q_bat.numpy())
        return torch.from_numpy(Pe), torch.from_numpy(Qe)

    def adam(self, P, Q, P_EM, Q_EM, st, t, lr, b1, b2, eps):
        Pn, Qn = P.numpy(), Q.numpy()
        orc.adam_update(Pn, P_EM.numpy(), st["mP"].numpy(), st["vP"].numpy(), float(t), lr, b1, b2, eps)
        orc.adam_update(Qn, Q_EM.numpy(), st["mQ"].numpy(), st["vQ"].numpy(), float(t), lr, b1, b2, eps)
        np.clip(Pn, 1e-5, 1 - 1e-5, out=Pn)
        np.clip(Qn, 1e-5, 1 - 1e-5, out=Qn)
        Qn /= Qn.sum(1, keepdims=True)

    def loglik(self, G, P, Q, M):
        return torch.tensor([orc.loglik(G, P.numpy(), Q.numpy())], dtype=torch.float64)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, path, out):
    import torch.distributed as dist

    from adamixture_b200.model.em_adam_dist import optimize_parameters_dist, shard_rows

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        with np.load(path) as z:
            M = int(z["M"])
            G = orc.unpack(z["packed"], M)
            P0, Q0 = z["P0"], z["Q0"]
        j0, j1 = shard_rows(M, world, rank)
        P = torch.from_numpy(P0[j0:j1].copy())
        Q = torch.from_numpy(Q0.copy())
        trace = []
        Pb, Qb = optimize_parameters_dist(np.ascontiguousarray(G[j0:j1]), P, Q, 0.005, 0.80, 0.88, 1e-8, 20, 5,
                                          Q.shape[1], j1 - j0, Q.shape[0], 0.5, 1e-4, 3, 0.1,
                                          backend=OracleBackend(), trace=trace)
        np.savez(os.path.join(out, f"r{rank}.npz"), P=Pb.numpy(), Q=Qb.numpy(), j0=j0, j1=j1,
                 trace=np.array([t[1] for t in trace]))
    finally:
        dist.destroy_process_group()


def test_shard_rows_cover_whole_packed_rows():
    from adamixture_b200.model.em_adam_dist import shard_rows

    for M in (1, 3, 4, 5, 2003, 8451):
        for world in (1, 2, 3, 8):
            parts = [shard_rows(M, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == M
            for (a, b), (c, d) in zip(parts, parts[1:]):
                assert b == c and a % 4 == 0
            assert all(a <= b for a, b in parts)


def test_two_rank_sharded_adam_em_matches_single_process(tmp_path):
    from tests.conftest import GOLDEN

    path = str(GOLDEN / "synth.npz")
    mp.start_processes(_rank, args=(2, _free_port(), path, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    with np.load(path) as z:
        M = int(z["M"])
        G = orc.unpack(z["packed"], M)
        P0, Q0 = z["P0"], z["Q0"]
    Pr, Qr, Lr, tr = orc.optimize(G, P0, Q0, max_iter=20)
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(2)]
    P = np.concatenate([p["P"] for p in parts])
    np.testing.assert_allclose(P, Pr, atol=1e-9)
    for p in parts:
        np.testing.assert_allclose(p["Q"], Qr, atol=1e-9)
        np.testing.assert_allclose(p["trace"], [L for _, L in tr.loglik], rtol=1e-12)
    np.testing.assert_array_equal(parts[0]["Q"], parts[1]["Q"])  # replicas identical
