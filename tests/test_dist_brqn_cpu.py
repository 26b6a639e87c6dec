"""The SNP-sharded SQP + ZAL QN (adamixture_b200.model.br_qn_dist) with two gloo ranks on the
CPU against the same code in one process, on a float64 backend that restates the passes
and solves (the oracle's gradient/Hessian sums, per-row SQP and log-likelihood).

Bars: after 4 iterations the gathered P rows and the replicated Q equal the one-process
run's within 1e-9 (the all-reduced Hessians and secant products differ from one sum only
in float64 rounding), the Q replicas are identical across the ranks, and the one-process
run raises the log-likelihood of its start.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import em_oracle as orc
from oracle import solvers as sol

N, M, K, ITERS = 60, 401, 4, 4


class OracleBrqnBackend:
    def grad_hess_q(self, G, P, Q, M_local):
        XtX, Xtz = sol.grad_hess_q(G, P.numpy(), Q.numpy())
        return torch.from_numpy(np.ascontiguousarray(XtX)), torch.from_numpy(np.ascontiguousarray(Xtz))

    def grad_hess_p(self, G, P, Q, M_local):
        XtX, Xtz = sol.grad_hess_p(G, P.numpy(), Q.numpy())
        return torch.from_numpy(np.ascontiguousarray(XtX)), torch.from_numpy(np.ascontiguousarray(Xtz))

    def sqp_q(self, XtX, Xtz_neg, Q, v_kk):
        return torch.from_numpy(sol.sqp_solve_q(XtX.numpy(), Xtz_neg.numpy(), Q.numpy(), v_kk.numpy()))

    def sqp_p(self, XtX, Xtz_neg, P):
        return torch.from_numpy(sol.sqp_solve_p(XtX.numpy(), Xtz_neg.numpy(), P.numpy()))

    def loglik(self, G, P, Q, M_local):
        return torch.tensor([orc.loglik(G, P.numpy(), Q.numpy())], dtype=torch.float64)


def _cohort():
    rng = np.random.default_rng(11)
    Pt = rng.beta(0.5, 0.5, size=(M, K))
    Qt = rng.dirichlet(np.full(K, 0.4), size=N)
    G = rng.binomial(2, np.clip(Pt @ Qt.T, 0, 1)).astype(np.uint8)
    G[rng.random(G.shape) < 0.02] = 3
    P0 = np.clip(rng.random((M, K)), 1e-5, 1 - 1e-5)
    Q0 = np.clip(rng.random((N, K)), 1e-5, 1 - 1e-5)
    Q0 /= Q0.sum(1, keepdims=True)
    return G, P0, Q0


def _run(G, P0, Q0, j0, j1):
    from adamixture_b200.model.br_qn_dist import optimize_original_dist

    P = torch.from_numpy(P0[j0:j1].copy())
    Q = torch.from_numpy(Q0.copy())
    return optimize_original_dist(np.ascontiguousarray(G[j0:j1]), P, Q, ITERS, K, j1 - j0, N, 0.0, 3, ITERS + 1,
                                  backend=OracleBrqnBackend(), verbose=False)


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
        G, P0, Q0 = _cohort()
        j0, j1 = shard_rows(M, world, rank)
        P, Q = _run(G, P0, Q0, j0, j1)
        np.savez(os.path.join(out, f"r{rank}.npz"), P=P.numpy(), Q=Q.numpy(), j0=j0, j1=j1)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def one_process():
    G, P0, Q0 = _cohort()
    P, Q = _run(G, P0, Q0, 0, M)
    return G, P0, Q0, P.numpy(), Q.numpy()


def test_one_process_run_raises_the_log_likelihood(one_process):
    G, P0, Q0, P1, Q1 = one_process
    assert orc.loglik(G, P1, Q1) > orc.loglik(G, P0, Q0)
    np.testing.assert_allclose(Q1.sum(1), 1.0, atol=1e-12)
    assert np.all(P1 >= 1e-5) and np.all(P1 <= 1 - 1e-5)


def test_two_rank_sharded_brqn_matches_one_process(tmp_path, one_process):
    G, P0, Q0, P1, Q1 = one_process
    mp.start_processes(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(2)]
    P = np.concatenate([p["P"] for p in parts])
    np.testing.assert_allclose(P, P1, atol=1e-9)
    for p in parts:
        np.testing.assert_allclose(p["Q"], Q1, atol=1e-9)
    np.testing.assert_array_equal(parts[0]["Q"], parts[1]["Q"])   # replicas identical
