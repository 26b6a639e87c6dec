"""GPU parity of the initialisation and original-ADMIXTURE kernels:

* randomized-SVD products (float32) against the float64 oracle, relative 1e-4;
* BVLS, gradient/Hessian and SQP (float64) against the reference's CPU kernels' outputs
  (tests/golden/solvers.npz), 1e-9;
* the demo pipeline (K=7, seed 42) against the reference's GPU golden files: randomized SVD
  and ALS within the reference's own tolerance (rtol = atol = 2e-2, U/V columns sign-
  canonicalised), converged BR-QN and Adam-EM models after cluster alignment within 2e-2,
  and their log-likelihoods within 50 of the golden models' (tests/test_cuda.py:149-177
  in the reference).
"""
import numpy as np
import pytest
import torch

from oracle import em_oracle as orc
from oracle import solvers as osv

pytestmark = pytest.mark.gpu

RTOL = ATOL = 2e-2
LOGL_ATOL = 50.0


def dev(x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t if dtype is None else t.to(dtype)


@pytest.fixture(scope="module")
def ops(cuda):
    from adamixture_b200 import ops as _ops

    return _ops


@pytest.mark.parametrize("N,M,L", [(23, 37, 5), (300, 1001, 20), (1000, 257, 17), (129, 4099, 80),
                                   (2000, 3001, 32), (700, 1500, 33), (64, 5000, 12)])
def test_rsvd_products(ops, N, M, L):
    rng = np.random.default_rng(N + M + L)
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    f = rng.uniform(0.05, 0.95, M).astype(np.float32)
    B = rng.normal(size=(N, L)).astype(np.float32)
    Y0 = osv.rsvd_rows(G, f, B)
    Gd, fd = dev(orc.pack(G)), dev(f)
    Y = ops.rsvd_rows(Gd, fd, dev(B), M).cpu().numpy()
    np.testing.assert_allclose(Y, Y0, rtol=1e-4, atol=1e-4 * np.abs(Y0).max())
    Z0 = osv.rsvd_cols(G, f, Y0)
    Z = ops.rsvd_cols(Gd, fd, dev(Y0.astype(np.float32)), M).cpu().numpy()
    np.testing.assert_allclose(Z, Z0, rtol=1e-4, atol=1e-4 * np.abs(Z0).max())
    Z2 = ops.rsvd_cols(Gd, fd, dev(Y0.astype(np.float32)), M, out=torch.from_numpy(Z).cuda(),
                       accumulate=True).cpu().numpy()
    np.testing.assert_allclose(Z2, 2 * Z0, rtol=1e-4, atol=2e-4 * np.abs(Z0).max())


@pytest.mark.parametrize("K", (1, 3, 7, 12, 20, 40, 64))
def test_bvls_vs_reference(ops, solvers_golden, K):
    d = solvers_golden
    X = ops.bvls(dev(d[f"bvls{K}_A"]), dev(d[f"bvls{K}_B"]), 0.0, 1.0).cpu().numpy()
    np.testing.assert_allclose(X, d[f"bvls{K}_X"], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_grad_hess_vs_reference(ops, solvers_golden, tag):
    d = solvers_golden
    M = d[f"{tag}_G"].shape[0]
    Gp, P, Q = dev(d[f"{tag}_packed"]), dev(d[f"{tag}_P"]), dev(d[f"{tag}_Q"])
    XtX_q, Xtz_q = ops.grad_hess_q(Gp, P, Q, M)
    XtX_p, Xtz_p = ops.grad_hess_p(Gp, P, Q, M)
    for got, nm in ((XtX_q, "XtX_q"), (Xtz_q, "Xtz_q"), (XtX_p, "XtX_p"), (Xtz_p, "Xtz_p")):
        ref = d[f"{tag}_{nm}"]
        np.testing.assert_allclose(got.cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


@pytest.mark.parametrize("K", [7, 8, 10, 16, 20, 64])
def test_grad_hess_every_k_bound(ops, K):
    # every compile-time bound of K (exact 10, 8 and 16, 64 for the rest) against the float64
    # restatement; several row tiles, reduced-axis chunks and, for K = 64, pair blocks
    rng = np.random.default_rng(K)
    M, N = 333, 150
    G = rng.choice(4, size=(M, N), p=[0.3, 0.35, 0.3, 0.05]).astype(np.uint8)
    P = np.clip(rng.beta(0.8, 0.8, size=(M, K)), 1e-5, 1 - 1e-5)
    Q = rng.dirichlet(np.full(K, 0.5), size=N)
    Gp = dev(orc.pack(G))
    out = {"q": ops.grad_hess_q(Gp, dev(P), dev(Q), M), "p": ops.grad_hess_p(Gp, dev(P), dev(Q), M)}
    ref = {"q": osv.grad_hess_q(G, P, Q), "p": osv.grad_hess_p(G, P, Q)}
    for side in ("q", "p"):
        for got, want in zip(out[side], ref[side]):
            np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-9, atol=1e-9 * np.abs(want).max())


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_sqp_vs_reference(ops, solvers_golden, tag):
    d = solvers_golden
    N, K = d[f"{tag}_Q"].shape
    M = d[f"{tag}_P"].shape[0]
    Qn = ops.sqp_solve_q(dev(d[f"{tag}_XtX_q"]), dev(-d[f"{tag}_Xtz_q"]), dev(d[f"{tag}_Q"]),
                         dev(d[f"{tag}_v_kk"]), N, K).cpu().numpy()
    Pn = ops.sqp_solve_p(dev(d[f"{tag}_XtX_p"]), dev(-d[f"{tag}_Xtz_p"]), dev(d[f"{tag}_P"]), M, K).cpu().numpy()
    np.testing.assert_allclose(Qn, d[f"{tag}_Q_next"], atol=1e-9)
    np.testing.assert_allclose(Pn, d[f"{tag}_P_next"], atol=1e-9)


def test_reference_op_names_resolve(ops, solvers_golden):
    ops.register_reference_ops()
    d = solvers_golden
    X = torch.ops.bvls_kernel.batch_bvls_bpp_cuda(dev(d["bvls7_A"]), dev(d["bvls7_B"]), 0.0, 1.0)
    np.testing.assert_allclose(X.cpu().numpy(), d["bvls7_X"], rtol=1e-9, atol=1e-9)
    N, K = d["a_Q"].shape
    Qn = torch.ops.sqp_kernel.sqp_solve_q_cuda(dev(d["a_XtX_q"]), dev(-d["a_Xtz_q"]), dev(d["a_Q"]),
                                                dev(d["a_v_kk"]), N, K)
    np.testing.assert_allclose(Qn.cpu().numpy(), d["a_Q_next"], atol=1e-9)


# ---------------------------------------------------------------- demo pipeline

def canonical(U, V):
    U, V = U.copy(), V.copy()
    for c in range(U.shape[1]):
        p = int(np.argmax(np.abs(U[:, c])))
        if U[p, c] < 0:
            U[:, c] *= -1
            V[:, c] *= -1
    return U, V


def align(Q_ref, P, Q):
    from scipy.optimize import linear_sum_assignment

    cost = -np.abs(np.corrcoef(Q_ref.T, Q.T)[: Q_ref.shape[1], Q_ref.shape[1]:])
    _, perm = linear_sum_assignment(cost)
    return P[:, perm], Q[:, perm]


@pytest.fixture(scope="module")
def demo_setup(cuda, demo):
    from adamixture_b200.model.svd_gpu import SVD_gpu
    from adamixture_b200 import ops as _ops

    M, N = int(demo["M"]), int(demo["N"])
    G = dev(demo["packed"])
    f = _ops.allele_frequency(G, M)
    U, S, V = SVD_gpu(G, N, M, f, 7, 42, 5, 1e-1, 8192, G.device, 256)
    return G, f, U, S, V


def test_demo_svd_matches_reference_gpu_golden(demo_setup, demo_gpu):
    _, _, U, S, V = demo_setup
    Uc, Vc = canonical(U.cpu().numpy(), V.cpu().numpy())
    np.testing.assert_allclose(S.cpu().numpy(), demo_gpu["svd_S"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(Uc, demo_gpu["svd_U"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(Vc, demo_gpu["svd_V"], rtol=RTOL, atol=ATOL)


def test_demo_als_matches_reference_gpu_golden(demo_setup, demo, demo_gpu):
    from adamixture_b200.model.als_gpu import ALS_gpu

    G, f, U, S, V = demo_setup
    M = int(demo["M"])
    P, Q = ALS_gpu(U.contiguous(), S.contiguous(), V.contiguous(), f, 42, M, 7, 1000, 1e-4, G.device)
    np.testing.assert_allclose(P.cpu().numpy(), demo_gpu["als_P"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(Q.cpu().numpy(), demo_gpu["als_Q"], rtol=RTOL, atol=ATOL)


def _check_model(demo, P, Q, P_ref, Q_ref):
    P, Q = align(Q_ref, P, Q)
    assert P.min() >= 1e-5 - 1e-12 and P.max() <= 1 - 1e-5 + 1e-12
    np.testing.assert_allclose(Q.sum(1), 1.0, atol=1e-9)
    np.testing.assert_allclose(P, P_ref, rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(Q, Q_ref, rtol=RTOL, atol=ATOL)
    G = demo["unpacked"]
    assert abs(orc.loglik(G, P, Q) - orc.loglik(G, P_ref, Q_ref)) <= LOGL_ATOL


def test_demo_brqn_matches_reference_gpu_golden(cuda, demo, demo_gpu):
    from adamixture_b200.model.br_qn_gpu import optimize_original_gpu

    M, N = int(demo["M"]), int(demo["N"])
    G = dev(demo["packed"])
    # the reference test's settings: max_iter 10000, tol 0.1, Q_hist 3, patience 3
    P, Q = optimize_original_gpu(G, dev(demo_gpu["als_P"]), dev(demo_gpu["als_Q"]), 10000, 7, M, N,
                                 0.1, 3, 3, G.device, 8192, 256)
    _check_model(demo, P.cpu().numpy(), Q.cpu().numpy(), demo_gpu["brqn_P"], demo_gpu["brqn_Q"])


def test_demo_adamem_matches_reference_gpu_golden(cuda, demo, demo_gpu):
    from adamixture_b200.model.em_adam_gpu import optimize_parameters_gpu

    M, N = int(demo["M"]), int(demo["N"])
    G = dev(demo["packed"])
    P, Q = optimize_parameters_gpu(G, dev(demo_gpu["als_P"]), dev(demo_gpu["als_Q"]), 0.005, 0.80, 0.88,
                                   1e-8, 10000, 5, 7, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 256,
                                   precision="f64")
    _check_model(demo, P.cpu().numpy(), Q.cpu().numpy(), demo_gpu["adamem_P"], demo_gpu["adamem_Q"])
