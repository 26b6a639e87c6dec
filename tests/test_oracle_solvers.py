"""Pins the CPU restatement of the BVLS, gradient/Hessian and SQP kernels (oracle/solvers.py)
to the reference's own CPU implementations (tests/golden/solvers.npz, made by the
reference's compiled bvls.pyx / sqp.pyx)."""
import numpy as np
import pytest

from oracle import solvers as osv

KS = (1, 3, 7, 12, 20, 40, 64)


@pytest.mark.parametrize("K", KS)
def test_bvls_matches_reference(solvers_golden, K):
    d = solvers_golden
    X = osv.bvls_bpp(d[f"bvls{K}_A"], d[f"bvls{K}_B"], 0.0, 1.0)
    np.testing.assert_allclose(X, d[f"bvls{K}_X"], rtol=1e-9, atol=1e-9)
    # the box is active somewhere in every case
    assert ((X <= 1e-12) | (X >= 1 - 1e-12)).any()


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_grad_hess_matches_reference(solvers_golden, tag):
    d = solvers_golden
    G, P, Q = d[f"{tag}_G"], d[f"{tag}_P"], d[f"{tag}_Q"]
    XtX_q, Xtz_q = osv.grad_hess_q(G, P, Q)
    XtX_p, Xtz_p = osv.grad_hess_p(G, P, Q)
    np.testing.assert_allclose(XtX_q, d[f"{tag}_XtX_q"], rtol=1e-10)
    np.testing.assert_allclose(Xtz_q, d[f"{tag}_Xtz_q"], rtol=1e-10)
    np.testing.assert_allclose(XtX_p, d[f"{tag}_XtX_p"], rtol=1e-10)
    np.testing.assert_allclose(Xtz_p, d[f"{tag}_Xtz_p"], rtol=1e-10)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_sqp_matches_reference(solvers_golden, tag):
    d = solvers_golden
    Qn = osv.sqp_solve_q(d[f"{tag}_XtX_q"], -d[f"{tag}_Xtz_q"], d[f"{tag}_Q"], d[f"{tag}_v_kk"])
    Pn = osv.sqp_solve_p(d[f"{tag}_XtX_p"], -d[f"{tag}_Xtz_p"], d[f"{tag}_P"])
    np.testing.assert_allclose(Qn, d[f"{tag}_Q_next"], atol=1e-9)
    np.testing.assert_allclose(Pn, d[f"{tag}_P_next"], atol=1e-9)
    np.testing.assert_allclose(Qn.sum(1), 1.0, atol=1e-12)
    assert Pn.min() >= 1e-5 and Pn.max() <= 1 - 1e-5


def test_rsvd_products_are_the_centred_products():
    rng = np.random.default_rng(0)
    G = rng.choice(4, size=(37, 23), p=[0.3, 0.3, 0.3, 0.1]).astype(np.uint8)
    f = rng.uniform(0.05, 0.95, 37)
    B = rng.normal(size=(23, 5))
    X = np.where(G == 3, 0.0, G - 2 * f[:, None])
    np.testing.assert_allclose(osv.rsvd_rows(G, f, B), X @ B)
    np.testing.assert_allclose(osv.rsvd_cols(G, f, X @ B), X.T @ (X @ B))
