"""TEST INFRASTRUCTURE ONLY: CPU restatement (numpy / Python loops, float64) of the
reference's initialisation and original-ADMIXTURE kernels. Only tests, the smoke check and
the benchmark's CPU baseline may use it; the library never does.

* ``bvls_bpp``: block principal pivoting BVLS, adamixture/src/utils_c/cuda/bvls_kernel.cu:11-164
  with the unconstrained start solved by the same elimination
  (adamixture/src/utils_c/cython/bvls.pyx:130-227).
* ``sqp_solve_q`` / ``sqp_solve_p``: sweep-operator active-set QP and projections,
  adamixture/src/utils_c/cuda/sqp_kernel.cu:6-311 (Xtz passed negated, as its caller does).
* ``grad_hess_q`` / ``grad_hess_p``: adamixture/src/utils_c/cython/sqp.pyx:258-328
  (the CUDA path's br_qn_gpu.py:67-138 computes the same sums).
* ``rsvd_rows`` / ``rsvd_cols``: the centred products of adamixture/model/svd_gpu.py:80-139.

Pinned in tests/test_oracle_solvers.py against the reference's compiled Cython modules
(bvls, sqp) on random problems.
"""
from __future__ import annotations

import numpy as np

SINGULAR_TOL = 1e-12
PIVOT_TOL = 1e-8


# ---------------------------------------------------------------- BVLS

def _solve_subset(A, bs, x, F):
    """Gauss-Jordan with partial pivoting on the free subset; False if singular."""
    idx = [i for i in range(len(F)) if F[i]]
    n = len(idx)
    if n == 0:
        return True
    aug = np.empty((n, n + 1))
    for a, i in enumerate(idx):
        aug[a, :n] = A[i, idx]
        aug[a, n] = bs[i]
    for i in range(n):
        col = np.abs(aug[i:, i])
        r = i + int(np.argmax(col))          # first maximum
        if col.max() < SINGULAR_TOL:
            return False
        if r != i:
            aug[[i, r], i:] = aug[[r, i], i:]
        aug[i, i:] = aug[i, i:] / aug[i, i]
        for k in range(n):
            if k != i:
                aug[k, i:] -= aug[k, i] * aug[i, i:]
    for a, i in enumerate(idx):
        x[i] = aug[a, n]
    return True


def bvls_row(A, b, lower, upper):
    K = len(b)
    F = [True] * K
    U = [False] * K
    x = np.zeros(K)
    if not _solve_subset(A, b.copy(), x, F):
        return x
    changed = False
    for i in range(K):
        if x[i] < lower - PIVOT_TOL:
            F[i], U[i], changed = False, False, True
        elif x[i] > upper + PIVOT_TOL:
            F[i], U[i], changed = False, True, True
    it = 1
    while changed and it < 50:
        bs = b.copy()
        for i in range(K):
            if F[i]:
                v = b[i]
                for j in range(K):
                    if not F[j]:
                        v -= A[i, j] * (upper if U[j] else lower)
                bs[i] = v
        if not _solve_subset(A, bs, x, F):
            break
        for i in range(K):
            if not F[i]:
                x[i] = upper if U[i] else lower
        y = A @ x - b
        changed = False
        for i in range(K):
            if F[i]:
                if x[i] < lower - PIVOT_TOL:
                    F[i], U[i], changed = False, False, True
                elif x[i] > upper + PIVOT_TOL:
                    F[i], U[i], changed = False, True, True
            elif not U[i] and y[i] < -PIVOT_TOL:
                F[i], U[i], changed = True, False, True
            elif U[i] and y[i] > PIVOT_TOL:
                F[i], U[i], changed = True, False, True
        it += 1
    return x


def bvls_bpp(A, B, lower, upper):
    A = np.asarray(A, dtype=np.float64)
    return np.stack([bvls_row(A, np.asarray(b, dtype=np.float64), lower, upper) for b in B])


# ---------------------------------------------------------------- SQP

def _sweep(T, k, inverse):
    piv = T[k, k]
    if piv == 0.0:
        return
    p = 1.0 / piv
    tmp = T[:, k].copy()
    T[:, k] = 0.0
    T[k, :] = 0.0
    tmp[k] = 1.0 if inverse else -1.0
    T -= np.outer(tmp, p * tmp)   # T[j, i] -= (p tmp[i]) tmp[j]


def _quadratic_program(T, par, p, c):
    sz = p + c + 1
    small, tol = 1e-5, 1e-8
    delta = np.zeros(p)
    d = np.diag(T).copy()
    for i in range(p):
        if d[i] <= 0.0 or T[i, i] < d[i] * tol:
            return delta
        _sweep(T, i, False)
    swept = [True] * p
    for i in range(p, p + c):
        if T[i, i] >= 0.0:
            return delta
        _sweep(T, i, False)
    for _ in range(1000):
        a = 1.0
        for i in range(p):
            if swept[i]:
                ui = T[i, sz - 1]
                ai = (1.0 if ui > 0.0 else 0.0) - par[i] - delta[i]
                if abs(ui) > 1e-10 and ai / ui < a:
                    a = ai / ui
        for i in range(p):
            if swept[i]:
                ui = T[i, sz - 1]
                delta[i] += a * ui
                T[i, sz - 1] = (1.0 - a) * ui
                T[sz - 1, i] = T[i, sz - 1]
        hit = None
        for i in range(p):
            v = par[i] + delta[i]
            critical = (0.0 >= v - small) or (1.0 <= v + small)
            if swept[i] and abs(T[i, i]) > 1e-10 and critical:
                hit = i
                break
        if hit is not None:
            _sweep(T, hit, True)
            swept[hit] = False
            continue
        for i in range(p):
            ui = T[i, sz - 1]
            v = par[i] + delta[i]
            violation = (ui > 0.0 and 0.0 >= v - small) or (ui < 0.0 and 1.0 <= v + small)
            if not swept[i] and violation:
                hit = i
                break
        if hit is not None:
            _sweep(T, hit, False)
            swept[hit] = True
            continue
        return delta
    return delta


def project_simplex_row(b, pc=1e-5):
    n = len(b)
    b = b - pc
    tau = 1.0 - n * pc
    order = sorted(range(n), key=lambda i: -b[i])   # stable: equal values keep their order
    tsum, tmax, bget = 0.0, 0.0, False
    for i in range(n - 1):
        tsum += b[order[i]]
        tmax = (tsum - tau) / (i + 1)
        if tmax >= b[order[i + 1]]:
            bget = True
            break
    if not bget:
        tmax = (tsum + b[order[n - 1]] - tau) / n
    return np.maximum(b - tmax, 0.0) + pc


def sqp_solve_q(XtX, Xtz_neg, Q, v_kk):
    N, K = Q.shape
    out = np.empty_like(Q)
    for i in range(N):
        H, r, x = XtX[i], Xtz_neg[i], Q[i]
        t2 = v_kk @ (H @ v_kk[:, 0])
        mu = max(2.0 * ((np.abs(t2).sum() - 2.0 * abs(t2[0])) / K), 0.0)
        sz = K + 2
        T = np.zeros((sz, sz))
        T[:K, :K] = H + mu
        T[:K, K] = 1.0
        T[K, :K] = 1.0
        T[:K, K + 1] = -r
        T[K + 1, :K] = -r
        T[K, K + 1] = T[K + 1, K] = 1.0 - x.sum()
        delta = _quadratic_program(T, x, K, 1)
        out[i] = project_simplex_row(x + delta)
    return out


def sqp_solve_p(XtX, Xtz_neg, P):
    M, K = P.shape
    out = np.empty_like(P)
    for j in range(M):
        H, r, x = XtX[j], Xtz_neg[j], P[j]
        sz = K + 1
        T = np.zeros((sz, sz))
        T[:K, :K] = H
        T[:K, K] = -r
        T[K, :K] = -r
        delta = _quadratic_program(T, x, K, 0)
        out[j] = np.clip(x + delta, 1e-5, 1.0 - 1e-5)
    return out


# ---------------------------------------------------------------- gradient / Hessian

def _coeffs(G, P, Q):
    """Entrywise (M x N) coefficients: a = g/h, b = (2-g)/(1-h), a/h, b/(1-h); 0 if missing."""
    g = G.astype(np.float64)
    obs = G != 3
    h = np.clip(P @ Q.T, 1e-10, 1.0 - 1e-10)
    a = np.where(obs, g / h, 0.0)
    b = np.where(obs, (2.0 - g) / (1.0 - h), 0.0)
    return a, b, a / h, b / (1.0 - h)


def grad_hess_q(G, P, Q):
    """XtX_q [N,K,K], Xtz_q [N,K] from unpacked G [M,N]."""
    a, b, ha, hb = _coeffs(G, P, Q)
    Pc = 1.0 - P
    Xtz = a.T @ P + b.T @ Pc
    XtX = np.einsum("ji,jk,jl->ikl", ha, P, P) + np.einsum("ji,jk,jl->ikl", hb, Pc, Pc)
    return XtX, Xtz


def grad_hess_p(G, P, Q):
    """XtX_p [M,K,K], Xtz_p [M,K] from unpacked G [M,N]."""
    a, b, ha, hb = _coeffs(G, P, Q)
    Xtz = (a - b) @ Q
    XtX = np.einsum("ji,ik,il->jkl", ha + hb, Q, Q)
    return XtX, Xtz


# ---------------------------------------------------------------- randomized SVD products

def centred(G, f):
    """g - 2 f_j (0 where missing), float64 [M, N] from unpacked G."""
    X = G.astype(np.float64) - 2.0 * np.asarray(f, dtype=np.float64)[:, None]
    X[G == 3] = 0.0
    return X


def rsvd_rows(G, f, B):
    return centred(G, f) @ np.asarray(B, dtype=np.float64)


def rsvd_cols(G, f, Y):
    return centred(G, f).T @ np.asarray(Y, dtype=np.float64)


# ---------------------------------------------------------------- cross-validation score

def deviance_sum(G, P, Q, flat):
    """Sum of g log(g/mu) + (2-g) log((2-g)/(2-mu)) over the entries at flat indices j*N+i,
    mu = clamp(2 P_j.Q_i, 1e-10, 2-1e-10) (adamixture/src/utils_c/cython/br_qn.pyx:92-150)."""
    N = G.shape[1]
    j, i = np.divmod(np.asarray(flat, dtype=np.int64), N)
    g = G[j, i].astype(np.float64)
    keep = g != 3
    j, i, g = j[keep], i[keep], g[keep]
    mu = np.clip(2.0 * np.einsum("ek,ek->e", Q[i], P[j]), 1e-10, 2.0 - 1e-10)
    with np.errstate(divide="ignore", invalid="ignore"):
        ta = np.where(g > 0, g * np.log(np.where(g > 0, g, 1.0) / mu), 0.0)
        rem = 2.0 - g
        tb = np.where(rem > 0, rem * np.log(np.where(rem > 0, rem, 1.0) / (2.0 - mu)), 0.0)
    return float((ta + tb).sum())
