"""Column alignment of Q matrices across runs (consecutive K of a sweep), as the reference
does before writing each K's outputs (adamixture/src/main.py:87-91, plot.py:618-678,
clumppling.py:148-207): clusters are matched at minimum total mean squared distance with
every query cluster assigned once and every reference cluster receiving at least one, by a
minimum-cost assignment on the row-reduced distances; surplus query clusters join their
nearest reference cluster and are appended after the matched ones. Host work on K x K
matrices.
"""
from __future__ import annotations

import numpy as np
from scipy.optimize import linear_sum_assignment


def cluster_distances(P: np.ndarray, Q: np.ndarray) -> np.ndarray:
    """[K_Q, K_P] mean squared distance between the columns of Q and of P."""
    return ((Q[:, :, None] - P[:, None, :]) ** 2).sum(axis=0) / Q.shape[0]


def align_ilp(P: np.ndarray, Q: np.ndarray) -> tuple[float, list[int]]:
    """Cluster of P that each cluster of Q maps to (K_Q >= K_P)."""
    D = cluster_distances(np.asarray(P, np.float64), np.asarray(Q, np.float64))
    K_P = P.shape[1]
    reduced = (D - D.min(axis=1, keepdims=True)).T          # [K_P, K_Q]
    _, reps = linear_sum_assignment(reduced)
    idx = np.argmin(D, axis=1)
    idx[reps] = np.arange(K_P)
    return float(D[np.arange(D.shape[0]), idx].sum()), [int(i) for i in idx]


def align_clusters(ref_Q: np.ndarray, query_Q: np.ndarray) -> np.ndarray:
    """Permutation of query_Q's columns matching ref_Q's."""
    K_ref, K_q = ref_Q.shape[1], query_Q.shape[1]
    perm, used = [], set()
    if K_ref <= K_q:
        _, q2p = align_ilp(ref_Q, query_Q)
        groups: dict[int, list[int]] = {}
        for q_col, r_col in enumerate(q2p):
            groups.setdefault(r_col, []).append(q_col)
        for r in range(K_ref):
            cols = groups.get(r)
            if cols:
                cols.sort(key=lambda j: float(np.dot(ref_Q[:, r] - query_Q[:, j], ref_Q[:, r] - query_Q[:, j])))
                perm.append(cols[0])
                used.add(cols[0])
    else:
        _, p2q = align_ilp(query_Q, ref_Q)
        for i in range(K_ref):
            if p2q[i] not in used:
                perm.append(p2q[i])
                used.add(p2q[i])
    perm += [j for j in range(K_q) if j not in used]
    return np.array(perm, dtype=int)
