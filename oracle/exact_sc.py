"""TEST INFRASTRUCTURE ONLY: exact edge spanning centrality (effective resistance) per CSR slot.

Restates scripts/paper_accuracy.py:13-54 (and src/exact_sc.cpp:15-55): per connected component, the
grounded Laplacian (last vertex removed) is factored by dense Cholesky and inverted; the score of
slot (u, v) is G[u,u] + G[v,v] - 2 G[u,v] with G the inverse padded by a zero row / column.  The
solve is certified on seeded probe vectors and by Foster's theorem (the undirected scores sum to
n - #components), as the reference script does.  Dense, so for graphs up to ~20k vertices.
"""
from __future__ import annotations

import numpy as np


def exact_scores(idx: np.ndarray, adj: np.ndarray) -> np.ndarray:
    from scipy.linalg import cho_factor, cho_solve
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    n = len(idx) - 1
    m = int(idx[-1])
    rows = np.repeat(np.arange(n), np.diff(idx.astype(np.int64)))
    cols = adj.astype(np.int64)
    a = csr_matrix((np.ones(m), (rows, cols)), shape=(n, n))
    ncomp, labels = connected_components(a, directed=False)
    result = np.zeros(m)
    worst = 0.0
    for comp in range(ncomp):
        nodes = np.flatnonzero(labels == comp)
        sub = a[nodes][:, nodes].toarray()
        lap = np.diag(sub.sum(axis=1)) - sub
        grounded = lap[:-1, :-1]
        if grounded.size == 0:
            continue
        factor = cho_factor(grounded, lower=True)
        inverse = cho_solve(factor, np.eye(len(nodes) - 1))
        probe = np.random.default_rng(42).normal(size=(len(nodes) - 1, 4))
        worst = max(worst, float(np.max(np.abs(grounded @ cho_solve(factor, probe) - probe))))
        green = np.zeros((len(nodes), len(nodes)))
        green[:-1, :-1] = inverse
        local = np.full(n, -1, dtype=np.int64)
        local[nodes] = np.arange(len(nodes))
        pos = np.flatnonzero(labels[rows] == comp)
        u, v = local[rows[pos]], local[cols[pos]]
        result[pos] = green[u, u] + green[v, v] - 2 * green[u, v]
    foster = abs(result.sum() / 2 - (n - ncomp))
    if not np.all(np.isfinite(result)) or worst > 1e-6 or foster > 1e-5 * max(1, n):
        raise RuntimeError("exact reference failed residual/Foster checks")
    return result


def accuracy(scores: np.ndarray, exact: np.ndarray, eps: float) -> dict:
    """The statistics scripts/paper_accuracy.py:64-73 reports for one score vector."""
    err = np.abs(scores.astype(np.float64) - exact)
    return {"max_absolute_error": float(err.max()), "mean_absolute_error": float(err.mean()),
            "rmse": float(np.sqrt(np.mean(err ** 2))),
            "directed_edges_over_epsilon": int(np.count_nonzero(err > eps)),
            "fraction_within_epsilon": float(np.mean(err <= eps)),
            "within_epsilon": bool(err.max() <= eps)}
