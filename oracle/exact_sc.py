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


def sampled_scores(idx: np.ndarray, adj: np.ndarray, slots: np.ndarray, device: str = "cpu",
                   tol: float = 1e-9, max_iter: int = 5000, batch: int = 128) -> np.ndarray:
    """Exact spanning centrality of selected CSR slots for graphs beyond a dense solve (the
    sampled-edge oracle of src/exact_sc.cpp:24-49's quantity): R(u, v) = (e_u - e_v)^T L^+ (e_u -
    e_v), with L^+ b from Jacobi-preconditioned conjugate gradients on the graph Laplacian in FP64
    (b is orthogonal to the constant vector, so the iterates stay in the range of L; the residual
    is re-projected each step).  `batch` right-hand sides are solved together; every column must
    reach a relative residual below `tol`.  Connected graphs only."""
    import torch

    n = len(idx) - 1
    rows = np.repeat(np.arange(n), np.diff(idx.astype(np.int64)))
    cols = adj.astype(np.int64)
    deg = np.diff(idx.astype(np.int64)).astype(np.float64)
    import warnings

    dev = torch.device(device)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        a = torch.sparse_csr_tensor(torch.from_numpy(idx.astype(np.int64)), torch.from_numpy(cols),
                                    torch.ones(len(cols), dtype=torch.float64), (n, n),
                                    check_invariants=False).to(dev)
    d = torch.from_numpy(deg).to(dev)
    inv_d = 1.0 / d
    u_all = rows[slots]
    v_all = cols[slots]
    out = np.empty(len(slots))
    for s0 in range(0, len(slots), batch):
        u = torch.from_numpy(u_all[s0:s0 + batch]).to(dev)
        v = torch.from_numpy(v_all[s0:s0 + batch]).to(dev)
        k = len(u)
        ar = torch.arange(k, device=dev)
        b = torch.zeros(n, k, dtype=torch.float64, device=dev)
        b[u, ar] += 1.0
        b[v, ar] -= 1.0
        x = torch.zeros_like(b)
        r = b.clone()
        z = r * inv_d[:, None]
        p = z.clone()
        rz = (r * z).sum(0)
        bnorm = torch.linalg.vector_norm(b, dim=0)
        for _ in range(max_iter):
            lp = d[:, None] * p - (a @ p)
            alpha = rz / (p * lp).sum(0)
            x += alpha * p
            r -= alpha * lp
            r -= r.mean(0, keepdim=True)
            if bool((torch.linalg.vector_norm(r, dim=0) <= tol * bnorm).all()):
                break
            z = r * inv_d[:, None]
            rz_new = (r * z).sum(0)
            p = z + (rz_new / rz) * p
            rz = rz_new
        else:
            raise RuntimeError("conjugate gradients did not converge")
        out[s0:s0 + k] = (x[u, ar] - x[v, ar]).cpu().numpy()
    return out
