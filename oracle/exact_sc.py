"""TEST INFRASTRUCTURE ONLY: exact edge spanning centrality (effective resistance) per CSR slot.

The quantity of scripts/paper_accuracy.py:13-54 and src/exact_sc.cpp:15-55: for the slot (u, v),
R(u, v) = (e_u - e_v)^T L^+ (e_u - e_v) on the simple undirected graph of the CSR (repeated slots
count once, self-loops are ignored; a self-loop slot scores 0).  Computed per connected component C
of k vertices from M = (L_C + J/k)^-1, J the all-ones matrix: L_C + J/k is symmetric positive
definite (J/k lifts the one zero eigenvalue of L_C, on the constant vector, to 1), its inverse is
L_C^+ + J/k, and the J/k part cancels in R, so R(u, v) = M[u,u] + M[v,v] - 2 M[u,v] from one dense
Cholesky factorisation per component.  Certified by the factorisation's residual on seeded probe
columns and by Foster's theorem (the undirected resistances sum to n - #components).  Dense, so
for graphs up to ~20k vertices; `sampled_scores` covers larger ones.
"""
from __future__ import annotations

import numpy as np


def exact_scores(idx: np.ndarray, adj: np.ndarray) -> np.ndarray:
    from scipy.linalg import cho_factor, cho_solve
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    n = len(idx) - 1
    src = np.repeat(np.arange(n), np.diff(idx.astype(np.int64)))
    dst = adj.astype(np.int64)
    off = src != dst
    simple = csr_matrix((np.ones(int(off.sum())), (src[off], dst[off])), shape=(n, n))
    simple.sum_duplicates()
    simple.data[:] = 1.0  # one edge per vertex pair
    ncomp, comp_of = connected_components(simple, directed=False)
    out = np.zeros(len(dst))
    residual = 0.0
    undirected_sum = 0.0
    probes = np.random.default_rng(7)
    for c in range(ncomp):
        members = np.flatnonzero(comp_of == c)  # ascending: local index by searchsorted
        k = len(members)
        block = simple[members][:, members].toarray()
        shifted = np.diag(block.sum(axis=1)) - block + 1.0 / k
        factor = cho_factor(shifted, lower=True)
        inv = cho_solve(factor, np.eye(k))
        z = probes.standard_normal((k, 4))
        residual = max(residual, float(np.max(np.abs(shifted @ (inv @ z) - z))))
        slots = np.flatnonzero(off & (comp_of[src] == c))
        lu = np.searchsorted(members, src[slots])
        lv = np.searchsorted(members, dst[slots])
        out[slots] = inv[lu, lu] + inv[lv, lv] - 2.0 * inv[lu, lv]
        iu, iv = np.nonzero(np.triu(block, 1))
        undirected_sum += float(np.sum(inv[iu, iu] + inv[iv, iv] - 2.0 * inv[iu, iv]))
    foster = abs(undirected_sum - (n - ncomp))
    # an edge's effective resistance lies in [0, 1] (src/exact_sc.cpp:46 checks 1 + 1e-9)
    in_range = bool(np.all((out >= -1e-12) & (out <= 1 + 1e-9)))
    if not np.all(np.isfinite(out)) or residual > 1e-6 or foster > 1e-5 * max(1, n) or not in_range:
        raise RuntimeError(f"exact spanning centrality not certified: probe residual {residual:.3g}, "
                           f"Foster deviation {foster:.3g}, range ok {in_range}")
    return out


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
