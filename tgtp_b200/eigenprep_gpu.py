"""Eigenpair input preparation on the GPU, for graphs too large for the scipy restatement.

Produces what `eigenprep.compute` (src/eigenprep.h:95-189) produces -- the `omega` largest-magnitude
eigenpairs of the symmetrically normalised adjacency D^-1/2 A D^-1/2, each vector back-transformed
by sqrt(2m / deg_i), sorted by |lambda| descending -- with Chebyshev-filtered subspace iteration in
FP64 instead of Lanczos: a block of omega + 32 vectors is repeatedly multiplied by an even Chebyshev
polynomial of the matrix that is bounded by 1 on [-c, c] (c = the smallest Ritz magnitude of the
block, so the wanted |lambda| > c are amplified), re-orthonormalised, and Rayleigh-Ritz projected,
until the wanted pairs' residuals ||P x - lambda x|| fall below `tol`.  The reference's solver and
this one converge to the same eigenpairs to their tolerances; neither is on the measured path
(tgtp reads the pairs from memory or from the text file either way).  This is input preparation:
it uses torch's sparse and dense linear algebra on the GPU.
"""
from __future__ import annotations

import numpy as np


def compute(n: int, u: np.ndarray, v: np.ndarray, omega: int, seed: int = 0, tol: float = 1e-6,
            degree: int = 16, max_iter: int = 200, device: str = "cuda"):
    """(values, vectors (omega, n), m, iterations, max residual), like eigenprep.compute."""
    import torch

    if omega < 2 or omega >= n:
        raise RuntimeError(f"omega must satisfy 2 <= omega < n; got {omega} for n={n}")
    m = len(u)
    rs = np.bincount(u, minlength=n).astype(np.float64)
    rs += np.bincount(v[u != v], minlength=n)
    val = 1.0 / np.sqrt(rs[u] * rs[v])
    off = u != v
    rows = np.concatenate([u, v[off]])
    cols = np.concatenate([v, u[off]])
    data = np.concatenate([val, val[off]])
    import warnings

    dev = torch.device(device)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        coo = torch.sparse_coo_tensor(torch.from_numpy(np.stack([rows, cols])),
                                      torch.from_numpy(data), (n, n), dtype=torch.float64,
                                      check_invariants=False)
        p = coo.coalesce().to_sparse_csr().to(dev)
    b = min(n - 1, omega + 32)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn(n, b, generator=gen, dtype=torch.float64).to(dev)
    x, _ = torch.linalg.qr(x)

    def rayleigh_ritz(x):
        px = p @ x
        h = x.T @ px
        h = 0.5 * (h + h.T)
        theta, w = torch.linalg.eigh(h)
        order = torch.argsort(theta.abs(), descending=True)
        theta, w = theta[order], w[:, order]
        return theta, x @ w, px @ w

    it, worst = 0, float("inf")
    for it in range(1, max_iter + 1):
        theta, x, px = rayleigh_ritz(x)
        res = torch.linalg.vector_norm(px[:, :omega] - x[:, :omega] * theta[:omega], dim=0)
        worst = float(res.max())
        if worst < tol:
            break
        c = float(theta[-1].abs().clamp(min=1e-3))
        # even Chebyshev filter T_degree(P / c) by its three-term recurrence, rescaled each step
        y0, y1 = x, (p @ x) / c
        for _ in range(2, degree + 1):
            y2 = 2.0 * (p @ y1) / c - y0
            s = torch.linalg.vector_norm(y2, dim=0).clamp(min=1e-300)
            y0, y1 = y1 / s, y2 / s
        x, _ = torch.linalg.qr(y1)
    theta, x, _ = rayleigh_ritz(x)
    vals = theta[:omega].cpu().numpy()
    vecs = x[:, :omega].cpu().numpy()
    scale = np.where(rs > 0, np.sqrt(2.0 * m) / np.sqrt(np.where(rs > 0, rs, 1.0)), 0.0)
    vecs = vecs * scale[:, None]
    order = np.argsort(-np.abs(vals), kind="stable")
    return vals[order], np.ascontiguousarray(vecs[:, order].T), m, it, worst
