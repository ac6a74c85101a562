"""Eigenpair input preparation: a scipy restatement of the reference's `edgeutils -c`.

Follows src/eigenprep.h:95-189: rank-map and deduplicate the edges (:45-92), form the symmetrically
normalised adjacency A[i,j]/sqrt(deg_i*deg_j) (:108-124), take the `omega` largest-magnitude
eigenpairs with Lanczos (tolerance 1e-6, or 1e-4 above one million vertices; ncv =
min(n, max(2*omega+1, 20)), :128-138), back-transform each vector by sqrt(2m/deg_i) (:153-159),
stable-sort by |lambda| descending (:161-165) and write `stat.txt` and `sorted_eigens_<omega>.txt`
with 17 significant digits (:167-186).

The reference uses Spectra's SymEigsSolver; this uses ARPACK through scipy.sparse.linalg.eigsh.
Both are Lanczos solvers converged to the same tolerance, but they are different codes, so the
eigenpairs agree only to that tolerance: the eigen solver itself is not pinned against the
reference.  The hot path is unaffected by that, because both implementations read the very same
text file.
"""
from __future__ import annotations

import os
import time

import numpy as np


def read_edges(path: str):
    """Unique undirected (u, v) pairs with u <= v after rank-mapping ids (src/eigenprep.h:45-92)."""
    raw = []
    with open(path) as f:
        for line in f:
            if not line or line[0] in "#%":
                continue
            s = line.strip()
            if not s or s[0] in "#%":
                continue
            a, b = s.split()[:2]
            raw.append((int(a), int(b)))
    if not raw:
        raise RuntimeError("empty graph: " + path)
    e = np.asarray(raw, dtype=np.int64)
    if e.min() < 0:
        raise RuntimeError("invalid edge in " + path)
    ids = np.unique(e.ravel())
    r = np.searchsorted(ids, e)
    lo, hi = np.minimum(r[:, 0], r[:, 1]), np.maximum(r[:, 0], r[:, 1])
    key = np.unique(lo * len(ids) + hi)
    return len(ids), key // len(ids), key % len(ids)


def compute(n: int, u: np.ndarray, v: np.ndarray, omega: int, seed: int = 0):
    """Return (values, vectors) with vectors shaped (omega, n), sorted by |lambda| descending."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import eigsh

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
    p = sp.csr_matrix((data, (rows, cols)), shape=(n, n))
    tol = 1e-4 if n > 1_000_000 else 1e-6
    ncv = min(n, max(2 * omega + 1, 20))
    v0 = np.random.default_rng(seed).random(n) + 0.5
    vals, vecs = eigsh(p, k=omega, which="LM", tol=tol, ncv=ncv, v0=v0, maxiter=10 * n)
    scale = np.where(rs > 0, np.sqrt(2.0 * m) / np.sqrt(np.where(rs > 0, rs, 1.0)), 0.0)
    x = vecs * scale[:, None]
    # eigsh reports ascending algebraic order; the reference's stable |lambda|-descending sort
    # (src/eigenprep.h:161-165) is applied to it.  Ties of |lambda| are solver-order dependent.
    order = np.argsort(-np.abs(vals), kind="stable")
    return vals[order], np.ascontiguousarray(x[:, order].T), m


def write_files(folder: str, n: int, m: int, values: np.ndarray, vectors: np.ndarray) -> str:
    """stat.txt and sorted_eigens_<omega>.txt in the reference's text format (:167-186)."""
    os.makedirs(folder, exist_ok=True)
    omega = len(values)
    with open(os.path.join(folder, "stat.txt"), "w") as f:
        f.write(f"n={n}\nm={m}\nl={values[0]:f}")
    path = os.path.join(folder, f"sorted_eigens_{omega}.txt")
    with open(path, "w") as f:
        for j in range(omega):
            row = np.concatenate([[values[j]], vectors[j]])
            f.write(" ".join("%.17g" % x for x in row.tolist()))
            f.write("\n")
    return path


def eigenprep_folder(folder: str, omega: int, seed: int = 0, verbose: bool = False) -> str:
    """`edgeutils -c <folder> <omega>`: writes the eigen files next to `<folder>/graph.txt`."""
    n, u, v = read_edges(os.path.join(folder, "graph.txt"))
    t0 = time.time()
    vals, vecs, m = compute(n, u, v, omega, seed)
    if verbose:
        print(f"f={folder}, n={n}, m={m}, omega={omega}, time={time.time() - t0:.3f}s")
    return write_files(folder, n, m, vals, vecs)
