"""Seeded synthetic graphs standing in for the reference's downloaded datasets.

The reference reads `<folder>/<graph>/graph.txt` (src/graph.h:29-97), a whitespace edge list of
zero-based contiguous vertex ids with no isolated vertices, each undirected edge listed once
(datasets/README.md:3-9).  No dataset can be downloaded here, so every workload is generated from an
explicit seed:

* Chung-Lu power law: endpoint i drawn with probability proportional to (i+1)^(-1/(exponent-1)),
  edges sampled until `target_edges` distinct non-loop pairs exist;
* R-MAT (a, b, c, d = 1-a-b-c) recursive quadrant sampling of `edge_factor * 2^scale` pairs;
* 2-D grid with random chords up to a target average degree.

Every generator drops self-loops and duplicates, keeps the largest connected component and relabels
its vertices 0..n-1 in increasing original id, so the result is a simple connected graph that the
reference loader and ours accept unchanged.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class EdgeList:
    """Undirected simple graph: `u < v` for every row, rows unique, ids contiguous 0..n-1."""

    n: int
    u: np.ndarray  # int64
    v: np.ndarray  # int64
    name: str = ""

    @property
    def num_edges(self) -> int:
        return int(self.u.shape[0])

    def csr(self):
        """Reference CSR: both directions of every edge, rows sorted ascending (src/graph.h:63-95)."""
        src = np.concatenate([self.u, self.v])
        dst = np.concatenate([self.v, self.u])
        order = np.lexsort((dst, src))
        src, dst = src[order], dst[order]
        idx = np.zeros(self.n + 1, dtype=np.uint32)
        np.cumsum(np.bincount(src, minlength=self.n), out=idx[1:])
        return idx, dst.astype(np.uint32)


def _dedup_largest_component(n: int, a: np.ndarray, b: np.ndarray, name: str) -> EdgeList:
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    keep = a != b
    a, b = a[keep], b[keep]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(lo.astype(np.int64) * n + hi)
    lo, hi = key // n, key % n
    adj = coo_matrix((np.ones(lo.size, dtype=np.int8), (lo, hi)), shape=(n, n))
    ncomp, labels = connected_components(adj, directed=False)
    sizes = np.bincount(labels, minlength=ncomp)
    # Isolated ids (never sampled) form singleton components; the largest component wins.
    big = int(np.argmax(sizes))
    inside = labels == big
    new_id = np.cumsum(inside) - 1
    sel = inside[lo] & inside[hi]
    lo, hi = new_id[lo[sel]], new_id[hi[sel]]
    return EdgeList(int(inside.sum()), lo.astype(np.int64), hi.astype(np.int64), name)


def chung_lu(n: int, target_edges: int, exponent: float, seed: int) -> EdgeList:
    """Chung-Lu graph with power-law expected degrees (exponent > 2)."""
    rng = np.random.default_rng(seed)
    w = np.arange(1, n + 1, dtype=np.float64) ** (-1.0 / (exponent - 1.0))
    cdf = np.cumsum(w / w.sum())
    cdf[-1] = 1.0
    keys = np.empty(0, dtype=np.int64)
    order = np.empty(0, dtype=np.int64)
    drawn = 0
    while keys.size < target_edges:
        k = int((target_edges - keys.size) * 1.5) + 4096
        a = np.searchsorted(cdf, rng.random(k), side="right")
        b = np.searchsorted(cdf, rng.random(k), side="right")
        a = np.minimum(a, n - 1)
        b = np.minimum(b, n - 1)
        ok = a != b
        new = np.minimum(a, b)[ok] * n + np.maximum(a, b)[ok]
        allk = np.concatenate([keys, new])
        allo = np.concatenate([order, drawn + np.arange(new.size)])
        drawn += new.size
        uniq, first = np.unique(allk, return_index=True)
        # keep first occurrences, in sampling order
        sel = np.sort(first)
        keys, order = allk[sel], allo[sel]
    keys = keys[:target_edges]
    return _dedup_largest_component(n, keys // n, keys % n,
                                    f"chunglu_n{n}_e{target_edges}_x{exponent}_s{seed}")


def rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int) -> EdgeList:
    """R-MAT graph: each of edge_factor*2^scale pairs picks one quadrant per level."""
    rng = np.random.default_rng(seed)
    m = edge_factor << scale
    n = 1 << scale
    u = np.zeros(m, dtype=np.int64)
    v = np.zeros(m, dtype=np.int64)
    ab, abc = a + b, a + b + c
    for _ in range(scale):
        r = rng.random(m)
        bit_u = r >= ab
        bit_v = ((r >= a) & (r < ab)) | (r >= abc)
        u = (u << 1) | bit_u
        v = (v << 1) | bit_v
    return _dedup_largest_component(n, u, v, f"rmat_s{scale}_ef{edge_factor}_a{a}_s{seed}")


def grid_chords(rows: int, cols: int, avg_degree: float, seed: int) -> EdgeList:
    """rows x cols 4-neighbour grid plus uniformly random chords up to `avg_degree`."""
    rng = np.random.default_rng(seed)
    n = rows * cols
    ids = np.arange(n, dtype=np.int64).reshape(rows, cols)
    hu = ids[:, :-1].ravel()
    hv = ids[:, 1:].ravel()
    vu = ids[:-1, :].ravel()
    vv = ids[1:, :].ravel()
    base = hu.size + vu.size
    extra = max(0, int(avg_degree * n / 2) - base)
    cu = rng.integers(0, n, size=int(extra * 1.05) + 16)
    cv = rng.integers(0, n, size=cu.size)
    a = np.concatenate([hu, vu, cu])
    b = np.concatenate([hv, vv, cv])
    return _dedup_largest_component(n, a, b, f"grid_{rows}x{cols}_d{avg_degree}_s{seed}")


def write_graph_txt(g: EdgeList, path: str) -> None:
    """One `u v` line per undirected edge (datasets/README.md:3-9)."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savetxt(path, np.stack([g.u, g.v], axis=1), fmt="%d", delimiter=" ")


def config1_graph(seed: int = 1) -> EdgeList:
    """Chung-Lu n=4,039, 88,234 target edges, exponent 2.5: the SABA / AESC single-GPU workload."""
    return chung_lu(4039, 88234, 2.5, seed)


def config3_graph(seed: int = 1) -> EdgeList:
    """R-MAT scale 18, edge factor 16, a=0.57, b=c=0.19: the SABA throughput workload."""
    return rmat(18, 16, 0.57, 0.19, 0.19, seed)


def config5_graphs(seed: int = 5, count: int = 64):
    """The batched workload: `count` graphs of uneven size, n log-uniform in [1,000, 200,000], a
    third each Chung-Lu (exponent 2.1-2.8), R-MAT (a=0.57, b=c=0.19) and 2-D grid with random
    chords, average degree 8-40, each with its own epsilon from {0.05, 0.01, 0.005}.  Returns a
    list of (EdgeList, epsilon); every graph has its own seed derived from `seed`."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(1000), np.log(200000)))))
        deg = float(rng.uniform(8, 40))
        eps = float(rng.choice([0.05, 0.01, 0.005]))
        gseed = int(rng.integers(1, 2**31 - 1))
        kind = i % 3
        if kind == 0:
            g = chung_lu(n, int(n * deg / 2), float(rng.uniform(2.1, 2.8)), gseed)
        elif kind == 1:
            scale = max(10, int(round(np.log2(n))))
            g = rmat(scale, max(4, int(round(deg / 2))), 0.57, 0.19, 0.19, gseed)
        else:
            rows = max(2, int(round(np.sqrt(n))))
            g = grid_chords(rows, max(2, n // rows), deg, gseed)
        out.append((g, eps))
    return out
