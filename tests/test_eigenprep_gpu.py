"""The GPU eigen prep (tgtp_b200/eigenprep_gpu.py, the input preparation of src/eigenprep.h:95-189
for graphs too large for the scipy restatement), checked on the CPU against its definition: the
omega largest-magnitude eigenpairs of D^-1/2 A D^-1/2, back-transformed by sqrt(2m / deg_i)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", ["config1", "sparse5k"])
def test_gpu_eigenprep_pairs_have_small_residuals_and_match_lanczos(cuda_device, graph):
    import scipy.sparse as sp

    from tgtp_b200 import eigenprep, eigenprep_gpu, synth

    g = synth.config1_graph(1) if graph == "config1" else synth.chung_lu(5000, 12000, 2.1, 7)
    n, u, v = g.n, g.u, g.v
    omega = 128
    vals, vecs, m, iters, worst = eigenprep_gpu.compute(n, u, v, omega, seed=1, tol=1e-8)
    assert worst < 1e-8 and vals.shape == (omega,) and vecs.shape == (omega, n)
    # the operator, built here with scipy (independent of the torch code)
    deg = np.bincount(u, minlength=n).astype(np.float64) + np.bincount(v[u != v], minlength=n)
    w = 1.0 / np.sqrt(deg[u] * deg[v])
    off = u != v
    P = sp.csr_matrix((np.concatenate([w, w[off]]),
                       (np.concatenate([u, v[off]]), np.concatenate([v, u[off]]))), shape=(n, n))
    scale = np.sqrt(2.0 * m) / np.sqrt(deg)
    y = (vecs / scale[None, :]).T  # columns: unit eigenvectors of P
    res = np.linalg.norm(P @ y - y * vals[None, :], axis=0)
    assert res.max() < 1e-7, res.max()
    gram = y.T @ y
    assert np.abs(gram - np.eye(omega)).max() < 1e-8
    assert np.all(np.diff(np.abs(vals)) <= 1e-12)  # sorted by |lambda| descending
    # the same eigenvalues as the Lanczos restatement (scipy eigsh, tolerance 1e-6)
    ref_vals = eigenprep.compute(n, u, v, omega, seed=0)[0]
    assert np.max(np.abs(np.sort(vals) - np.sort(ref_vals))) < 1e-6
