"""The batched workload's accuracy: the graphs of the 64-graph batch with at most 4,000 vertices
(their exact spanning centrality is a dense solve), scored in the plain FP64 form one by one and in
the mixed form (BF16 vectors) as one batch.  The batch must equal the mixed form's single runs bit
for bit, and its scores must be about as close to the exact ones as the FP64 form's."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batched_mixed_is_as_accurate_as_fp64(cuda_device):
    import torch

    from oracle import exact_sc
    from tgtp_b200 import eigenprep_gpu, synth
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, Batch, PRECISION_FP64,
                                PRECISION_MIXED, VEC_BF16, VEC_F64)

    small = [(g, eps) for g, eps in synth.config5_graphs(5, 64) if g.n <= 4000]
    assert len(small) >= 8
    within64 = withinm = 0
    slots = 0
    graphs, runs, single = [], [], []
    for g, eps in small:
        vals, vecs, _, _, _ = eigenprep_gpu.compute(g.n, g.u, g.v, 128, seed=1, tol=1e-6,
                                                    max_iter=60)
        idx, adj = g.csr()
        dg = AESCGraph.from_csr(idx, adj)
        v64 = np.ascontiguousarray(vecs.T).ravel()
        dg.upload_eigens(vals, v64, VEC_F64)
        dg.upload_eigens(vals, v64.astype(np.float32), VEC_BF16)
        exact = exact_sc.exact_scores(idx, adj)
        f64 = AESC(dg, AESCConfig(eps, precision=PRECISION_FP64)).tgtp()
        a = AESC(dg, AESCConfig(eps, precision=PRECISION_MIXED, vec_dtype=VEC_BF16))
        mixed = a.tgtp()
        acc64 = exact_sc.accuracy(f64, exact, eps)
        accm = exact_sc.accuracy(mixed, exact, eps)
        within64 += round(acc64["fraction_within_epsilon"] * len(exact))
        withinm += round(accm["fraction_within_epsilon"] * len(exact))
        slots += len(exact)
        assert accm["max_absolute_error"] <= max(2 * acc64["max_absolute_error"], eps), (
            g.name, eps, accm, acc64)
        graphs.append(dg)
        runs.append((a, torch.empty(dg.m, dtype=torch.float32, device="cuda")))
        single.append(mixed)
    assert withinm >= within64 - 0.01 * slots, (withinm, within64, slots)
    b = Batch([(a, o.data_ptr()) for a, o in runs])
    b.run()
    b.wait()
    for (a, o), want in zip(runs, single):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), want.view(np.uint32))
    b.free()
    for dg in graphs:
        dg.free()
