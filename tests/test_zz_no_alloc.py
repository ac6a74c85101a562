"""The allocation-free walk counter (saba_count_static) against the regular one.

Callers that cannot allocate device memory (their device memory belongs to another allocator or
budget, or they run in a loop where cudaMalloc/cudaFree would synchronise the device) keep the CSR
in their own device buffers and call saba_count_static, which uses a fixed array inside the library
as its scratch.  This file is collected last so that a failure here comes after every other test.
It must pass alone in a fresh process and after the other tests (the array keeps the previous
call's contents, so each call has to clear what it uses)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_call(d_idx, d_adj, n, depth, walks):
    from tgtp_b200 import _lib

    res = _lib.SabaResult()
    _lib.check(_lib.lib().saba_count_static(C.c_void_p(d_idx.data_ptr()),
                                            C.c_void_p(d_adj.data_ptr()), n, depth, walks,
                                            None, C.byref(res)))
    return int(res.visit_count), int(res.checksum), int(res.fallback_bouquets)


@pytest.mark.parametrize("kind", ["config1", "rmat"])
def test_static_walk_counter_matches_regular_entry_point_twice(cuda_device, kind):
    import torch

    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    g = synth.config1_graph(1) if kind == "config1" else synth.rmat(15, 8, 0.57, 0.19, 0.19, 9)
    idx, adj = g.csr()
    # caller-owned device buffers (here: torch's allocator, standing in for the caller's arena)
    d_idx = torch.from_numpy(idx.astype(np.int32)).cuda()
    d_adj = torch.from_numpy(adj.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    ref = AESCGraph.from_csr(idx, adj)
    for depth, walks in ((5, 2048), (10, 64)):
        _, visits, checksum, fb = saba_count(ref, depth, walks, counters=False)
        want = (visits, checksum, fb)
        first = _static_call(d_idx, d_adj, g.n, depth, walks)
        second = _static_call(d_idx, d_adj, g.n, depth, walks)
        assert first == want and second == want, (depth, walks, first, second, want)
    ref.free()


def test_static_walk_counter_rejects_oversized_graph(cuda_device):
    import torch

    from tgtp_b200.aesc import TgtpError

    d = torch.zeros(8, dtype=torch.int32, device="cuda")
    from tgtp_b200 import _lib

    res = _lib.SabaResult()
    status = _lib.lib().saba_count_static(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
                                          (1 << 22) + 1, 5, 64, None, C.byref(res))
    assert status == 1
    assert b"4194304" in _lib.lib().tgtp_last_error()
    with pytest.raises(TgtpError):
        _lib.check(status)
