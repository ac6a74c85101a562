"""The allocation-free walk counter (saba_count_static) against the regular one.

Callers that cannot allocate device memory (their device memory belongs to another allocator or
budget, or they run in a loop where cudaMalloc/cudaFree would synchronise the device) keep the CSR
in their own device buffers and call saba_count_static, which uses a fixed array inside the library
as its scratch.  This file is collected last so that a failure here comes after every other test.
It must pass alone in a fresh process and after the other tests (the array keeps the previous
call's contents, so each call has to clear what it uses).

The argument checks that come before any CUDA call run on the CPU; the rest needs a GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def _static_call(d_idx, d_adj, n, depth, walks):
    from tgtp_b200 import _lib

    res = _lib.SabaResult()
    _lib.check(_lib.lib().saba_count_static(C.c_void_p(d_idx.data_ptr()),
                                            C.c_void_p(d_adj.data_ptr()), n, depth, walks,
                                            None, C.byref(res)))
    return int(res.visit_count), int(res.checksum), int(res.fallback_bouquets)


@pytest.mark.gpu
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


@pytest.mark.gpu
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


@pytest.mark.gpu
@pytest.mark.parametrize("bad", ["neighbour_out_of_range", "decreasing_offsets",
                                 "nonzero_first_offset", "edge_into_vertex_without_neighbours"])
def test_static_walk_counter_refuses_a_malformed_csr_before_walking(cuda_device, bad):
    """A CSR built on the host with one defect: the device check refuses it with
    TGTP_ERR_INVALID_ARGUMENT before any walk is launched (so no walk ever reads out of bounds),
    and a valid call right after it still gives the regular counter's summary."""
    import torch

    from tgtp_b200 import _lib
    from tgtp_b200.aesc import AESCGraph, saba_count

    # a triangle 0-1-2 plus vertex 3 joined to 0: every id < 4, every degree > 0
    idx = np.array([0, 3, 5, 7, 8], np.uint32)
    adj = np.array([1, 2, 3, 0, 2, 0, 1, 0], np.uint32)
    bidx, badj = idx.copy(), adj.copy()
    if bad == "neighbour_out_of_range":
        badj[4] = 4  # vertex 4 does not exist
    elif bad == "decreasing_offsets":
        bidx[2] = 2  # idx[2] < idx[1]
    elif bad == "nonzero_first_offset":
        bidx[0] = 1
    else:
        # vertex 3 keeps no neighbours (idx[4] = idx[3]) while 0 -> 3 stays: a walk would reach
        # a vertex it cannot leave; adj holds the 7 slots the offsets declare
        bidx[4] = 7
        badj = badj[:7].copy()
    d_idx = torch.from_numpy(bidx.astype(np.int32)).cuda()
    d_adj = torch.from_numpy(badj.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    res = _lib.SabaResult()
    status = _lib.lib().saba_count_static(C.c_void_p(d_idx.data_ptr()),
                                          C.c_void_p(d_adj.data_ptr()), 4, 5, 64, None,
                                          C.byref(res))
    assert status == 1, bad
    assert b"CSR" in _lib.lib().tgtp_last_error()
    g_idx = torch.from_numpy(idx.astype(np.int32)).cuda()
    g_adj = torch.from_numpy(adj.astype(np.int32)).cuda()
    ref = AESCGraph.from_csr(idx, adj)
    _, visits, checksum, fb = saba_count(ref, 5, 64, counters=False)
    assert _static_call(g_idx, g_adj, 4, 5, 64) == (visits, checksum, fb)
    ref.free()


@pytest.mark.gpu
def test_static_walk_counter_zero_depth_or_walks_gives_a_zero_summary(cuda_device):
    import torch

    from tgtp_b200 import synth

    g = synth.config1_graph(1)
    idx, adj = g.csr()
    d_idx = torch.from_numpy(idx.astype(np.int32)).cuda()
    d_adj = torch.from_numpy(adj.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    _static_call(d_idx, d_adj, g.n, 5, 64)  # leaves nonzero counters in the shared array
    for depth, walks in ((0, 64), (5, 0)):
        assert _static_call(d_idx, d_adj, g.n, depth, walks) == (0, 0, 0)


@pytest.mark.parametrize("n,walks,message", [(100, 12, b"multiple of 8"),
                                             (0, 64, b"empty graph"),
                                             ((1 << 22) + 1, 64, b"4194304")])
def test_static_walk_counter_argument_checks_need_no_gpu(tgtp_lib, n, walks, message):
    """These checks come before any CUDA call, so they run (and must refuse) without a GPU; the
    pointers are never dereferenced."""
    from tgtp_b200 import _lib

    res = _lib.SabaResult()
    fake = C.c_void_p(256)
    status = tgtp_lib.saba_count_static(fake, fake, n, 5, walks, None, C.byref(res))
    assert status == 1
    assert message in tgtp_lib.tgtp_last_error()
    assert tgtp_lib.saba_count_static(None, fake, 100, 5, 64, None, C.byref(res)) == 1
