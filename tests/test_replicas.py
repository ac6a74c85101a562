"""The multi-GPU host logic (tgtp_b200/replicas.py) on CPU: two gloo ranks, each with its own
seeded workload and its own time; the job's time is the slowest rank's and the job's rate counts
every rank's units."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    from tgtp_b200 import replicas, synth

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, w, local = replicas.rank_info()
    g = synth.chung_lu(300, 1500, 2.5, replicas.workload_seed(1, r))
    my_seconds = 0.5 + r  # rank 1 is the slow one
    slow, other = replicas.slowest([my_seconds, 10.0 - my_seconds])
    digest = int((g.u * 7919 + g.v).sum())
    out.put((r, w, local, g.num_edges, slow, other, replicas.job_rate(g.num_edges, slow, w),
             digest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_count_all_units():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, e0, s0, o0, rate0, d0), (r1, w1, l1, e1, s1, o1, rate1, d1) = got
    assert (r0, r1) == (0, 1) and w0 == w1 == 2 and (l0, l1) == (0, 1)
    assert s0 == s1 == pytest.approx(1.5)          # the slower rank's time
    assert o0 == o1 == pytest.approx(9.5)          # element-wise over the list
    assert d0 != d1                                # distinct seeded graphs per rank
    assert rate0 == pytest.approx(2 * e0 / 1.5)


def test_single_process_needs_no_process_group():
    from tgtp_b200 import replicas

    assert replicas.slowest([1.25, 2.0]) == [1.25, 2.0]
    assert replicas.job_rate(100, 2.0, 1) == 50.0
