"""The multi-rank host logic of bench.py (replicas, whole-job throughput from
the slowest rank's time) on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, REPO)
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    import bench
    t = bench.reduce_max(1.0 + rank)  # rank 1 is the slow one
    out[rank] = (t, bench.whole_job_gcups(1e9, 2, t, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0] == res[1] == (2.0, pytest.approx(2 * 1e9 * 2 / 2.0 / 1e9))


def test_single_process_reduce_is_identity():
    import sys
    sys.path.insert(0, REPO)
    import bench
    assert bench.reduce_max(3.5) == 3.5
    assert bench.whole_job_gcups(1e9, 4, 2.0, 1) == 2.0
