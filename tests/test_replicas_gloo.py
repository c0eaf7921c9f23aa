"""The multi-GPU path of bench.py is replicas only: every rank solves its own
copy of the workload, the timed region is the slowest rank's, and the job's
value is world x steps / that time.  Checked here with two gloo ranks on the
CPU (no GPU): the maximum over ranks every rank receives, the replica value,
and that the reference arm does its work on rank 0 only.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        e2e, res = [1000.0 + 500.0 * rank, 800.0 + 100.0 * rank]
        m = bench.max_over_ranks(dist, [e2e, res], "cpu")
        out[rank] = (m[0], m[1], bench.replica_value(world, 3, m[1]))
        # the reference arm: ranks other than 0 return at once without output
        if rank != 0:
            bench.run_reference(None, rank, world)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_report_replica_throughput():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        for r in range(2):
            e2e, res, value = out[r]
            assert e2e == 1500.0 and res == 900.0
            assert value == pytest.approx(2 * 3 / 0.9)
