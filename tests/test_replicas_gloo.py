"""The multi-GPU bench path on CPU: two ranks over gloo take the max of their timings and
report whole-job throughput (replicas, weak scaling)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    local_seconds = [2.0, 3.0][rank]
    m = bench.reduce_max(local_seconds, dist, "cpu")
    out[rank] = (m, bench.aggregate(1000, 4, world, m))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1]
    m, value = out[0]
    assert m == 3.0
    assert value == pytest.approx(1000 * 4 * 2 / 3.0 / 1e6)
