"""Host logic of the multi-GPU run on CPU: two gloo ranks, each timing its
own replica of the batch; the job's step time is the maximum over ranks and
its throughput counts every rank's problems (bench.py's contract)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.job_ms(100.0 + 25.0 * rank, ws, "cpu")  # rank 1 is the slower one
        out[rank] = (ms, bench.job_throughput(64, ws, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    ws, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    for rank in range(ws):
        ms, value = res[rank]
        assert ms == pytest.approx(125.0)
        assert value == pytest.approx(2 * 64 / 0.125)


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.job_ms(80.0, 1, "cpu") == 80.0
    assert bench.job_throughput(64, 1, 80.0) == pytest.approx(800.0)
