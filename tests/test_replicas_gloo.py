"""Multi-rank replica protocol of bench.py on CPU: two gloo ranks time
different amounts of work, take the max over ranks and agree on the
whole-job throughput (the GPU runs use the same functions over NCCL)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    ms = 10.0 * (rank + 1)  # rank 1 is the slow one
    ms_max = bench.max_over_ranks(ms, device="cpu")
    out[rank] = (ms_max, bench.replica_value(1000.0, world, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert out[0] == out[1]
    ms_max, value = out[0]
    assert ms_max == 20.0
    assert value == pytest.approx(2 * 1000.0 / 0.020)


def test_single_process_is_identity():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5
    assert bench.replica_value(100.0, 1, 1000.0) == pytest.approx(100.0)
