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


def _partition_rank(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import ctypes
    import mahyco_b200 as mb
    from mahyco_b200.partition import partition_by_bytes, imbalance, gather_results
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    lib = mb.load()  # mhc_case_device_bytes is host-only
    cases = bench.batch_cases(300)
    sizes = [lib.mhc_case_device_bytes(ctypes.byref(p)) for p in cases]
    parts = partition_by_bytes(sizes, world)
    mine = parts[rank]
    # each rank "runs" its cases (a per-case result) and rank 0 gathers them
    got = gather_results({i: (i * 7 + 3, rank) for i in mine}, world)
    allparts = [None] * world
    dist.all_gather_object(allparts, parts)
    out[rank] = {"parts_agree": all(p == parts for p in allparts), "mine": mine,
                 "imbalance": imbalance(sizes, parts), "gathered": got, "ncases": len(cases)}
    dist.barrier()
    dist.destroy_process_group()


def test_case_partition_two_gloo_ranks():
    """The batched and served cases are split between ranks by device
    bytes: both ranks compute the same partition, every case is run by
    exactly one rank, the shares are balanced, and rank 0 gathers every
    case's result (mahyco_b200.partition, used by bench.py for N > 1)."""
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_partition_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    r0, r1 = out[0], out[1]
    assert r0["parts_agree"] and r1["parts_agree"]
    n = r0["ncases"]
    assert sorted(r0["mine"] + r1["mine"]) == list(range(n))
    assert not set(r0["mine"]) & set(r1["mine"])
    assert r0["imbalance"] < 1.02
    g = r0["gathered"]
    assert sorted(g) == list(range(n)) and r1["gathered"] is None
    assert all(g[i][0] == i * 7 + 3 for i in g)
    assert {g[i][1] for i in r0["mine"]} == {0} and {g[i][1] for i in r1["mine"]} == {1}


def test_partition_balances_and_is_deterministic():
    from mahyco_b200.partition import partition_by_bytes, imbalance
    import random
    rng = random.Random(3)
    sizes = [int(rng.lognormvariate(15, 1.5)) for _ in range(1000)]
    for world in (1, 2, 4, 8):
        parts = partition_by_bytes(sizes, world)
        assert parts == partition_by_bytes(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        assert imbalance(sizes, parts) < 1.05
