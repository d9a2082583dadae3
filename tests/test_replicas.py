"""The multi-GPU form of bench.py is N independent replicas (the path has no
exchange step): its whole-job rate is every rank's entries over the slowest
rank's time.  Checked here with two gloo ranks on the CPU."""
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
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r: 1e9 (r + 1) entries in (1 + r) s and (2 + r) s
        rates, times = bench.replica_rates([1.0 + rank, 2.0 + rank],
                                           1e9 * (rank + 1), world, "cpu")
        out[rank] = (rates, times)
    finally:
        dist.destroy_process_group()


def test_replica_rates_two_gloo_ranks():
    world = 2
    port = _free_port()
    # the manager process is spawned too: forking this multi-threaded
    # process could deadlock the child
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    total = 1e9 * (1 + 2)
    for rank in range(world):
        rates, times = res[rank]
        assert times == [2.0, 3.0]                      # max over ranks
        assert rates == pytest.approx([total / 2.0 / 1e6, total / 3.0 / 1e6])


def test_replica_rates_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    rates, times = bench.replica_rates([0.5], 2e9, 1, "cpu")
    assert times == [0.5] and rates == [4000.0]
