"""Multi-rank timing of bench.py on CPU: two gloo ranks, each with its own
replica size and device time; the job time is the slowest rank's and the
throughput counts every rank's particles."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [12.0, 20.0][rank]
    n = [1000, 3000][rank]
    res = bench.combine_ranks(ms, n, 10, dist, "cpu")
    out[rank] = res
    dist.destroy_process_group()


def test_two_gloo_ranks_combine_as_max_time_and_summed_work():
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    for r in (0, 1):
        ms, n, value = out[r]
        assert ms == 20.0 and n == 4000.0
        assert value == pytest.approx(4000 * 10 / 0.020)


def test_single_rank_without_process_group():
    import bench
    ms, n, value = bench.combine_ranks(5.0, 200, 4)
    assert (ms, n) == (5.0, 200.0) and value == pytest.approx(200 * 4 / 0.005)
