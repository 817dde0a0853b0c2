"""Replica aggregation of bench.py over world_size 2 with gloo on the CPU."""
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


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    from sph_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank r steps 1000 (r + 1) particles for 4 steps in 10 (r + 1) ms
    value, ms = replicas.throughput(1000 * (rank + 1), 4, 10.0 * (rank + 1))
    out[rank] = (value, ms)
    dist.destroy_process_group()


def test_two_ranks_sum_units_and_take_the_slowest_time():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    # (1000 + 2000) x 4 particle-steps over the slower 20 ms, on every rank
    for r in (0, 1):
        value, ms = res[r]
        assert ms == pytest.approx(20.0)
        assert value == pytest.approx(3000 * 4 / 0.020)


def test_single_process_is_unchanged():
    from sph_b200 import replicas
    value, ms = replicas.throughput(500, 2, 4.0)
    assert ms == 4.0 and value == pytest.approx(1000 / 0.004)
