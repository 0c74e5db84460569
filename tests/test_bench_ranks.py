"""The multi-GPU bench path on CPU: two gloo ranks run the same max-over-ranks
reduction bench.py uses under torchrun (independent replicas, weak scaling),
so the whole-job figure is (units of all ranks) / (slowest rank's time)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    value, ms_max = bench.replica_throughput(10.0 * (rank + 1), 1000, dist, device="cpu")
    out.put((rank, value, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms_max in res:
        assert ms_max == 20.0  # the slower rank's time on every rank
        assert value == pytest.approx(2 * 1000 / 0.020)


def test_replica_throughput_single_process():
    sys.path.insert(0, ROOT)
    import bench
    value, ms = bench.replica_throughput(4.0, 100, None, device="cpu")
    assert ms == 4.0 and value == pytest.approx(100 / 0.004)
