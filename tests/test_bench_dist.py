"""The multi-process path of bench.py on CPU: two gloo ranks reduce their step times to
the slowest rank's, as the GPU replicas do over NCCL."""
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


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        times = [0.10 + 0.05 * rank, 1.0 + rank]
        out = bench.reduce_max(times, dist, "cpu")
        q.put((rank, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    for r in range(2):
        assert got[r] == pytest.approx([0.15, 2.0])


def test_reduce_max_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max([0.3, 4.0]) == [0.3, 4.0]
