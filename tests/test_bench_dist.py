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


def test_reference_arm_of_a_workload_without_a_reference_counterpart():
    """--impl reference prints an 'unavailable' line for the learned-preconditioner workload."""
    import json
    import subprocess
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "vardiff"], capture_output=True, text=True, timeout=120, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_reference_arm_on_other_ranks_does_no_work():
    """Under torchrun only rank 0 runs the reference arm; the others exit 0 at once."""
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    for wl in ("convdiff128", "ddcg160", "ddgmres128"):
        r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", wl],
                           capture_output=True, text=True, timeout=120, env=env)
        assert r.returncode == 0 and r.stdout.strip() == "", (wl, r.stdout, r.stderr[-500:])
