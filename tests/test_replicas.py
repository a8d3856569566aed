"""The multi-GPU form of the path is independent replicas (one placement per
GPU, no data-path collective).  What runs on the host around them is checked
here on CPU with world_size 2 over gloo: the timing reduction takes the
maximum over ranks on every rank, and the reference arm runs on rank 0 only
(the other ranks exit 0 without output)."""
import datetime
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r = bench.max_over_ranks(dist, [rank + 1.0, 10.0 - rank, 0.5], "cpu")
        dist.barrier()
        q.put((rank, r))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got[0] == got[1] == [2.0, 10.0, 0.5]


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks(None, [3.0, 1.5], "cpu") == [3.0, 1.5]


def test_reference_arm_runs_on_rank0_only(capsys):
    class A:
        steps, warmup, gpus = 1, 0, 2
    assert bench.run_reference(A(), rank=1) == 0
    assert capsys.readouterr().out == ""
