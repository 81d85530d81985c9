"""The multi-rank logic of bench.py on CPU with the gloo backend, world size
2: every rank gets the slowest rank's time, ranks share the points and get
their own column block of weights, and the whole-job throughput counts all
ranks' columns against the slowest rank's time."""
import os
import queue
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys

    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    t_max = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
    wl = dict(bench.WORKLOADS["bench"], N=1000)
    pts, w = bench.gen_inputs(wl, rank)
    q.put((rank, t_max, pts[:3].tolist(), w[:4].tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            rank, t_max, pts, w = q.get(timeout=120)
            out[rank] = (t_max, pts, w)
    except queue.Empty:
        pass
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert sorted(out) == [0, 1]
    assert out[0][0] == out[1][0] == 20.0          # max over ranks, seen by all
    assert out[0][1] == out[1][1]                  # same points on every rank
    assert not np.allclose(out[0][2], out[1][2])   # own weight block per rank
    assert all(p.exitcode == 0 for p in procs)


def test_job_throughput():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    # 2 ranks x 1e6 points x 8 columns x 5 steps in 250 ms (slowest rank)
    assert bench.job_throughput(2, 1_000_000, 8, 5, 250.0) == pytest.approx(3.2e8)
