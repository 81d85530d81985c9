"""The column-split matvec over ranks (pbbfmm3d_b200.columns) with the gloo
backend, world size 2.

CPU: the block split and the exchange, with the single-GPU matvec replaced
by a dense float64 product (the host logic only: which rank computes which
columns and where the gathered blocks land).  GPU: two ranks, each with its
own tree on cuda:0, against one full matvec of all columns (the ranks never
wait on each other inside a kernel; only the host-side all-gather joins
them)."""
import os
import queue
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs(N=3000, Ns=2500, C=5):
    rng = np.random.default_rng(7)
    return (rng.uniform(-0.5, 0.5, (N, 3)), rng.uniform(-0.5, 0.5, (Ns, 3)),
            rng.standard_normal(Ns * C), C)


def _dense(target, source, weight, C):
    d = np.linalg.norm(target[:, None, :] - source[None, :, :], axis=2)
    K = np.exp(-d / 0.3)
    return (K @ weight.reshape(C, -1).T).T.ravel()


def _worker(rank, world, port, q, use_gpu):
    import datetime
    import sys

    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    import pbbfmm3d_b200 as fmm
    from pbbfmm3d_b200 import columns

    tg, sr, w, C = _inputs()
    calls = []
    if use_gpu:
        tree = fmm.kernel_ExpCov(1.0, 4, 4, 1e-5, 0, ell=0.3, device=0)
        tree.buildFMMTree()
    else:
        tree = None

        def fake(tree_, t, s, ww, nc, out):
            calls.append(nc)
            out += _dense(t, s, ww, nc)
            return out

        columns.H2_3D_Compute = fake
    out = np.full(tg.shape[0] * C, 1.0)
    columns.H2_3D_Compute_columns(tree, tg, sr, w, C, out)
    q.put((rank, out, calls))
    dist.barrier()
    dist.destroy_process_group()


def _run_ranks(use_gpu):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, use_gpu)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(2):
            rank, out, calls = q.get(timeout=600)
            got[rank] = (out, calls)
    except queue.Empty:
        pass
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
    assert sorted(got) == [0, 1]
    assert all(p.exitcode == 0 for p in procs)
    return got


def test_column_blocks():
    import sys

    sys.path.insert(0, ROOT)
    from pbbfmm3d_b200.columns import column_blocks

    for nc in range(0, 20):
        for world in range(1, 9):
            b = column_blocks(nc, world)
            assert len(b) == world and b[0][0] == 0 and b[-1][1] == nc
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [y - x for x, y in b]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_two_ranks_host_logic_gloo():
    got = _run_ranks(use_gpu=False)
    tg, sr, w, C = _inputs()
    ref = 1.0 + _dense(tg, sr, w, C)
    assert got[0][1] == [3] and got[1][1] == [2]  # 5 columns: 3 + 2
    for r in (0, 1):
        np.testing.assert_allclose(got[r][0], ref, rtol=1e-13, atol=1e-12)


@pytest.mark.gpu
def test_two_ranks_matvec_gloo():
    import sys

    sys.path.insert(0, ROOT)
    import pbbfmm3d_b200 as fmm

    got = _run_ranks(use_gpu=True)
    tg, sr, w, C = _inputs()
    tree = fmm.kernel_ExpCov(1.0, 4, 4, 1e-5, 0, ell=0.3, device=0)
    tree.buildFMMTree()
    full = np.full(tg.shape[0] * C, 1.0)
    fmm.H2_3D_Compute(tree, tg, sr, w, C, full)
    for r in (0, 1):
        assert np.linalg.norm(got[r][0] - full) <= 1e-14 * np.linalg.norm(full)
