"""Host logic of the data-parallel step on CPU ranks (gloo, world size 2): each rank owns
its own views, the gradients are summed across ranks between the adjoints and Adam, and the
parameters stay replicated.  Also the rank-failure path: a rank that raises before the
exchange makes the others' collective end with an error instead of hanging."""
import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _init(rank, world, port):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))


def _worker_allreduce(rank, world, port, out):
    sys.path.insert(0, ROOT)
    _init(rank, world, port)
    import bench
    from svraster_b200 import synthetic as S
    # views of rank r are the r-th block of the Fibonacci set (bench.make_workload)
    cams = S.fibonacci_cameras(2 * (rank + 1), 3.0, 8, 8)[2 * rank:2 * (rank + 1)]
    # stand-in per-rank gradients: a deterministic function of the rank's cameras
    g = [torch.full((5,), float(sum(c.position.sum() for c in cams)), dtype=torch.float32),
         torch.arange(3, dtype=torch.float32) * (rank + 1)]
    for t in g:
        dist.all_reduce(t)
    # Adam on replicated params gives identical params on every rank
    p = torch.zeros(5)
    p -= 0.1 * g[0]
    gathered = [torch.zeros(5) for _ in range(world)]
    dist.all_gather(gathered, p)
    out[rank] = (g[0][0].item(), g[1].tolist(), all(torch.equal(gathered[0], x) for x in gathered))
    dist.barrier()
    dist.destroy_process_group()


def _worker_fail(rank, world, port, out):
    _init(rank, world, port)
    try:
        if rank == 1:
            raise RuntimeError("rank 1 failed before the gradient exchange")
        t = torch.ones(3)
        dist.all_reduce(t)
        out[rank] = "completed"
    except Exception as e:          # noqa: BLE001 - any collective error is the expected outcome
        out[rank] = f"error: {type(e).__name__}"
    finally:
        try:
            dist.destroy_process_group()
        except Exception:           # noqa: BLE001
            pass


def _run(fn, world=2):
    port = 29500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=fn, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=90)
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
    return dict(out)


def test_data_parallel_gradient_allreduce_gloo():
    out = _run(_worker_allreduce)
    assert len(out) == 2
    a, b = out[0], out[1]
    assert a[0] == pytest.approx(b[0]) and a[1] == b[1] == [0.0, 3.0, 6.0]
    assert a[2] and b[2]


def test_failed_rank_does_not_hang_the_others():
    out = _run(_worker_fail)
    assert out[1].startswith("error")
    assert out[0].startswith("error") or out[0] == "completed"
