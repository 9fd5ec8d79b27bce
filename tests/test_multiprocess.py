"""Host logic of the data-parallel step on CPU ranks (gloo, world size 2): each rank owns
its own views (``bench.rank_cameras``), the gradients live in one flat buffer
(``svraster_b200.step.flat_views``) that one all-reduce sums across ranks between the
adjoints and Adam, the parameters stay replicated, and the job time is the slowest rank's
(``bench.max_over_ranks``).  Also the rank-failure path: a rank that raises before the
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
    from svraster_b200.step import flat_views
    # the rank's views: bench.rank_cameras, as the data-parallel bench assigns them
    cams = bench.rank_cameras(rank, 2)
    positions = torch.tensor(np.stack([c.position for c in cams]), dtype=torch.float64)
    gathered_pos = [torch.zeros_like(positions) for _ in range(world)]
    dist.all_gather(gathered_pos, positions)
    # gradients of the three parameter groups (grid, sh0, shs shapes of a small scene) as
    # views of one flat buffer, filled with a per-rank pattern; one all-reduce of the flat
    # buffer is the exchange the bench's gradient hook makes
    shapes = [(37, 1), (11, 3), (11, 45)]
    flat, grads = flat_views(shapes, "cpu")
    for gi, gv in enumerate(grads):
        gv.copy_(torch.arange(gv.numel(), dtype=torch.float32).view(gv.shape) * (rank + 1) + gi)
    dist.all_reduce(flat)
    # Adam-like update on replicated parameters stays identical on every rank
    p = torch.zeros(11, 45)
    p -= 0.1 * grads[2]
    gathered = [torch.zeros_like(p) for _ in range(world)]
    dist.all_gather(gathered, p)
    # the job time is the slowest rank's
    job_ms = bench.max_over_ranks(10.0 + rank, "cpu")
    pad_zero = True
    off = 0
    for gv in grads:
        n = gv.numel()
        end = (n + 63) // 64 * 64
        pad_zero &= bool((flat[off + n:off + end] == 0).all())
        off += end
    out[rank] = dict(grads=[g.clone().numpy() for g in grads], same_params=all(torch.equal(gathered[0], x) for x in gathered),
                     positions=[x.numpy() for x in gathered_pos], job_ms=job_ms, pad_zero=pad_zero,
                     aligned=[(g.data_ptr() - flat.data_ptr()) % 256 == 0 for g in grads])
    dist.barrier()
    dist.destroy_process_group()


def _view_gradients(sc, cams, views):
    """The oracle's adjoint over views ``views`` of ``cams``, summed, as the step's gradient groups: grid-point
    gradients (corner terms scattered by vox_key) and the sh0 / shs gradients of the SH
    adjoint, in one flat float64 vector."""
    from oracle import oracle as O
    O.set_threads(1)                              # deterministic sums (other tests may raise it)
    N = sc.n_vox
    geos = O.gather_geo(np.arange(N), sc.vox_key, sc.geo_grid_pts, N)
    dgrid = np.zeros(len(sc.geo_grid_pts), np.float64)
    dsh0 = np.zeros((N, 3), np.float64)
    dshs = np.zeros((N, 15, 3), np.float64)
    for k in views:
        cam = cams[k]
        rgbs = O.sh_eval(3, None, sc.vox_center, cam.position, sc.sh0, sc.shs)
        nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
        keys, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
        f = O.render_fwd(cam, np.zeros(3, np.float32), 3, True, True, ranges, vals, bb, sc.vox_center, sc.vox_size,
                         geos, rgbs, sc.s_val)
        rng = np.random.default_rng(100 + k)          # view k's own upstream gradients
        g = [rng.normal(size=(c, cam.height, cam.width)).astype(np.float32) for c in (3, 4, 3)]
        dvox, _ = O.render_bwd(cam, np.zeros(3, np.float32), True, True, ranges, f["tile_last"], vals, bb,
                               sc.vox_center, sc.vox_size, geos, rgbs, sc.s_val, f["T"], f["n_contrib"], g[0], g[1],
                               g[2], np.zeros((1, cam.height, cam.width), np.float32))
        np.add.at(dgrid, sc.vox_key.reshape(-1), dvox[:, :8].reshape(-1).astype(np.float64))
        d0, d1 = O.sh_eval_bw(3, None, sc.vox_center, cam.position, dvox[:, 8:11].copy(), 16)
        dsh0 += d0
        dshs += d1.reshape(N, 15, 3)
    return np.concatenate([dgrid, dsh0.reshape(-1), dshs.reshape(-1)])


def _scene_and_views():
    from svraster_b200 import synthetic as S
    sc = S.scene_tiny(seed=4)
    return sc, S.ring_cameras(4, 3.0, 64, 48, fovx_deg=50.0, phase=0.1)


def _worker_view_adjoint(rank, world, port, out):
    sys.path.insert(0, ROOT)
    _init(rank, world, port)
    sc, cams = _scene_and_views()
    mine = list(range(rank, len(cams), world))    # disjoint views per rank
    local = torch.from_numpy(_view_gradients(sc, cams, mine))
    dist.all_reduce(local)                        # the step's one exchange
    out[rank] = local.numpy()
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
    world = 2
    shapes = [(37, 1), (11, 3), (11, 45)]
    for r in range(world):
        o = out[r]
        # every view holds the sum over ranks of rank-scaled patterns: arange * (1 + 2) + 2 * gi
        for gi, (g, shape) in enumerate(zip(o["grads"], shapes)):
            expect = np.arange(int(np.prod(shape)), dtype=np.float32).reshape(shape) * 3 + 2 * gi
            assert np.array_equal(g, expect)
        assert o["pad_zero"] and all(o["aligned"])
        assert o["same_params"]
        assert o["job_ms"] == 11.0
    # ranks own different views (weak scaling over views)
    p0, p1 = out[0]["positions"]
    assert p0.shape == p1.shape == (2, 3)
    assert not np.allclose(p0, p1)


def test_failed_rank_does_not_hang_the_others():
    out = _run(_worker_fail)
    assert out[1].startswith("error")
    assert out[0].startswith("error") or out[0] == "completed"


def test_data_parallel_adjoint_equals_single_process():
    """Two ranks, each running the oracle's adjoint on its own views and summing the ranks'
    gradients with one all-reduce, get the gradients one process computes over all the views
    (the property the data-parallel step rests on), up to the order of the summation."""
    sys.path.insert(0, ROOT)
    out = _run(_worker_view_adjoint)
    sc, cams = _scene_and_views()
    ref = _view_gradients(sc, cams, range(len(cams)))
    assert np.abs(ref).max() > 0
    for r in (0, 1):
        got = out[r]
        assert got.shape == ref.shape
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-9 * np.abs(ref).max() + 1e-12)
    assert np.array_equal(out[0], out[1]), "the ranks' reduced gradients differ"
