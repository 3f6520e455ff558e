"""Multi-rank path on CPU: two gloo ranks shard the visibilities, each grids
its rows (the FP64 DFT stands in for the GPU gridder, which is linear in the
same way) and the all-reduced image equals the single-rank image."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from wsclean_b200.dist import shard_rows, sharded_dirty2ms, sharded_ms2dirty


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _inputs():
    rng = np.random.default_rng(11)
    nrow = 501
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([400.0, 400.0, 100.0])
    freq = np.array([1.5e8])
    vis = rng.normal(size=(nrow, 1)) + 1j * rng.normal(size=(nrow, 1))
    return uvw, freq, vis


def _worker(rank, world, port, q):
    import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    uvw, freq, vis = _inputs()
    px = np.deg2rad(40 / 3600)

    def grid(u, f, v):
        return O.dft_ms2dirty(u, f, v, 16, 16, px, px, negate_v=True, divide_by_n=False)

    img = sharded_ms2dirty(grid, uvw, freq, vis)
    model = np.zeros((16, 16))
    model[3, 5] = 1.0

    def degrid(u, f, d):
        return O.dft_dirty2ms(u, f, d, px, px, negate_v=True, divide_by_n=False)

    lo, hi, v = sharded_dirty2ms(degrid, uvw, freq, model)
    q.put((rank, img.numpy(), lo, hi, v))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_gridding():
    import oracle as O
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    uvw, freq, vis = _inputs()
    px = np.deg2rad(40 / 3600)
    full = O.dft_ms2dirty(uvw, freq, vis, 16, 16, px, px, negate_v=True, divide_by_n=False)
    model = np.zeros((16, 16))
    model[3, 5] = 1.0
    vfull = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=True, divide_by_n=False)
    for rank, img, lo, hi, v in res:
        assert np.allclose(img, full, rtol=1e-12, atol=1e-12)
        assert (lo, hi) == shard_rows(len(uvw), rank, world)
        assert np.allclose(v, vfull[lo:hi], rtol=1e-12, atol=1e-12)
