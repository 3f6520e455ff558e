"""The grid-correction and column-twiddle tables are cached on the device, two
sets per context, the least recently used one replaced.  Calls that cycle
through three grid geometries evict a set on every call; in synchronous and
in pipelined mode they must give the results of a fresh context per geometry
(to FP32 rounding: the spreading atomics reorder sums)."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
# (nx, ny, eps): each its own kernel, grid and u transform
GEOMS = [(128, 128, 1e-5), (192, 160, 1e-4), (320, 256, 1e-6)]


def data(seed=31, nrow=20000):
    rng = np.random.default_rng(seed)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([2000.0, 2000.0, 250.0])
    vis = (rng.normal(size=(nrow, 1)) + 1j * rng.normal(size=(nrow, 1))).astype(np.complex64)
    return uvw, np.array([1.4e8]), vis, np.deg2rad(15.0 / 3600)


@pytest.mark.parametrize("pipelined", [False, True])
def test_cycling_geometries_evicts_tables_correctly(pipelined):
    from wsclean_b200.gridder import Context
    uvw, freq, vis, px = data()
    rng = np.random.default_rng(5)
    models = [rng.normal(size=(nx, ny)).astype(np.float32) for nx, ny, _ in GEOMS]
    want = []
    for (nx, ny, eps), m in zip(GEOMS, models):
        fresh = Context(0)
        want.append((fresh.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, **KW),
                     fresh.dirty2ms(uvw, freq, m, px, px, eps, **KW)))
    ctx = Context(0)
    reps = 3
    if not pipelined:
        for _ in range(reps):
            for (nx, ny, eps), m, (wd, wv) in zip(GEOMS, models, want):
                assert O.rel_rms(ctx.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, **KW), wd) < 5e-6
                assert O.rel_rms(ctx.dirty2ms(uvw, freq, m, px, px, eps, **KW), wv) < 5e-6
        return
    ctx.set_async(True)
    h_uvw = torch.as_tensor(uvw).pin_memory()
    h_vis = torch.as_tensor(vis).pin_memory()
    h_mod = [torch.as_tensor(m).pin_memory() for m in models]
    outs = []
    for _ in range(reps):
        for (nx, ny, eps), hm in zip(GEOMS, h_mod):
            od = torch.zeros((nx, ny), dtype=torch.float32).pin_memory()
            ov = torch.zeros((len(uvw), 1), dtype=torch.complex64).pin_memory()
            ctx.ms2dirty(h_uvw, freq, h_vis, nx, ny, px, px, eps, dirty=od, **KW)
            ctx.dirty2ms(h_uvw, freq, hm, px, px, eps, vis=ov, **KW)
            outs.append((od, ov))
    ctx.synchronize()
    ctx.set_async(False)
    for k, (od, ov) in enumerate(outs):
        wd, wv = want[k % len(GEOMS)]
        assert O.rel_rms(od.numpy(), wd) < 5e-6, k
        assert O.rel_rms(ov.numpy(), wv) < 5e-6, k
