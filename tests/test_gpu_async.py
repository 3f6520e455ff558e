"""Pipelined raw operators (wsg_ctx_set_async): a sequence of ms2dirty /
dirty2ms calls on page-locked host buffers and on device tensors returns
before the work is done, overlaps transfers with kernels through the three
staging slots, and after synchronize() gives the synchronous results (to
FP32 rounding: atomics reorder sums)."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


def test_pipelined_sequence_matches_synchronous():
    from wsclean_b200 import gridder as G
    from wsclean_b200 import synth
    c = synth.config2(scale=0.05, npix=512, pixsize_arcsec=40.0)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(12)
    n = 5
    vis = [(rng.normal(size=(len(uvw), 1)) + 1j * rng.normal(size=(len(uvw), 1))).astype(np.complex64)
           for _ in range(n)]
    models = [rng.normal(size=(nx, nx)).astype(np.float32) for _ in range(n)]
    sync = G.Context(0)
    want_d = [sync.ms2dirty(uvw, freq, v, nx, nx, px, px, 1e-5, **KW) for v in vis]
    want_v = [sync.dirty2ms(uvw, freq, m, px, px, 1e-5, **KW) for m in models]

    ctx = G.Context(0)
    ctx.set_async(True)
    h_uvw = torch.as_tensor(uvw).pin_memory()
    h_vis = [torch.as_tensor(v).pin_memory() for v in vis]
    h_mod = [torch.as_tensor(m).pin_memory() for m in models]
    out_d = [torch.zeros((nx, nx), dtype=torch.float32).pin_memory() for _ in range(n)]
    out_v = [torch.zeros((len(uvw), 1), dtype=torch.complex64).pin_memory() for _ in range(n)]
    for k in range(n):
        ctx.ms2dirty(h_uvw, freq, h_vis[k], nx, nx, px, px, 1e-5, dirty=out_d[k], **KW)
        ctx.dirty2ms(h_uvw, freq, h_mod[k], px, px, 1e-5, vis=out_v[k], **KW)
    ctx.synchronize()
    for k in range(n):
        assert O.rel_rms(out_d[k].numpy(), want_d[k]) < 1e-6
        assert O.rel_rms(out_v[k].numpy(), want_v[k]) < 1e-6
    # device tensors produced on torch's stream, consumed in pipelined calls
    tu = torch.as_tensor(uvw, device="cuda")
    dv = torch.as_tensor(vis[0], device="cuda") * 2.0
    d = ctx.ms2dirty(tu, freq, dv, nx, nx, px, px, 1e-5, **KW)
    ctx.synchronize()
    assert O.rel_rms(d.cpu().numpy(), 2 * want_d[0]) < 1e-6
    ctx.set_async(False)
    d2 = ctx.ms2dirty(uvw, freq, vis[1], nx, nx, px, px, 1e-5, **KW)
    assert O.rel_rms(d2, want_d[1]) < 1e-6
