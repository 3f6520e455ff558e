"""Streaming into a resident grid (wsg_stream_*): chunks of rows added
from pageable host memory, page-locked host memory and the device, gridded
into one w-stack and transformed once, against the single-call operators on
the same data (the same declared extent gives the same grid, so they agree
to FP32 rounding: the grid sums the chunks in a different order) and the
FP64 DFT; prediction chunk by chunk; and rejection of
a chunk outside the declared extent.  Geometry: the config-5 wide field
(8192^2 at 2", |w| up to 40% of max|uv|) on a 2% time subsample."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


@pytest.fixture(scope="module")
def cfg5():
    from wsclean_b200 import synth
    c = synth.config5(scale=0.02)
    rng = np.random.default_rng(55)
    vis = (rng.normal(size=(len(c["uvw"]), len(c["freq"])))
           + 1j * rng.normal(size=(len(c["uvw"]), len(c["freq"])))).astype(np.complex64)
    return c, vis


def chunks(n, k):
    b = np.linspace(0, n, k + 1).astype(int)
    return list(zip(b[:-1], b[1:]))


def test_stream_matches_single_call_and_dft(cfg5):
    from wsclean_b200 import gridder as G
    c, vis = cfg5
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    ext = G.data_extent(uvw, freq)
    with G.Stream(freq, nx, nx, px, px, 1e-5, ext, nvis=vis.size, dirty_dtype=np.float64,
                  **KW) as s:
        parts = chunks(len(uvw), 7)
        for i, (a, b) in enumerate(parts):
            if i % 3 == 0:     # pageable numpy
                s.add(uvw[a:b], vis[a:b])
            elif i % 3 == 1:   # page-locked torch CPU tensors
                s.add(torch.as_tensor(uvw[a:b]).pin_memory(), torch.as_tensor(vis[a:b]).pin_memory())
            else:              # device
                s.add(torch.as_tensor(uvw[a:b], device="cuda"), torch.as_tensor(vis[a:b], device="cuda"))
        d = s.finish()
        st = s.stats()
    ref = G.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, dirty_dtype=np.float64, **KW)
    assert O.rel_rms(d, ref) < 5e-6
    rng = np.random.default_rng(1)
    pix = rng.integers(0, nx * nx, 48)
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, pixels=pix, negate_v=True,
                         divide_by_n=False)
    assert O.rel_rms(d.ravel()[pix], dft) < 1e-5
    assert st["nu"] > 0 and st["nplanes"] > 1


def test_stream_prediction_matches_single_call(cfg5):
    from wsclean_b200 import gridder as G
    from wsclean_b200 import synth
    c, vis = cfg5
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(2)
    ix, iy, flux = synth.point_sky(300, nx, nx, rng)
    model = synth.sky_image(nx, nx, ix, iy, flux).astype(np.float32)
    ext = G.data_extent(uvw, freq)
    with G.Stream(freq, nx, nx, px, px, 1e-5, ext, nvis=vis.size, **KW) as s:
        s.predict_begin(model)
        out = np.concatenate([s.predict(uvw[a:b]) for a, b in chunks(len(uvw), 5)])
    ref = G.dirty2ms(uvw, freq, model, px, px, 1e-5, **KW)
    assert O.rel_rms(out, ref) < 1e-6
    sel = rng.choice(out.size, 5000, replace=False)
    dft = O.dft_dirty2ms(uvw, freq, model.astype(np.float64), px, px, negate_v=True,
                         divide_by_n=False, select=sel)
    assert O.rel_rms(out.ravel()[sel], dft) < 1e-5


def test_stream_fp64_weights_and_mask():
    from wsclean_b200 import gridder as G
    rng = np.random.default_rng(3)
    nrow, nchan, nx = 5000, 4, 96
    px = np.deg2rad(30 / 3600)
    freq = np.linspace(1.4e8, 1.6e8, nchan)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([800.0, 800.0, 250.0])
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    wgt = rng.uniform(0.5, 2, (nrow, nchan))
    mask = (rng.uniform(size=(nrow, nchan)) > 0.2).astype(np.uint8)
    ext = G.data_extent(uvw, freq)
    with G.Stream(freq, nx, nx, px, px, 1e-11, ext, nvis=vis.size, precision="fp64",
                  vis_dtype=np.complex128, wgt_dtype=np.float64, **KW) as s:
        for a, b in chunks(nrow, 4):
            s.add(uvw[a:b], vis[a:b], wgt=wgt[a:b], mask=mask[a:b])
        d = s.finish()
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, wgt=wgt, mask=mask, negate_v=True,
                         divide_by_n=False)
    assert O.rel_rms(d, dft) < 1e-10


def test_stream_rejects_chunk_outside_extent():
    from wsclean_b200 import gridder as G
    from wsclean_b200 import _lib as L
    rng = np.random.default_rng(4)
    freq = np.array([1.5e8])
    uvw = rng.uniform(-1, 1, (1000, 3)) * np.array([800.0, 800.0, 250.0])
    vis = np.ones((1000, 1), np.complex64)
    px = np.deg2rad(30 / 3600)
    ext = G.data_extent(uvw[:500], freq)
    wide = uvw[500:].copy()
    wide[:, 2] *= 3.0
    with G.Stream(freq, 64, 64, px, px, 1e-5, ext, **KW) as s:
        s.add(uvw[:500], vis[:500])
        # the rows are checked when their batch is sorted: at the latest by finish()
        with pytest.raises(L.InvalidArgument):
            s.add(wide, vis[500:])
            s.finish()


def test_stream_predict_then_grid(cfg5):
    """A major cycle on one stream: predict the model, then grid the
    predicted visibilities (the first add after a prediction clears the
    grid); the image equals the single-call ms2dirty of the same data."""
    from wsclean_b200 import gridder as G
    from wsclean_b200 import synth
    c, _ = cfg5
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(6)
    ix, iy, flux = synth.point_sky(50, nx, nx, rng)
    model = synth.sky_image(nx, nx, ix, iy, flux)
    ext = G.data_extent(uvw, freq)
    parts = chunks(len(uvw), 3)
    with G.Stream(freq, nx, nx, px, px, 1e-5, ext, dirty_dtype=np.float64, **KW) as s:
        s.predict_begin(model)
        vis = np.concatenate([s.predict(uvw[a:b]) for a, b in parts])
        for a, b in parts:
            s.add(uvw[a:b], vis[a:b])
        d = s.finish()
    ref = G.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, dirty_dtype=np.float64, **KW)
    assert O.rel_rms(d, ref) < 5e-6


def test_stream_pipelined_prediction(cfg5):
    """With the context pipelined (wsg_ctx_set_async), predictions into
    page-locked memory return once enqueued, are copied back while the next
    chunk is computed, and are in place after synchronize(): they equal the
    chunk-by-chunk synchronous predictions."""
    from wsclean_b200 import gridder as G
    from wsclean_b200 import synth
    c, _ = cfg5
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(7)
    ix, iy, flux = synth.point_sky(100, nx, nx, rng)
    model = synth.sky_image(nx, nx, ix, iy, flux).astype(np.float32)
    ext = G.data_extent(uvw, freq)
    parts = chunks(len(uvw), 6)
    ctx = G.Context(0)
    try:
        with G.Stream(freq, nx, nx, px, px, 1e-5, ext, context=ctx, **KW) as s:
            s.predict_begin(model)
            ref = np.concatenate([s.predict(uvw[a:b]) for a, b in parts])
            h_uvw = torch.as_tensor(uvw).pin_memory()
            out = torch.zeros((len(uvw), len(freq)), dtype=torch.complex64).pin_memory()
            ctx.set_async(True)
            s.predict_begin(model)
            for a, b in parts:
                s.predict(h_uvw[a:b], vis=out[a:b])
            ctx.synchronize()
            ctx.set_async(False)
    finally:
        ctx.close()
    assert O.rel_rms(out.numpy(), ref) < 1e-7


def test_stream_in_plane_passes(monkeypatch):
    """A stream whose w planes do not all fit its transformed-row buffer
    (here capped at three planes a pass, as memory pressure would) transforms
    the planes in passes; with several twisted passes a row is longer than
    the image, which the pass count must allow for.  The image and the
    predictions equal the single calls'."""
    from wsclean_b200 import gridder as G
    monkeypatch.setenv("WSG_MAX_PLANES", "3")
    rng = np.random.default_rng(8)
    nrow, nx, ny = 6000, 256, 200
    freq = np.array([1.40e8, 1.45e8])
    px = np.deg2rad(20 / 3600)
    umax = 0.1 / px * 299792458.0 / freq.max()
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([umax, umax, 0.6 * umax])
    vis = (rng.normal(size=(nrow, 2)) + 1j * rng.normal(size=(nrow, 2))).astype(np.complex64)
    ext = G.data_extent(uvw, freq)
    parts = chunks(nrow, 4)
    with G.Stream(freq, nx, ny, px, px, 1e-5, ext, nvis=vis.size, dirty_dtype=np.float64,
                  **KW) as s:
        for a, b in parts:
            s.add(uvw[a:b], vis[a:b])
        d = s.finish()
        st = s.stats()
        assert st["nplanes"] > 3 and 2 * st["band_rows"] <= st["nu"]
        model = np.zeros((nx, ny), np.float32)
        model[rng.integers(0, nx, 20), rng.integers(0, ny, 20)] = 1.0
        s.predict_begin(model)
        v = np.concatenate([s.predict(uvw[a:b]) for a, b in parts])
    ref = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-5, dirty_dtype=np.float64, **KW)
    assert O.rel_rms(d, ref) < 5e-6
    vref = G.dirty2ms(uvw, freq, model, px, px, 1e-5, **KW)
    assert O.rel_rms(v, vref) < 1e-6


def test_stream_fp64_long_transforms_in_plane_passes(monkeypatch):
    """FP64 with a u band wider than 4096 rows (8192-point column transforms,
    two twisted passes) through a stream whose planes are transformed three at
    a time: image and predictions equal the single FP64 calls'."""
    from wsclean_b200 import gridder as G
    monkeypatch.setenv("WSG_MAX_PLANES", "3")
    rng = np.random.default_rng(9)
    nrow, nx, ny = 4000, 6000, 32
    freq = np.array([1.40e8, 1.45e8])
    px = np.deg2rad(10 / 3600)
    umax = 0.2 / px * 299792458.0 / freq.max()
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([umax, umax, 0.2 * umax])
    vis = rng.normal(size=(nrow, 2)) + 1j * rng.normal(size=(nrow, 2))
    ext = G.data_extent(uvw, freq)
    parts = chunks(nrow, 3)
    kw = dict(KW, sigma_min=1.5)
    with G.Stream(freq, nx, ny, px, px, 1e-12, ext, nvis=vis.size, precision="fp64",
                  vis_dtype=np.complex128, dirty_dtype=np.float64, **kw) as s:
        for a, b in parts:
            s.add(uvw[a:b], vis[a:b])
        d = s.finish()
        st = s.stats()
        assert st["nplanes"] > 3 and st["nu"] == 16384 and st["band_rows"] > 4096
        model = np.zeros((nx, ny))
        model[rng.integers(0, nx, 20), rng.integers(0, ny, 20)] = 1.0
        s.predict_begin(model)
        v = np.concatenate([s.predict(uvw[a:b]) for a, b in parts])
    ref = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                     dirty_dtype=np.float64, **kw)
    assert O.rel_rms(d, ref) < 1e-12
    vref = G.dirty2ms(uvw, freq, model, px, px, 1e-12, precision="fp64",
                      vis_dtype=np.complex128, **kw)
    assert O.rel_rms(v, vref) < 1e-12


def test_stream_band_wider_than_the_pruned_transform(monkeypatch):
    """A u band wider than the longest pruned column transform (the full-grid
    layout, u transform by the library FFT) through a stream, five planes a
    pass: image and predictions equal the single calls'."""
    from wsclean_b200 import gridder as G
    monkeypatch.setenv("WSG_MAX_PLANES", "5")
    rng = np.random.default_rng(10)
    nrow, nx, ny = 4000, 6000, 32
    freq = np.array([1.40e8, 1.45e8])
    px = np.deg2rad(10 / 3600)
    umax = 0.45 / px * 299792458.0 / freq.max()
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([umax, umax, 0.2 * umax])
    vis = (rng.normal(size=(nrow, 2)) + 1j * rng.normal(size=(nrow, 2))).astype(np.complex64)
    ext = G.data_extent(uvw, freq)
    parts = chunks(nrow, 3)
    kw = dict(KW, sigma_min=1.5)
    with G.Stream(freq, nx, ny, px, px, 1e-5, ext, nvis=vis.size, dirty_dtype=np.float64,
                  **kw) as s:
        for a, b in parts:
            s.add(uvw[a:b], vis[a:b])
        d = s.finish()
        st = s.stats()
        assert st["band_rows"] == st["nu"] > 8192 and st["nplanes"] > 5
        model = np.zeros((nx, ny), np.float32)
        model[rng.integers(0, nx, 20), rng.integers(0, ny, 20)] = 1.0
        s.predict_begin(model)
        v = np.concatenate([s.predict(uvw[a:b]) for a, b in parts])
    ref = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-5, dirty_dtype=np.float64, **kw)
    assert O.rel_rms(d, ref) < 5e-6
    vref = G.dirty2ms(uvw, freq, model, px, px, 1e-5, **kw)
    assert O.rel_rms(v, vref) < 1e-6
