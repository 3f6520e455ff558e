"""GPU imaging weights (wsg_weights_*) against the numpy restatement of
WSClean's ImageWeights (oracle/imageweights.py): identical cell selection
(the same zero pattern) and weights within 1e-12 relative (the GPU sums
with atomics, in a different order), for natural, uniform and Briggs
weighting, the weights-as-taper flag, a super-weight factor, several
polarisations and chunked gridding, on the config-3 geometry (config-2 array
at 2048^2, 8")."""
import numpy as np
import pytest
import torch

from oracle.imageweights import ImageWeights as Ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    from wsclean_b200 import synth
    c = synth.config3(scale=0.1)
    rng = np.random.default_rng(8)
    w = rng.uniform(0.5, 2.0, (len(c["uvw"]), len(c["freq"]))).astype(np.float32)
    w[rng.uniform(size=w.shape) < 0.05] = 0.0
    return c, w


@pytest.mark.parametrize("mode,robust,taper,sw", [
    ("natural", 0.0, False, 1.0), ("uniform", 0.0, False, 1.0), ("briggs", 0.0, False, 1.0),
    ("briggs", -1.0, False, 2.0), ("briggs", 2.0, True, 1.0), ("uniform", 0.0, True, 3.0)])
def test_weights_match_restatement(data, mode, robust, taper, sw):
    from wsclean_b200.gridder import ImageWeights
    c, w = data
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    m = {"natural": 0, "uniform": 1, "briggs": 2}[mode]
    ref = Ref(m, robust, nx, nx, px, px, taper, sw)
    half = len(uvw) // 2
    ref.grid_weights(uvw[:half], freq, w[:half])
    ref.grid_weights(uvw[half:], freq, w[half:])
    with ImageWeights(mode, robust, nx, nx, px, px, taper, sw) as iw:
        iw.grid(uvw[:half], freq, w[:half])
        iw.grid(torch.as_tensor(uvw[half:], device="cuda"), freq,
                torch.as_tensor(w[half:], device="cuda"))
        g, tot = iw.grid_array()
        assert g.shape == (ref.H // 2, ref.W)
        assert abs(tot - ref.total) <= 1e-12 * ref.total
        np.testing.assert_allclose(g.ravel(), ref.grid, rtol=1e-12, atol=0)
        iw.finish()
        ref.finish()
        g, _ = iw.grid_array()
        np.testing.assert_allclose(g.ravel(), ref.grid, rtol=1e-12, atol=0)
        out = iw.apply(uvw, freq, w)
    want = ref.apply(uvw, freq, w)[..., 0]
    assert np.array_equal(out == 0, want == 0)
    np.testing.assert_allclose(out, want, rtol=1e-6, atol=0)


def test_weights_polarisations_and_briggs_into_gridding(data):
    from wsclean_b200 import gridder as G
    from wsclean_b200 import synth
    import oracle as O
    c, w = data
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    w2 = np.stack([w, 0.5 * w], axis=-1)
    ref = Ref(2, 0.5, nx, nx, px, px)
    ref.grid_weights(uvw, freq, w2, npol=2)
    ref.finish()
    with G.ImageWeights("briggs", 0.5, nx, nx, px, px) as iw:
        iw.grid(uvw, freq, w2, npol=2)
        iw.finish()
        out = iw.apply(uvw, freq, w2, npol=2)
        np.testing.assert_allclose(out, ref.apply(uvw, freq, w2, npol=2), rtol=1e-6, atol=0)
        # the imaging weights feed the gridder as its weight array
        wi = iw.apply(uvw, freq, w)
    rng = np.random.default_rng(3)
    vis = (rng.normal(size=w.shape) + 1j * rng.normal(size=w.shape)).astype(np.complex64)
    d = G.ms2dirty(uvw, freq, vis, 256, 256, 4 * px, 4 * px, 1e-5, wgt=wi, negate_v=True,
                   divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
    pix = rng.integers(0, 256 * 256, 32)
    dft = O.dft_ms2dirty(uvw, freq, vis, 256, 256, 4 * px, 4 * px, wgt=wi.astype(np.float64),
                         pixels=pix, negate_v=True, divide_by_n=False)
    assert O.rel_rms(d.ravel()[pix], dft) < 1e-5


def test_stream_fuses_imaging_weights(data):
    """A stream with imaging weights set grids every visibility with weight x
    imaging weight looked up on the device (the product WSClean's
    readAndWeightVisibilities forms, msgridderbase.cpp:583-590,640-659),
    equal to gridding the weights that wsg_weights_apply returns, and to the
    FP64 DFT with those weights; cells outside the weight grid (a weight grid
    of a quarter of the image's extent in uv) drop their visibilities."""
    from wsclean_b200 import gridder as G
    from wsclean_b200.gridder import ImageWeights
    import oracle as O
    c, w = data
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    kw = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
    rng = np.random.default_rng(9)
    vis = (rng.normal(size=w.shape) + 1j * rng.normal(size=w.shape)).astype(np.complex64)
    ext = G.data_extent(uvw, freq)
    parts = [(0, len(uvw) // 3), (len(uvw) // 3, len(uvw))]
    for scale in (1.0, 0.25):   # 0.25: a coarser weight grid that misses the outer uv cells
        with ImageWeights("briggs", 0.0, nx, nx, px / scale, px / scale) as iw:
            iw.grid(uvw, freq, w)
            iw.finish()
            weff = iw.apply(uvw, freq, w)
            with G.Stream(freq, nx, nx, px, px, 1e-5, ext, nvis=vis.size, dirty_dtype=np.float64,
                          **kw) as s:
                s.set_imaging_weights(iw)
                for a, b in parts:
                    s.add(uvw[a:b], vis[a:b], wgt=w[a:b])
                fused = s.finish()
            with G.Stream(freq, nx, nx, px, px, 1e-5, ext, nvis=vis.size, dirty_dtype=np.float64,
                          **kw) as s:
                for a, b in parts:
                    s.add(uvw[a:b], vis[a:b], wgt=weff[a:b])
                unfused = s.finish()
        if scale < 1.0:
            assert (weff == 0).sum() > (w == 0).sum()   # some cells fell outside
        assert O.rel_rms(fused, unfused) < 1e-6
        pix = rng.integers(0, nx * nx, 32)
        dft = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, wgt=weff.astype(np.float64),
                             pixels=pix, negate_v=True, divide_by_n=False)
        assert O.rel_rms(fused.ravel()[pix], dft) < 1e-5
