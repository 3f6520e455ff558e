"""The WGriddingGridder_Simple replacement through the C ABI: chunked
inversion, normalisation, untrimming with NaN borders, and prediction."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def setup(seed=2):
    rng = np.random.default_rng(seed)
    nrow, nchan = 3000, 2
    freq = np.array([1.45e8, 1.5e8])
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([700.0, 700.0, 200.0])
    vis = (rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))).astype(np.complex64)
    return rng, uvw, freq, vis


@pytest.mark.parametrize("precision,eps", [("mixed", 1e-4), ("fp64", 1e-8)])
def test_inversion_and_prediction(precision, eps):
    from wsclean_b200.gridder import WGriddingGridder
    rng, uvw, freq, vis = setup()
    width, height, wt, ht = 80, 72, 64, 56
    px = np.deg2rad(30 / 3600)
    lsh, msh = 2 * px, -3 * px
    g = WGriddingGridder(width, height, wt, ht, px, px, lsh, msh, 4, eps, 0, False, precision)
    g.InitializeInversion()
    g.AddInversionData(uvw[:1700], freq, vis[:1700])
    g.AddInversionData(uvw[1700:], freq, vis[1700:])
    g.FinalizeImage(0.5)
    img = g.RealImage()
    assert img.shape == (height, width)
    dx, dy = (width - wt) // 2, (height - ht) // 2
    inner = img[dy:dy + ht, dx:dx + wt]
    assert np.isfinite(inner).all()
    assert np.isnan(img[:dy]).all() and np.isnan(img[:, :dx]).all()
    # WSClean's call: negate_v, no divide_by_n, center = -shift; image x-major inside
    ref = 0.5 * O.dft_ms2dirty(uvw, freq, vis, wt, ht, px, px, negate_v=True, divide_by_n=False,
                               center_x=-lsh, center_y=-msh)
    tol = 1e-5 if precision == "mixed" else 1e-7
    assert O.rel_rms(inner.T, ref) < max(tol, eps) * 10
    # prediction from the untrimmed float image
    model = np.full((height, width), np.nan, np.float32)
    sky = np.zeros((wt, ht))
    sky[rng.integers(0, wt, 6), rng.integers(0, ht, 6)] = 1.0
    model[dy:dy + ht, dx:dx + wt] = sky.T
    g.InitializePrediction(model)
    v = g.PredictVisibilities(uvw, freq)
    vref = O.dft_dirty2ms(uvw, freq, sky, px, px, negate_v=True, divide_by_n=False,
                          center_x=-lsh, center_y=-msh)
    assert O.rel_rms(v, vref) < max(tol, eps) * 10
    c, pv = g.MemoryUsage()
    assert c >= wt * ht * 8 and pv > 0
    st = g.stats()
    assert st["nvis"] == uvw.shape[0] * 2 and st["kernel_launches"] > 0
    g.close()


def test_gridder_rejects_bad_state():
    from wsclean_b200.gridder import WGriddingGridder
    from wsclean_b200._lib import WsgError
    rng, uvw, freq, vis = setup()
    px = np.deg2rad(30 / 3600)
    g = WGriddingGridder(64, 64, 64, 64, px, px, 0.0, 0.0)
    with pytest.raises(WsgError):
        g.AddInversionData(uvw, freq, vis)  # before InitializeInversion
    with pytest.raises(WsgError):
        WGriddingGridder(64, 64, 63, 64, px, px, 0.0, 0.0)  # odd trimmed size
    g.close()
