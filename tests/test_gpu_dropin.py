"""The C++ WGriddingGridderBase adapter (wsclean_b200/host), driven by a
compiled program the way WSClean's WGriddingMSGridder drives its gridder:
chunked AddInversionData, FinalizeImage, RealImage (x + y*width, NaN border),
InitializePrediction + chunked PredictVisibilities, and std::runtime_error on
invalid arguments."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "wsclean_b200", "host", "dropin_demo")


@pytest.mark.gpu
@pytest.mark.parametrize("eps", [1e-4, 1e-6])
def test_cpp_dropin_inversion_and_prediction(tmp_path, eps):
    assert os.path.exists(DEMO), "build with make -C wsclean_b200/csrc demo"
    rng = np.random.default_rng(31)
    nrows, nchan, width, height, wt, ht = 2500, 3, 100, 84, 80, 64
    px = np.deg2rad(25 / 3600)
    lsh, msh = 1.5 * px, -2.5 * px
    uvw = rng.uniform(-1, 1, (nrows, 3)) * np.array([800.0, 800.0, 250.0])
    freq = np.array([1.30e8, 1.35e8, 1.40e8])
    vis = (rng.normal(size=(nrows, nchan)) + 1j * rng.normal(size=(nrows, nchan))).astype(np.complex64)
    sky = np.zeros((wt, ht))
    sky[rng.integers(0, wt, 7), rng.integers(0, ht, 7)] = 1.0
    dx, dy = (width - wt) // 2, (height - ht) // 2
    model = np.zeros((height, width), np.float32)
    model[dy:dy + ht, dx:dx + wt] = sky.T
    hdr = np.array([nrows, nchan, width, height, wt, ht, px, eps, lsh, msh], np.float64)
    fin = tmp_path / "in.bin"
    with open(fin, "wb") as f:
        for arr in (hdr, uvw, freq, vis, model):
            f.write(np.ascontiguousarray(arr).tobytes())
    fimg, fvis = tmp_path / "img.bin", tmp_path / "vis.bin"
    r = subprocess.run([DEMO, str(fin), str(fimg), str(fvis)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    img = np.fromfile(fimg, np.float32).reshape(height, width)
    pred = np.fromfile(fvis, np.complex64).reshape(nrows, nchan)
    inner = img[dy:dy + ht, dx:dx + wt]
    assert np.isnan(img[:dy]).all() and np.isfinite(inner).all()
    ref = 0.5 * O.dft_ms2dirty(uvw, freq, vis, wt, ht, px, px, negate_v=True, divide_by_n=False,
                               center_x=-lsh, center_y=-msh)
    # the accuracy request itself; eps <= 1.01e-5 selects the FP64 instance
    # (as WSClean does), whose float image output is still exact to ~1e-7
    tol = eps
    assert O.rel_rms(inner.T, ref) < tol
    vref = O.dft_dirty2ms(uvw, freq, sky, px, px, negate_v=True, divide_by_n=False,
                          center_x=-lsh, center_y=-msh)
    assert O.rel_rms(pred, vref) < tol
