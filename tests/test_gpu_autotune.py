"""The autotuner (wsg_autotune): it times the cheapest kernel / tile
candidates on the data, stores the winner, later calls with the same image
size, precision and accuracy use it, and the results still meet epsilon
against the FP64 DFT."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


def test_autotune_choice_is_used_and_accurate():
    from wsclean_b200 import gridder as G
    from wsclean_b200 import synth
    c = synth.config2(scale=0.1, npix=1024, pixsize_arcsec=20.0)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(6)
    vis = (rng.normal(size=(len(uvw), 1)) + 1j * rng.normal(size=(len(uvw), 1))).astype(np.complex64)
    ctx = G.Context(0)
    best = ctx.autotune(uvw, freq, vis, nx, nx, px, px, 1e-5, candidates=3, **KW)
    assert best["supp"] >= 4 and best["ms_total"] > 0 and best["kernel_err"] <= 1e-5
    # a later call of the same geometry uses the tuned kernel and grid
    d = ctx.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, dirty_dtype=np.float64, **KW)
    st = ctx.stats()
    assert (st["supp"], st["nu"], st["nv"], st["nplanes"]) == (best["supp"], best["nu"],
                                                               best["nv"], best["nplanes"])
    pix = rng.integers(0, nx * nx, 64)
    dft = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, pixels=pix, negate_v=True,
                         divide_by_n=False)
    assert O.rel_rms(d.ravel()[pix], dft) < 1e-5
    # another context of the same process shares the table
    ctx2 = G.Context(0)
    ctx2.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, **KW)
    assert ctx2.stats()["supp"] == best["supp"]
