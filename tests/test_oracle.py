"""The CPU checkers, pinned against the reference's own outputs.

The reference ships no golden vectors for this path, so the pins are the
fixtures in tests/golden/ (made by tests/golden/make_golden.py from the
compiled reference) and, where oracle/_ref is built, fresh reference runs.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    d["prec"] = str(d["prec"])
    d["eps"] = float(d["eps"])
    return d


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_dft_reproduces_fixture(path):
    g = load(path)
    nx, ny = g["npix"]
    px, py = g["pixsize"]
    cx, cy = g["center"]
    d = O.dft_ms2dirty(g["uvw"], g["freq"], g["vis"], nx, ny, px, py, wgt=g["wgt"],
                       mask=g["mask"], negate_v=True, divide_by_n=False, center_x=cx, center_y=cy)
    assert O.rel_rms(d, g["dirty_dft"]) < 1e-13
    v = O.dft_dirty2ms(g["uvw"], g["freq"], g["model"], px, py, wgt=g["wgt"], mask=g["mask"],
                       negate_v=True, divide_by_n=False, center_x=cx, center_y=cy)
    assert O.rel_rms(v, g["vis_dft"]) < 1e-13


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_reference_agrees_with_dft(path):
    """The pin: the reference w-gridder's own output is within its epsilon of
    the FP64 DFT, both directions, incl. weights, flags and phase-centre shifts."""
    g = load(path)
    tol = max(g["eps"], 1e-12)
    assert O.rel_rms(g["dirty_ref"], g["dirty_dft"]) < tol
    assert O.rel_rms(g["vis_ref"], g["vis_dft"]) < tol


def test_dft_adjoint():
    rng = np.random.default_rng(3)
    nrow, nchan, nx, ny = 300, 2, 24, 20
    px = py = np.deg2rad(60 / 3600)
    freq = np.array([1.2e8, 1.3e8])
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([500, 500, 200])
    x = rng.normal(size=(nx, ny))
    y = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    Ax = O.dft_dirty2ms(uvw, freq, x, px, py, center_x=2 * px, center_y=-py)
    Aty = O.dft_ms2dirty(uvw, freq, y, nx, ny, px, py, center_x=2 * px, center_y=-py)
    a = np.vdot(y, Ax).real
    b = np.vdot(Aty, x).real
    assert abs(a - b) <= 1e-12 * np.linalg.norm(y) * np.linalg.norm(Ax)


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
def test_reference_rerun_matches_fixture():
    g = load(GOLDEN[0])
    nx, ny = g["npix"]
    px, py = g["pixsize"]
    cx, cy = g["center"]
    d = O.ref_ms2dirty(g["uvw"], g["freq"], g["vis"], nx, ny, px, py, g["eps"], wgt=g["wgt"],
                       mask=g["mask"], prec=g["prec"], negate_v=True, divide_by_n=False,
                       sigma_min=1.1, sigma_max=2.0, center_x=cx, center_y=cy, nthreads=2)
    # thread count changes only the summation order
    assert O.rel_rms(d, g["dirty_ref"]) < 1e-6


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
def test_reference_report_parses():
    g = load(GOLDEN[1])
    nx, ny = g["npix"]
    px, py = g["pixsize"]
    _, rep = O.ref_ms2dirty(g["uvw"], g["freq"], g["vis"], nx, ny, px, py, g["eps"],
                            prec=g["prec"], nthreads=1, return_report=True)
    r = O.parse_report(rep)
    assert r and r[0]["nu"] >= nx and r[0]["supp"] >= 4


def test_imageweights_restatement_matches_briggs_helper():
    """The oracle's ImageWeights and the synthetic-data Briggs helper are two
    restatements of imageweights.cpp:113-143; they must agree."""
    from oracle.imageweights import ImageWeights
    from wsclean_b200 import synth
    c = synth.config3(scale=0.02)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(1)
    noise = rng.uniform(0.5, 2.0, (len(uvw), len(freq)))
    ref = ImageWeights(ImageWeights.BRIGGS, 0.0, nx, nx, px, px)
    ref.grid_weights(uvw, freq, noise.astype(np.float32))
    ref.finish()
    iw = ref.apply(uvw, freq)[..., 0]
    helper = synth.briggs_weights(uvw, freq, nx, nx, px, px, robust=0.0,
                                  noise_weights=noise.astype(np.float32))
    np.testing.assert_allclose(iw, helper, rtol=1e-6)


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
def test_recorded_reference_grids_config2():
    """The benchmark's roofline charges the grid the reference chooses for
    the headline workload, recorded in tests/golden/ducc_grids.json by
    tests/golden/make_ducc_grids.py: the reference chooses it again here."""
    import json
    import os
    from wsclean_b200 import synth
    rec = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ducc_grids.json")))
    c = synth.config2()
    rng = np.random.default_rng(2)
    v = (rng.normal(size=(len(c["uvw"]), 1)) + 1j * rng.normal(size=(len(c["uvw"]), 1)))
    kw = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0, return_report=True)
    for form, prec, eps, dt in (("mixed", "float", 1e-5, np.complex64),
                                ("fp64", "double", 1e-12, np.complex128)):
        _, rep = O.ref_ms2dirty(c["uvw"], c["freq"], v.astype(dt), c["npix_x"], c["npix_x"],
                                c["pixsize"], c["pixsize"], eps, prec=prec, **kw)
        g = O.parse_report(rep)[0]
        r = rec["config2"][form]
        assert (g["nu"], g["nv"], g["nplanes"], g["supp"]) == (r["nu"], r["nv"], r["nplanes"],
                                                             r["supp"]), form
