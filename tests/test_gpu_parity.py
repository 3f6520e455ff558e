"""GPU parity: the sm_100a path against the committed golden fixtures (made
with the reference's own w-gridder) and the FP64 direct Fourier transform.

Tolerances (relative RMS): mixed precision at epsilon 1e-5 must be within
1e-5 of the DFT; FP64 within 10*epsilon (floor 1e-12) of the DFT; against the
reference, the sum of both tolerances.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


def load(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    d["prec"] = str(d["prec"])
    d["eps"] = float(d["eps"])
    return d


def tol_of(eps, prec):
    return 1e-5 if prec == "float" else max(10 * eps, 1e-12)


@pytest.fixture(scope="module")
def G():
    from wsclean_b200 import gridder
    return gridder


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_golden_ms2dirty(G, path):
    g = load(path)
    nx, ny = g["npix"]
    px, py = g["pixsize"]
    cx, cy = g["center"]
    prec = "mixed" if g["prec"] == "float" else "fp64"
    d = G.ms2dirty(g["uvw"], g["freq"], g["vis"], nx, ny, px, py, g["eps"], wgt=g["wgt"],
                   mask=g["mask"], center_x=cx, center_y=cy, precision=prec, **KW)
    tol = tol_of(g["eps"], g["prec"])
    e_dft = O.rel_rms(d, g["dirty_dft"])
    e_ref = O.rel_rms(d, g["dirty_ref"])
    assert e_dft < tol, e_dft
    assert e_ref < 2 * tol, e_ref


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_golden_dirty2ms(G, path):
    g = load(path)
    px, py = g["pixsize"]
    cx, cy = g["center"]
    prec = "mixed" if g["prec"] == "float" else "fp64"
    vdt = np.complex64 if prec == "mixed" else np.complex128
    model = g["model"].astype(np.float32 if prec == "mixed" else np.float64)
    v = G.dirty2ms(g["uvw"], g["freq"], model, px, py, g["eps"], wgt=g["wgt"], mask=g["mask"],
                   center_x=cx, center_y=cy, precision=prec, vis_dtype=vdt, **KW)
    tol = tol_of(g["eps"], g["prec"])
    assert O.rel_rms(v, g["vis_dft"]) < tol
    assert O.rel_rms(v, g["vis_ref"]) < 2 * tol
    # flagged visibilities are written as zero (ducc0 scanData, wgridder.h:1606-1607)
    assert np.all(v[g["mask"] == 0] == 0)


def random_problem(seed, nrow=3000, nchan=2, nx=64, ny=64, pixas=30.0, wscale=200.0):
    rng = np.random.default_rng(seed)
    px = np.deg2rad(pixas / 3600)
    freq = np.linspace(1.4e8, 1.5e8, nchan)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([800.0, 800.0, wscale])
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    return rng, uvw, freq, vis, nx, ny, px


@pytest.mark.parametrize("prec,eps", [("mixed", 1e-5), ("mixed", 1e-3), ("fp64", 1e-12),
                                      ("fp64", 1e-7)])
@pytest.mark.parametrize("opts", [dict(), dict(negate_v=False, divide_by_n=True),
                                  dict(do_wgridding=False), dict(center_x=4.0, center_y=-3.0)])
def test_variants_vs_dft(G, prec, eps, opts):
    rng, uvw, freq, vis, nx, ny, px = random_problem(7, ny=48)
    o = dict(KW)
    o.update({k: v for k, v in opts.items() if k not in ("center_x", "center_y")})
    cx, cy = opts.get("center_x", 0.0) * px, opts.get("center_y", 0.0) * px
    if o.get("do_wgridding", True) is False:
        uvw = uvw.copy()
        uvw[:, 2] = 0.0   # without w-gridding the DFT is exact only for w=0
    d = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec, center_x=cx,
                   center_y=cy, dirty_dtype=np.float64, **o)
    ref = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, negate_v=o["negate_v"],
                         divide_by_n=o["divide_by_n"] and o.get("do_wgridding", True),
                         center_x=cx, center_y=cy)
    tol = max(eps, 1e-12) * 10 if prec == "fp64" else max(eps, 1e-5)
    assert O.rel_rms(d, ref) < tol
    model = np.zeros((nx, ny))
    model[rng.integers(0, nx, 8), rng.integers(0, ny, 8)] = rng.normal(size=8)
    v = G.dirty2ms(uvw, freq, model, px, px, eps, precision=prec, center_x=cx, center_y=cy,
                   vis_dtype=np.complex128, **o)
    vref = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=o["negate_v"],
                          divide_by_n=o["divide_by_n"] and o.get("do_wgridding", True),
                          center_x=cx, center_y=cy)
    assert O.rel_rms(v, vref) < tol


def test_device_and_host_inputs_agree(G):
    import torch
    rng, uvw, freq, vis, nx, ny, px = random_problem(8)
    dev = torch.device("cuda", 0)
    d_h = G.ms2dirty(uvw, freq, vis.astype(np.complex64), nx, ny, px, px, 1e-5, **KW)
    d_d = G.ms2dirty(torch.as_tensor(uvw, device=dev), torch.as_tensor(freq, device=dev),
                     torch.as_tensor(vis.astype(np.complex64), device=dev), nx, ny, px, px,
                     1e-5, **KW)
    assert d_d.is_cuda
    assert O.rel_rms(d_d.cpu().numpy(), d_h) < 1e-6


def test_accumulate(G):
    rng, uvw, freq, vis, nx, ny, px = random_problem(9)
    base = rng.normal(size=(nx, ny))
    d = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                   dirty_dtype=np.float64, **KW)
    acc = base.copy()
    G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64", dirty=acc,
               accumulate=True, **KW)
    assert np.allclose(acc, base + d, rtol=1e-12, atol=1e-10)


def test_all_flagged_and_single_visibility(G):
    rng, uvw, freq, vis, nx, ny, px = random_problem(10, nrow=50)
    mask = np.zeros(vis.shape, np.uint8)
    d = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-5, mask=mask, **KW)
    assert np.all(d == 0)
    v = G.dirty2ms(uvw, freq, rng.normal(size=(nx, ny)), px, px, 1e-5, mask=mask, **KW)
    assert np.all(v == 0)
    one = np.zeros(vis.shape, np.uint8)
    one[7, 1] = 1
    d1 = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, mask=one, precision="fp64",
                    dirty_dtype=np.float64, **KW)
    ref = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, mask=one, negate_v=True,
                         divide_by_n=False)
    assert O.rel_rms(d1, ref) < 1e-11


def test_zero_weight_visibilities_are_skipped(G):
    rng, uvw, freq, vis, nx, ny, px = random_problem(12)
    wgt = rng.uniform(0.5, 2.0, vis.shape)
    wgt[::3] = 0.0
    v = G.dirty2ms(uvw, freq, rng.normal(size=(nx, ny)), px, px, 1e-5, wgt=wgt, **KW)
    assert np.all(v[::3] == 0)


def test_plane_batching_matches_single_pass(G, monkeypatch):
    rng, uvw, freq, vis, nx, ny, px = random_problem(13, wscale=2000.0)
    model = rng.normal(size=(nx, ny))
    d1 = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                    dirty_dtype=np.float64, **KW)
    v1 = G.dirty2ms(uvw, freq, model, px, px, 1e-12, precision="fp64", vis_dtype=np.complex128, **KW)
    npl = G.default_context().stats()["nplanes"]
    assert npl > 4
    monkeypatch.setenv("WSG_MAX_PLANES", "3")
    d2 = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                    dirty_dtype=np.float64, **KW)
    assert G.default_context().stats()["plane_batch"] == 3
    v2 = G.dirty2ms(uvw, freq, model, px, px, 1e-12, precision="fp64", vis_dtype=np.complex128, **KW)
    assert O.rel_rms(d2, d1) < 1e-13
    assert O.rel_rms(v2, v1) < 1e-13


def test_full_band_grid(G):
    """uv coverage reaching the grid edge: no u-band pruning."""
    rng, uvw, freq, vis, nx, ny, px = random_problem(14, nrow=2000, pixas=400.0, wscale=50.0)
    d = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                   dirty_dtype=np.float64, **KW)
    assert G.default_context().stats()["band_rows"] == G.default_context().stats()["nu"]
    ref = O.dft_ms2dirty(uvw, freq, vis, nx, ny, px, px, negate_v=True, divide_by_n=False)
    assert O.rel_rms(d, ref) < 1e-11


@pytest.mark.parametrize("bad", ["odd", "freq_order", "freq_neg", "eps_mixed"])
def test_invalid_arguments_raise(G, bad):
    from wsclean_b200._lib import InvalidArgument
    rng, uvw, freq, vis, nx, ny, px = random_problem(15, nrow=20)
    eps, prec = 1e-5, "mixed"
    if bad == "odd":
        nx = 63
    elif bad == "freq_order":
        freq = freq[::-1].copy()
    elif bad == "freq_neg":
        freq = -freq
    elif bad == "eps_mixed":
        eps = 1e-9
    with pytest.raises(InvalidArgument):
        G.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec, **KW)


def test_degridding_is_deterministic(G):
    rng, uvw, freq, vis, nx, ny, px = random_problem(16)
    model = rng.normal(size=(nx, ny)).astype(np.float32)
    v1 = G.dirty2ms(uvw, freq, model, px, px, 1e-5, **KW)
    v2 = G.dirty2ms(uvw, freq, model, px, px, 1e-5, **KW)
    assert np.array_equal(v1, v2)
    d1 = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-5, **KW)
    d2 = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-5, **KW)
    assert O.rel_rms(d1, d2) < 1e-6


def test_config2_geometry_scaled(G):
    """The benchmark's Earth-rotation geometry at reduced size, against the
    DFT on 64 pixels and the reference on the whole image."""
    from wsclean_b200 import synth
    c = synth.config2(scale=0.04, npix=512, pixsize_arcsec=40.0)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(21)
    vis = (rng.normal(size=(len(uvw), 1)) + 1j * rng.normal(size=(len(uvw), 1))).astype(np.complex64)
    d = G.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, **KW)
    pix = rng.integers(0, nx * nx, 64)
    ref = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, negate_v=True, divide_by_n=False,
                         pixels=pix)
    assert O.rel_rms(d.ravel()[pix], ref) < 1e-5
    if O.ref_available():
        dr = O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, prec="float")
        assert O.rel_rms(d, dr) < 2e-5


def test_repeated_gridding_with_changing_uv_extent(G):
    """One context grids data sets whose v extents differ, in turn: each call
    clears exactly what the previous spread wrote, so the results equal those
    of a fresh context."""
    from wsclean_b200.gridder import Context
    ctx = Context(0)
    probs = []
    for seed, vscale in ((31, 800.0), (32, 200.0), (33, 500.0), (34, 800.0)):
        rng, uvw, freq, vis, nx, ny, px = random_problem(seed, nrow=2500)
        uvw = uvw.copy()
        uvw[:, 1] *= vscale / 800.0   # same u extent (same band layout), varying v extent
        probs.append((uvw, freq, vis, nx, ny, px))
    for rep in range(2):
        for uvw, freq, vis, nx, ny, px in probs:
            d = ctx.ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                             dirty_dtype=np.float64, **KW)
            fresh = Context(0).ms2dirty(uvw, freq, vis, nx, ny, px, px, 1e-12, precision="fp64",
                                        dirty_dtype=np.float64, **KW)
            assert O.rel_rms(d, fresh) < 1e-13
