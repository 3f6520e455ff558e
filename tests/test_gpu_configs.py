"""Parity on the geometries of the four other benchmark configurations (the
headline bench runs config 2):

* config 2 at full size (the headline workload): 8.1M visibilities, 4096^2
  at 5", both directions in mixed precision (epsilon 1e-5) and in FP64
  (epsilon 1e-12) against the reference w-gridder over the whole image and
  all visibilities, against the FP64 DFT on 64 pixels and 10k visibilities,
  and the adjoint (dot-product) test;
* config 1 at full size: 2.9M complex128 visibilities, 1024^2 at 10",
  epsilon 1e-12, FP64 -- against the FP64 DFT and the reference w-gridder;
* config 3 at full size: the chi^2 gradient at 2048^2 / 8" with Briggs
  (robust 0) x U[0.5, 2] noise weights and a 5%-perturbed model, against
  central finite differences (h = 1e-3 Jy, 64 pixels, tolerance 1e-4) and
  the gradient computed with the reference w-gridder;
* config 4: facets of the seeded Voronoi tessellation (512^2 .. 2048^2 boxes,
  phase centre at the box centre) on output channels of 8 input channels,
  over a quarter of the observation;
* config 5: the 8192^2 / 2" wide-field geometry with |w| up to 40% of
  max|uv| on a 2% time subsample (10.4M visibilities), against the DFT on
  64 pixels and on a 20k-visibility subsample; and at full size (522M
  visibilities) streamed from page-locked host memory in 256 MiB chunks,
  predicted from the sky model (2000 point sources and 5 Gaussians) and
  gridded back, against the DFT on 20k visibilities and on image pixels."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


@pytest.fixture(scope="module")
def G():
    from wsclean_b200 import gridder
    return gridder


@pytest.fixture(scope="module")
def config2_data():
    from wsclean_b200 import synth
    c = synth.config2()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(22)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    vis = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux, device="cuda:0")
    vis = vis + 0.1 * (rng.normal(size=vis.shape) + 1j * rng.normal(size=vis.shape))
    model = synth.sky_image(nx, nx, ix, iy, flux)
    return dict(uvw=uvw, freq=freq, nx=nx, px=px, vis=vis, model=model, rng=rng)


# (precision, epsilon, tolerance vs the reference at the same epsilon,
#  tolerance vs the DFT, adjoint tolerance)
CONFIG2_FORMS = [("mixed", 1e-5, 2e-5, 1e-5, 1e-6), ("fp64", 1e-12, 1e-11, 1e-11, 1e-12)]


@pytest.mark.parametrize("prec,eps,tol_ref,tol_dft,tol_adj", CONFIG2_FORMS)
def test_config2_full(G, config2_data, prec, eps, tol_ref, tol_dft, tol_adj):
    """The headline workload at full size, checked over the whole image and
    every visibility against the reference w-gridder called as WSClean calls
    it (wgriddinggridder_simple.cpp:56-58, :106-108), with the same epsilon
    and the instance of the same width (<float,float> for the mixed form)."""
    d2 = config2_data
    uvw, freq, nx, px, model = d2["uvw"], d2["freq"], d2["nx"], d2["px"], d2["model"]
    rng = np.random.default_rng(23)
    dev = torch.device("cuda", 0)
    cdt = np.complex64 if prec == "mixed" else np.complex128
    fdt = np.float32 if prec == "mixed" else np.float64
    vis = d2["vis"].astype(cdt)
    tu, tf = torch.as_tensor(uvw, device=dev), torch.as_tensor(freq, device=dev)
    tv = torch.as_tensor(vis, device=dev)
    d = G.ms2dirty(tu, tf, tv, nx, nx, px, px, eps, precision=prec, dirty_dtype=np.float64,
                   **KW).cpu().numpy()
    pix = rng.integers(0, nx * nx, 64)
    ref_pix = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, pixels=pix, negate_v=True,
                             divide_by_n=False)
    assert O.rel_rms(d.ravel()[pix], ref_pix) < tol_dft
    tm = torch.as_tensor(model.astype(fdt), device=dev)
    v = G.dirty2ms(tu, tf, tm, px, px, eps, precision=prec, vis_dtype=np.complex128,
                   **KW).cpu().numpy()
    sel = rng.choice(v.size, 10000, replace=False)
    vref_sel = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=True, divide_by_n=False,
                              select=sel)
    assert O.rel_rms(v.ravel()[sel], vref_sel) < tol_dft
    # adjointness on seeded random vectors: |<y, A x> - <A^H y, x>| / (|y| |A x|)
    g = torch.Generator(device="cpu").manual_seed(5)
    x = torch.randn((nx, nx), generator=g, dtype=torch.float64).to(dev)
    y = (torch.randn(vis.shape, generator=g, dtype=torch.float64)
         + 1j * torch.randn(vis.shape, generator=g, dtype=torch.float64)).to(dev)
    Ax = G.dirty2ms(tu, tf, x.to(torch.float32 if prec == "mixed" else torch.float64), px, px,
                    eps, precision=prec, vis_dtype=np.complex128, **KW)
    Aty = G.ms2dirty(tu, tf, y.to(torch.complex64 if prec == "mixed" else torch.complex128),
                     nx, nx, px, px, eps, precision=prec, dirty_dtype=np.float64, **KW)
    if prec == "mixed":  # the operator saw the rounded inputs
        x = x.to(torch.float32).double()
        y = y.to(torch.complex64).to(torch.complex128)
    a = torch.vdot(y.ravel(), Ax.ravel()).real.item()
    b = torch.vdot(Aty.ravel().to(torch.complex128), x.ravel().to(torch.complex128)).real.item()
    assert abs(a - b) / (y.norm().item() * Ax.norm().item()) < tol_adj
    del x, y, Ax, Aty
    if O.ref_available():
        rp = "float" if prec == "mixed" else "double"
        dr = O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, eps, prec=rp)
        assert O.rel_rms(d, dr.astype(np.float64)) < tol_ref
        vr = O.ref_dirty2ms(uvw, freq, model.astype(fdt), px, px, eps, prec=rp, vis_dtype=cdt)
        assert O.rel_rms(v, vr.astype(np.complex128)) < tol_ref


def test_config1_fp64_full(G):
    from wsclean_b200 import synth
    c = synth.config1()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(1)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    vis = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux, device="cuda:0")
    vis = vis + 0.1 * (rng.normal(size=vis.shape) + 1j * rng.normal(size=vis.shape))
    assert vis.size == 2_903_040 and vis.dtype == np.complex128
    d = G.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-12, precision="fp64",
                   dirty_dtype=np.float64, **KW)
    pix = rng.integers(0, nx * nx, 64)
    ref = O.dft_ms2dirty(uvw, freq, vis, nx, nx, px, px, pixels=pix, negate_v=True,
                         divide_by_n=False)
    assert O.rel_rms(d.ravel()[pix], ref) < 1e-11
    if O.ref_available():
        dr = O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-12, prec="double")
        assert O.rel_rms(d, dr) < 1e-11
    model = synth.sky_image(nx, nx, ix, iy, flux)
    v = G.dirty2ms(uvw, freq, model, px, px, 1e-12, precision="fp64", vis_dtype=np.complex128,
                   **KW)
    sel = rng.choice(vis.size, 10000, replace=False)
    vref = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=True, divide_by_n=False, select=sel)
    assert O.rel_rms(v.ravel()[sel], vref) < 1e-11


def test_config3_gradient_full(G):
    from wsclean_b200 import synth
    from wsclean_b200.interface import ImagingParameters, Operator, chi2
    c = synth.config3()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(3)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    vis = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux, device="cuda:0")
    noise = rng.uniform(0.5, 2.0, vis.shape)
    w = noise * synth.briggs_weights(uvw, freq, nx, nx, px, px, robust=0.0, noise_weights=noise)
    sky = synth.sky_image(nx, nx, ix, iy, flux)
    model = sky * (1 + 0.05 * rng.normal(size=sky.shape))
    p = ImagingParameters(uvw, freq, nx, nx, px, px, epsilon=1e-10, precision="fp64")
    dev = torch.device("cuda", 0)
    V, Wt = torch.as_tensor(vis, device=dev), torch.as_tensor(w, device=dev)
    h = 1e-3
    with Operator(p) as op:
        x = torch.as_tensor(model, device=dev).requires_grad_(True)
        chi2(op, x, V, Wt).backward()
        grad = x.grad.cpu().numpy()
        # half the pixels at sources (large gradients), half at random
        src = np.flatnonzero(sky.ravel())
        pix = np.concatenate([rng.choice(src, 32, replace=False), rng.integers(0, nx * nx, 32)])
        fd = []
        for k in pix:
            e = torch.zeros(nx * nx, dtype=torch.float64, device=dev)
            e[k] = h
            e = e.reshape(nx, nx)
            with torch.no_grad():
                fd.append((chi2(op, x + e, V, Wt).item() - chi2(op, x - e, V, Wt).item()) / (2 * h))
    fd = np.array(fd)
    g = grad.ravel()[pix]
    assert np.max(np.abs(g - fd)) / np.max(np.abs(fd)) < 1e-4
    if O.ref_available():
        kw = dict(KW, prec="double")
        Ax = O.ref_dirty2ms(uvw, freq, model, px, px, 1e-10, vis_dtype=np.complex128, **kw)
        gref = -2.0 * O.ref_ms2dirty(uvw, freq, w * (vis - Ax), nx, nx, px, px, 1e-10, **kw)
        assert O.rel_rms(grad, gref) < 1e-7


@pytest.mark.parametrize("prec,eps,tol", [("mixed", 1e-5, 1e-5), ("fp64", 1e-10, 1e-9)])
def test_config4_facets(G, prec, eps, tol):
    from wsclean_b200 import synth
    c = synth.config4(scale=0.25)
    uvw, freq, px = c["uvw"], c["freq"], c["pixsize"]
    facets = synth.facets4()
    sizes = [f["nx"] * f["ny"] for f in facets]
    pick = [int(np.argmin(sizes)), int(np.argmax(sizes)), 5]
    rng = np.random.default_rng(44)
    for oc in (0, 7):
        fr = freq[8 * oc:8 * oc + 8]
        vis = (rng.normal(size=(len(uvw), 8)) + 1j * rng.normal(size=(len(uvw), 8)))
        vis = vis.astype(np.complex64 if prec == "mixed" else np.complex128)
        for fi in pick:
            f = facets[fi]
            cx, cy = f["dx"] * px, f["dy"] * px
            d = G.ms2dirty(uvw, fr, vis, f["nx"], f["ny"], px, px, eps, precision=prec,
                           center_x=cx, center_y=cy, dirty_dtype=np.float64, **KW)
            pix = rng.integers(0, f["nx"] * f["ny"], 48)
            ref = O.dft_ms2dirty(uvw, fr, vis, f["nx"], f["ny"], px, px, pixels=pix,
                                 negate_v=True, divide_by_n=False, center_x=cx, center_y=cy)
            assert O.rel_rms(d.ravel()[pix], ref) < tol, (oc, fi)
            model = np.zeros((f["nx"], f["ny"]))
            model[rng.integers(0, f["nx"], 30), rng.integers(0, f["ny"], 30)] = rng.uniform(0.1, 5, 30)
            v = G.dirty2ms(uvw, fr, model, px, px, eps, precision=prec, center_x=cx, center_y=cy,
                           vis_dtype=np.complex128, **KW)
            sel = rng.choice(v.size, 5000, replace=False)
            vref = O.dft_dirty2ms(uvw, fr, model, px, px, negate_v=True, divide_by_n=False,
                                  center_x=cx, center_y=cy, select=sel)
            assert O.rel_rms(v.ravel()[sel], vref) < tol, (oc, fi)


def test_config5_widefield_subsample(G):
    from wsclean_b200 import synth
    c = synth.config5(scale=0.02)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(5)
    nvis = uvw.shape[0] * len(freq)
    assert nvis > 10_000_000
    dev = torch.device("cuda", 0)
    vis = torch.complex(torch.randn(uvw.shape[0], len(freq), device=dev),
                        torch.randn(uvw.shape[0], len(freq), device=dev))
    d = G.ms2dirty(uvw, freq, vis, nx, nx, px, px, 1e-5, dirty_dtype=np.float64, **KW)
    pix = rng.integers(0, nx * nx, 64)
    ref = O.dft_ms2dirty(uvw, freq, vis.cpu().numpy(), nx, nx, px, px, pixels=pix,
                         negate_v=True, divide_by_n=False)
    assert O.rel_rms(d.cpu().numpy().ravel()[pix], ref) < 1e-5
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    model = synth.sky_image(nx, nx, ix, iy, flux) + synth.gaussian_blobs(nx, nx, c["ngauss"], rng)
    v = G.dirty2ms(uvw, freq, torch.as_tensor(model, device=dev), px, px, 1e-5,
                   vis_dtype=np.complex128, **KW)
    sel = rng.choice(nvis, 20000, replace=False)
    vref = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=True, divide_by_n=False, select=sel)
    assert O.rel_rms(v.cpu().numpy().ravel()[sel], vref) < 1e-5


def _config5_full():
    """The full config-5 observation in page-locked host memory, the sky
    model, and the row chunks of 256 MiB of uvw + visibilities each."""
    from wsclean_b200 import synth
    c = synth.config5()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(5)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    model = synth.sky_image(nx, nx, ix, iy, flux) + synth.gaussian_blobs(nx, nx, c["ngauss"], rng)
    nchan = len(freq)
    rows = (256 << 20) // (24 + 8 * nchan)
    bounds = list(range(0, len(uvw), rows)) + [len(uvw)]
    return c, uvw, freq, nx, px, model, rng, list(zip(bounds[:-1], bounds[1:]))


def test_config5_full_streamed(G):
    c, uvw, freq, nx, px, model, rng, parts = _config5_full()
    nrows, nchan = uvw.shape[0], len(freq)
    assert nrows * nchan == 522_240_000
    h_uvw = torch.as_tensor(uvw).pin_memory()
    h_vis = torch.empty((nrows, nchan), dtype=torch.complex64).pin_memory()
    ext = G.data_extent(uvw, freq)
    with G.Stream(freq, nx, nx, px, px, 1e-5, ext, nvis=nrows * nchan, dirty_dtype=np.float64,
                  **KW) as s:
        # dirty2ms: the visibilities of the sky model, chunk by chunk
        s.predict_begin(model)
        for a, b in parts:
            s.predict(h_uvw[a:b], vis=h_vis[a:b])
        sel = rng.choice(nrows * nchan, 20000, replace=False)
        vref = O.dft_dirty2ms(uvw, freq, model, px, px, negate_v=True, divide_by_n=False,
                              select=sel)
        vis = h_vis.numpy()
        assert O.rel_rms(vis.ravel()[sel], vref) < 1e-5
        # ms2dirty of those visibilities, streamed back in the same chunks
        for a, b in parts:
            s.add(h_uvw[a:b], h_vis[a:b])
        d = s.finish()
        st = s.stats()
    assert st["nplanes"] > 8
    # FP64 DFT of all 522M visibilities at 16 pixels (8 on sources), summed
    # over row blocks (the transform is linear in the visibilities)
    src = np.flatnonzero(model.ravel())
    pix = np.concatenate([rng.choice(src, 8, replace=False), rng.integers(0, nx * nx, 8)])
    ref = np.zeros(len(pix))
    step = 4_000_000
    for r0 in range(0, nrows, step):
        ref += O.dft_ms2dirty(uvw[r0:r0 + step], freq, vis[r0:r0 + step], nx, nx, px, px,
                              pixels=pix, negate_v=True, divide_by_n=False)
    assert O.rel_rms(d.ravel()[pix], ref) < 1e-5
