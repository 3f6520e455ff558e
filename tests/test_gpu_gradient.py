"""chi^2 gradient through the torch.autograd binding (the config-3 check at
reduced size): the config-2 array and sky at 512^2 and 32" pixels (the same
field as 2048^2 at 8"), Briggs robust=0 imaging weights times seeded U[0.5,2]
noise weights, model = true sky perturbed by 5% Gaussian noise.

* autograd gradient vs central finite differences on 64 random pixels
  (FP64 operator: h = 1e-3 Jy, tolerance 1e-6; mixed operator: the FP32
  rounding of a single evaluation needs h = 1 Jy, tolerance 1e-4 -- chi^2 is
  exactly quadratic, so any h is unbiased);
* autograd gradient vs the gradient computed with the reference w-gridder
  (-2 ms2dirty(w (V - A x)) from the compiled ducc0)."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def setup(precision):
    from wsclean_b200 import synth
    from wsclean_b200.interface import ImagingParameters, Operator
    c = synth.config2(scale=0.05, npix=512, pixsize_arcsec=32.0)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(3)
    ix, iy, flux = synth.point_sky(200, nx, nx, rng)
    vis = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux)
    noise = rng.uniform(0.5, 2.0, vis.shape)
    wimg = synth.briggs_weights(uvw, freq, nx, nx, px, px, robust=0.0, noise_weights=noise)
    w = noise * wimg
    sky = synth.sky_image(nx, nx, ix, iy, flux)
    model = sky * (1 + 0.05 * rng.normal(size=sky.shape)) * (sky != 0)
    eps = 1e-5 if precision == "mixed" else 1e-10
    p = ImagingParameters(uvw, freq, nx, nx, px, px, epsilon=eps, precision=precision)
    return uvw, freq, nx, px, vis, w, model, p, Operator


@pytest.mark.parametrize("precision,h,tol", [("fp64", 1e-3, 1e-6), ("mixed", 1.0, 1e-4)])
def test_chi2_gradient_vs_finite_differences(precision, h, tol):
    from wsclean_b200.interface import chi2
    uvw, freq, nx, px, vis, w, model, p, Operator = setup(precision)
    dev = torch.device("cuda", 0)
    V = torch.as_tensor(vis, device=dev)
    Wt = torch.as_tensor(w, device=dev)
    with Operator(p) as op:
        x = torch.as_tensor(model, device=dev).requires_grad_(True)
        f = chi2(op, x, V, Wt)
        f.backward()
        grad = x.grad.cpu().numpy()
        rng = np.random.default_rng(9)
        pix = rng.integers(0, nx * nx, 64)
        fd = []
        for k in pix:
            e = torch.zeros(nx * nx, dtype=torch.float64, device=dev)
            e[k] = h
            e = e.reshape(nx, nx)
            with torch.no_grad():
                fp = chi2(op, x + e, V, Wt).item()
                fm = chi2(op, x - e, V, Wt).item()
            fd.append((fp - fm) / (2 * h))
    fd = np.array(fd)
    g = grad.ravel()[pix]
    assert np.max(np.abs(g - fd)) / np.max(np.abs(fd)) < tol


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-4)])
def test_chi2_gradient_vs_reference(precision, tol):
    from wsclean_b200.interface import chi2
    uvw, freq, nx, px, vis, w, model, p, Operator = setup(precision)
    dev = torch.device("cuda", 0)
    with Operator(p) as op:
        x = torch.as_tensor(model, device=dev).requires_grad_(True)
        chi2(op, x, torch.as_tensor(vis, device=dev), torch.as_tensor(w, device=dev)).backward()
        grad = x.grad.cpu().numpy()
    prec = "double" if precision == "fp64" else "float"
    kw = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0, prec=prec)
    Ax = O.ref_dirty2ms(uvw, freq, model, px, px, p.epsilon, vis_dtype=np.complex128, **kw)
    r = w * (vis - Ax)
    gref = -2.0 * O.ref_ms2dirty(uvw, freq, r.astype(np.complex128), nx, nx, px, px, p.epsilon,
                                 **dict(kw, prec="double" if precision == "fp64" else "double"))
    assert O.rel_rms(grad, gref) < tol
