"""chi^2 gradient through the torch.autograd binding (the config-3 check at
reduced size): the config-2 array and sky at 512^2 and 32" pixels (the same
field as 2048^2 at 8"), Briggs robust=0 imaging weights times seeded U[0.5,2]
noise weights, model = true sky perturbed by 5% Gaussian noise.

* autograd gradient vs central finite differences on 64 random pixels
  (FP64 operator: h = 1e-3 Jy, tolerance 1e-6; mixed operator: the FP32
  rounding of a single evaluation needs h = 1 Jy, tolerance 1e-4 -- chi^2 is
  exactly quadratic, so any h is unbiased);
* autograd gradient vs the gradient computed with the reference w-gridder
  (-2 ms2dirty(w (V - A x)) from the compiled ducc0).  The residual V - A x
  is about 5% of the visibilities, so the operators' own accuracy epsilon
  grows to about epsilon/0.05 in the residual: 1e-8 relative RMS for the
  FP64 form (epsilon 1e-10), 1e-3 for the mixed form (epsilon 1e-5);
* the Operator's forward/backward against the raw calls, and the autograd
  pair's dot-product (adjoint) identity."""
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
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-3)])
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
    vdt = np.complex128 if precision == "fp64" else np.complex64   # ducc0's Tms for Tcalc
    Ax = O.ref_dirty2ms(uvw, freq, model, px, px, p.epsilon, vis_dtype=vdt, **kw)
    r = w * (vis - Ax)
    gref = -2.0 * O.ref_ms2dirty(uvw, freq, r.astype(np.complex128), nx, nx, px, px, p.epsilon,
                                 **dict(kw, prec="double"))
    assert O.rel_rms(grad, gref) < tol


def test_operator_matches_raw_calls_and_autograd_adjoint():
    from wsclean_b200 import gridder as G
    from wsclean_b200.interface import DirtyToVis, VisToDirty
    uvw, freq, nx, px, vis, w, model, p, Operator = setup("fp64")
    rng = np.random.default_rng(11)
    with Operator(p) as op:
        assert op.data_size() == vis.size and op.image_size() == nx * nx
        out = np.zeros(op.data_size(), dtype=np.complex128)
        op.forward(out, model.ravel())
        ref = G.dirty2ms(uvw, freq, model, px, px, p.epsilon, negate_v=True, divide_by_n=False,
                         sigma_min=1.1, sigma_max=2.0, precision="fp64",
                         vis_dtype=np.complex128)
        # atomics make the summation order (and the last bits) vary between calls
        assert O.rel_rms(out.reshape(vis.shape), ref) < 1e-12
        img = np.zeros(op.image_size())
        op.backward(img, vis.ravel())
        ref = G.ms2dirty(uvw, freq, vis, nx, nx, px, px, p.epsilon, negate_v=True,
                         divide_by_n=False, sigma_min=1.1, sigma_max=2.0, precision="fp64",
                         dirty_dtype=np.float64)
        assert O.rel_rms(img.reshape(nx, nx), ref) < 1e-12
        with pytest.raises(RuntimeError):
            op.forward(np.zeros(3, dtype=np.complex128), model.ravel())

        dev = torch.device("cuda", 0)
        x = torch.as_tensor(rng.normal(size=(nx, nx)), device=dev)
        y = torch.as_tensor(rng.normal(size=vis.shape) + 1j * rng.normal(size=vis.shape),
                            device=dev)
        lhs = torch.sum((DirtyToVis.apply(x, op) * y.conj()).real).item()
        rhs = torch.sum(x * VisToDirty.apply(y, op)).item()
        assert abs(lhs - rhs) / abs(rhs) < 1e-10

        # backward of VisToDirty is the forward operator
        y.requires_grad_(True)
        gx = torch.as_tensor(rng.normal(size=(nx, nx)), device=dev)
        torch.sum(VisToDirty.apply(y, op) * gx).backward()
        fwd = DirtyToVis.apply(gx, op)
        assert torch.allclose(y.grad, fwd, rtol=0, atol=1e-12 * fwd.abs().max().item())
    with pytest.raises(RuntimeError):
        op.forward(out, model.ravel())
